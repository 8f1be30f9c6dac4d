#!/usr/bin/env python
"""Benchmark of the B200 AWP-ODC-SGT stepper (Gcell-updates/s).

Workload: the batched fx+fy+fz SGT solve on a 400x400x200 grid (h = 100 m,
dt = 0.005 s, 4000 source steps, 5000 SGT points every 10 steps), seeded
layered medium with 5 % Gaussian-correlated perturbations (synthetic data; no
public dataset is involved).

  value   device-resident throughput: one bench step = one SGT sample period
          (NTISKP_SGT = 10 time steps of all components plus the SGT gather),
          state already in HBM (5.8 GB, far larger than the 126 MB L2).
  e2e     the same metric through the C ABI with host buffers: every e2e step
          is one complete SGT job (create, media/source/points host->device,
          4001 time steps, SGT file images device->host, destroy).
  roofline  dominant kernel: algorithmic bytes per launch / CUDA-event time of
          one launch on the solver's stream, against MEASURED_PEAKS.json.
  cpu_baseline  the FP32 CPU oracle (restatement of the Fortran, OpenMP over
          all host cores) on a bounded sample of the same grid.

Multi-GPU (torchrun, one process per GPU): every rank runs its own SGT job
(independent components/requests, no data-path collective); value = all
ranks' cell-updates / max-over-ranks time; scaling "weak".

--impl reference: the reference's CPU path (the FP32 oracle; the Fortran/MPI
reference cannot be built in this image) on rank 0, all host threads, one
time step of one component of the same grid per bench step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cybershake-core_b200"))

import numpy as np  # noqa: E402

import awp_inputs as ai  # noqa: E402

METRIC = "Gcell-updates/s"
CONFIG_N = 2


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    if n_gpus <= 1 or "RANK" not in os.environ:
        return None, 0, 1, 0
    import torch.distributed as dist
    import datetime
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = "nccl"
    import torch
    torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600),
                            device_id=torch.device("cuda", local))
    return dist, rank, world, local


def barrier(dist):
    if dist is not None:
        dist.barrier()


def _reduce(dist, x, local, op):
    import torch
    dev = "cuda:%d" % local if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, x, local):
    if dist is None:
        return x
    return _reduce(dist, x, local, dist.ReduceOp.MAX)


def aggregate(dist, units, seconds, local):
    """Whole-job throughput of independent per-rank jobs: all ranks' units
    divided by the slowest rank's time (weak scaling, no data-path
    collective)."""
    if dist is None:
        return units / seconds, units, seconds
    tot = _reduce(dist, units, local, dist.ReduceOp.SUM)
    mx = _reduce(dist, seconds, local, dist.ReduceOp.MAX)
    return tot / mx, tot, mx


def shard_jobs(jobs, rank, world):
    """Independent SGT jobs (components or requests) dealt round-robin to
    ranks."""
    return [j for n, j in enumerate(jobs) if n % world == rank]


def workload(args=None):
    """The config-2 job, or a reduced grid / component set for small profiling
    captures (--grid, --components); the name records any change."""
    w = ai.config(CONFIG_N)
    if args is None:
        return w
    import dataclasses
    if args.grid:
        nx, ny, nz = (int(v) for v in args.grid.split(","))
        w = dataclasses.replace(w, name="layered_%dx%dx%d" % (nx, ny, nz), nx=nx, ny=ny, nz=nz,
                                src_xyz=(nx // 2, ny // 2, min(21, nz)), npts=min(w.npts, nx * ny // 4))
    if args.components:
        w = dataclasses.replace(w, name=w.name + "_c%d" % args.components, igreen=w.igreen[:args.components])
    return w


def solver_params(w, device, precision="f32", kernel="auto"):
    import awpsgt
    return awpsgt.make_params(w.nx, w.ny, w.nz, w.dh, w.dt, w.nt, nst=w.nst, igreen=w.igreen, nd=20,
                              arbc=0.92, fl=w.fl, fh=w.fh, fp=w.fp, socalq=w.socalq, ntiskp_sgt=w.ntiskp_sgt,
                              write_step=w.nst // w.ntiskp_sgt, precision=precision, kernel=kernel,
                              device=device)


def make_solver(w, media, pts, stfs, device, precision="f32", kernel="auto"):
    import awpsgt
    s = awpsgt.Solver(solver_params(w, device, precision, kernel))
    s.load_media(media)
    for q in range(len(w.igreen)):
        s.set_source(q, [w.src_xyz], stfs[q])
    s.set_points(pts)
    return s


def cpu_oracle_rate(w, media, stf, nsteps, warm=1):
    """FP32 oracle, one component, all host threads: cell-updates/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.Oracle(nx=w.nx, ny=w.ny, nz=w.nz, dh=w.dh, dt=w.dt, nt=w.nt, nst=w.nst, nd=20, arbc=0.92,
                      fl=w.fl, fh=w.fh, fp=w.fp, socalq=w.socalq, ntiskp_sgt=w.ntiskp_sgt,
                      write_step=w.nst // w.ntiskp_sgt, igreen=w.igreen[0], precision="f32")
    o.load_media(media)
    o.set_source([w.src_xyz], stf)
    o.set_points(w.points())
    o.run(warm)
    times = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        o.run(1)
        times.append(time.perf_counter() - t0)
    cells = w.nx * w.ny * w.nz
    threads = oracle.threads()
    o.close()
    return cells / statistics.median(times), threads, times


def run_reference(args):
    """--impl reference: the CPU path on the host cores, rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    w = workload(args)
    media = w.media()
    stf = w.stf(0)
    rate, threads, times = cpu_oracle_rate(w, media, stf, nsteps=max(args.steps, 1), warm=max(args.warmup, 1))
    value = rate * 1e-9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": statistics.median(times) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded layered medium, splitmix64 points)",
        "config": {"workload": w.name + " (one component per reference step)", "grid": [w.nx, w.ny, w.nz],
                   "steps_per_solve": w.nt},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": "%d time steps of one component on the %dx%dx%d grid (FP32 oracle, "
                                   "OpenMP %d threads)" % (args.steps, w.nx, w.ny, w.nz, threads)},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--precision", default="f32")
    ap.add_argument("--kernel", default="auto")
    ap.add_argument("--e2e-solves", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--grid", default="", help="nx,ny,nz: reduced grid for profiling captures")
    ap.add_argument("--components", type=int, default=0, help="first n of the fx, fy, fz components")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    dist, rank, world, local = dist_setup(args.gpus)
    import awpsgt
    w = workload(args)
    media = w.media()
    pts = w.points()
    stfs = [w.stf(q) for q in range(len(w.igreen))]
    ncomp = len(w.igreen)
    cells = w.nx * w.ny * w.nz
    per_step_ts = w.ntiskp_sgt                      # time steps per bench step
    steps_needed = (args.warmup + args.steps) * per_step_ts + 40
    assert steps_needed <= w.nt, "too many bench steps for one solve"

    # ---------------- device-resident throughput ----------------
    s = make_solver(w, media, pts, stfs, local, args.precision, args.kernel)
    s.run(args.warmup * per_step_ts)
    barrier(dist)
    with ClockSampler(local) as clk:
        st0 = s.stats()
        s.run(args.steps * per_step_ts)
        st1 = s.stats()
    barrier(dist)
    dev_s = st1.seconds_loop - st0.seconds_loop
    rate, updates, dev_s = aggregate(dist, float(cells * ncomp * per_step_ts * args.steps), dev_s, local)
    value = rate * 1e-9
    ms_per_step = dev_s / args.steps * 1e3

    # per-kernel CUDA-event times (same solver, same stream, right after)
    prof = s.profile(2 * per_step_ts)
    bpcu = awpsgt.bytes_per_cell_update(s.p)
    s.close()

    # ---------------- end to end through the C ABI ----------------
    e2e_vals, h2d, d2h = [], 0, 0
    media_pinned = media
    try:
        import torch
        mt = torch.from_numpy(media).pin_memory()
        media_pinned = mt.numpy()
    except Exception:
        pass
    for it in range(0 if args.no_e2e else 1 + args.e2e_solves):
        barrier(dist)
        t0 = time.perf_counter()
        s = make_solver(w, media_pinned, pts, stfs, local, args.precision, args.kernel)
        out = s.run(w.nt, with_sgt=True)
        s.close()
        el = time.perf_counter() - t0
        el = max_over_ranks(dist, el, local)
        if it > 0:
            e2e_vals.append(cells * ncomp * w.nt * world / el * 1e-9)
        h2d = media.nbytes + sum(x.nbytes for x in stfs) + pts.nbytes
        d2h = out.nbytes
    e2e = None
    if e2e_vals:
        e2e = {"value": statistics.median(e2e_vals), "unit": METRIC, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "step": "one complete SGT job: %d time steps x %d components" % (w.nt, ncomp)}

    # ---------------- roofline of the dominant kernel ----------------
    peak, peak_kind = peaks()
    dom = max((k for k in prof if prof[k]["launches"] and prof[k]["bytes"] > 0), key=lambda k: prof[k]["ms"] * prof[k]["launches"])
    ach = prof[dom]["bytes"] / (prof[dom]["ms"] * 1e-3) / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get("%s:%s" % (w.name, dom))
    except Exception:
        pass
    step_bytes = bpcu * cells * ncomp
    roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "traffic": traffic,
                "bytes_per_launch": prof[dom]["bytes"], "ms_per_launch": prof[dom]["ms"],
                "step_frac": (step_bytes * value * 1e9 / (cells * ncomp * world)) / 1e9 / peak,
                "bytes_per_cell_update": bpcu}

    launches_per_ts = 2 if "k_fused" in prof else 4    # stepper kernel(s) + k_post
    gpu_launches = args.steps * (per_step_ts * launches_per_ts + 1)

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision == "f32" else "f32+%s" % args.precision,
        "data": "synthetic (seeded layered medium + 5% correlated perturbation, splitmix64 points)",
        "config": {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "components": list(w.igreen),
                   "time_steps_per_bench_step": per_step_ts, "sgt_points": int(pts.shape[0]),
                   "precision": args.precision, "l2": "inputs larger than L2 (%.1f GB state)" % (
                       s.p.nx * s.p.ny * s.p.nz * 4 * (15 * ncomp + 5) / 1e9),
                   "parallelism": "independent SGT jobs, one per GPU" if world > 1 else "single GPU"},
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "kernels": prof,
    }
    if rank == 0:
        line["clocks"] = clk.summary()
        if not args.no_cpu and world == 1:
            rate, threads, times = cpu_oracle_rate(w, media, stfs[0], nsteps=3)
            line["cpu_baseline"] = {"value": rate * 1e-9, "unit": METRIC, "cores": threads, "kind": "port",
                                    "sample": "3 time steps of one component on the %dx%dx%d grid (FP32 "
                                              "oracle, OpenMP)" % (w.nx, w.ny, w.nz)}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
