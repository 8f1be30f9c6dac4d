#!/usr/bin/env python
"""Benchmark of the B200 AWP-ODC-SGT stepper (Gcell-updates/s), default
TMA-staged two-sweep kernels (k_vel_tma, k_fsvel, k_str_tma).

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

Other modes: --config N (workloads 1-4), --grid / --components (reduced
grids for profiling captures), --serve (the 64-request serving stream:
p50/p99 latency and throughput against serial solves), --synth (the
reciprocity synthesis of 64 rupture variations against a resident SGT set).
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

    def power_w(self):
        w = []
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                w.append(float(f[3]))
            except (IndexError, ValueError):
                pass
        return statistics.median(w) if w else None


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
    w = ai.config(args.config if args is not None and args.config else CONFIG_N)
    if args is None:
        return w
    import dataclasses
    if args.grid:
        nx, ny, nz = (int(v) for v in args.grid.split(","))
        w = dataclasses.replace(w, name="layered_%dx%dx%d" % (nx, ny, nz), nx=nx, ny=ny, nz=nz,
                                src_xyz=(nx // 2, ny // 2, min(21, nz)), npts=min(w.npts, nx * ny // 4))
    if args.components:
        w = dataclasses.replace(w, name=w.name + "_c%d" % args.components, igreen=w.igreen[:args.components])
    if getattr(args, "npc", 0):
        w = dataclasses.replace(w, name=w.name + "_pml")
    return w


def boundary(w):
    """NPC of a workload: 1 (PML) when its name says so, else 0 (Cerjan)."""
    return 1 if w.name.endswith("_pml") else 0


def solver_params(w, device, precision="f32", kernel="auto"):
    import awpsgt
    return awpsgt.make_params(w.nx, w.ny, w.nz, w.dh, w.dt, w.nt, nst=w.nst, igreen=w.igreen, nd=20,
                              arbc=0.92, fl=w.fl, fh=w.fh, fp=w.fp, socalq=w.socalq, ntiskp_sgt=w.ntiskp_sgt,
                              write_step=w.nst // w.ntiskp_sgt, precision=precision, kernel=kernel,
                              device=device, npc=boundary(w))


def make_solver(w, media, pts, stfs, device, precision="f32", kernel="auto", tuning=None):
    import awpsgt
    s = awpsgt.Solver(solver_params(w, device, precision, kernel))
    if tuning is not None:
        s.set_tuning(tuning)
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


def run_job_profile(args):
    """Step time, median SM clock and board power over one complete job, chunk by
    chunk; then the same solver with its wavefield zeroed, for comparison."""
    w = workload(args)
    media, pts = w.media(), w.points()
    stfs = [w.stf(q) for q in range(len(w.igreen))]
    s = make_solver(w, media, pts, stfs, 0, args.precision, args.kernel)

    def chunk(n, tag):
        with ClockSampler(0) as clk:
            a = s.stats()
            s.run(n)
            b = s.stats()
        c = clk.summary()
        line = {"workload": w.name, "chunk": tag, "steps": [int(a.steps_done), int(b.steps_done)],
                "ms_per_step": (b.seconds_loop - a.seconds_loop) / n * 1e3, "sm_mhz": c["sm_mhz"],
                "power_w": clk.power_w(), "reasons": c["reasons"]}
        print(json.dumps(line), flush=True)

    n = args.job_profile
    done = 0
    while done < w.nt:
        k = min(n, w.nt - done)
        chunk(k, "job")
        done += k
    s.reset()
    chunk(n, "zeroed wavefield")
    s.close()
    return 0


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


# ---------------------------------------------------------------------------
# serving stream (--serve): continuous batching against serial solves
# ---------------------------------------------------------------------------

def serve_requests(n, seed, nst_scale):
    """n request specs: sizes log-uniform 100x100x50 .. 500x500x250, DH 100-200,
    NST 1000-4000 (times nst_scale), a random non-empty component set, media
    seeded per request; Poisson arrivals are drawn later from the measured
    serial service rate."""
    rng = np.random.default_rng(seed)
    specs = []
    for r in range(n):
        f = float(np.exp(rng.uniform(0.0, np.log(5.0))))
        nx = ny = int(round(100 * f))
        nz = int(round(50 * f))
        dh = float(rng.choice([100.0, 150.0, 200.0]))
        nst = max(20, int(round(int(rng.integers(1000, 4001)) * nst_scale)))
        comps = [c for c in (1, 2, 3) if rng.random() < 0.5] or [int(rng.integers(1, 4))]
        specs.append({"id": r, "nx": nx, "ny": ny, "nz": nz, "dh": dh, "nst": nst, "igreen": tuple(comps),
                      "seed": 1000 + r})
    return specs


def build_request(sp):
    """Host inputs of one request (media, sources, points) and its params."""
    import awpsgt
    nx, ny, nz, dh, nst = sp["nx"], sp["ny"], sp["nz"], sp["dh"], sp["nst"]
    media = ai.layered_media(nx, ny, nz, dh, seed=sp["seed"], pert_std=0.05, corr_len=20 * dh)
    dt = ai.stable_dt(media, dh, 0.35)
    nt = nst + 1
    p = awpsgt.make_params(nx, ny, nz, dh, dt, nt, nst=nst, igreen=sp["igreen"], nd=20, arbc=0.92, socalq=1,
                           ntiskp_sgt=10, write_step=max(1, nt // 10))
    src = (nx // 2, ny // 2, max(1, min(nz, int(round(2000.0 / dh)) + 1)))
    sources = [([src], ai.gaussian_derivative_stf(nst, dt, f0=0.5, column=c - 1)) for c in sp["igreen"]]
    pts = ai.sgt_points(nx, ny, min(nz, int(10000.0 / dh) + 1), 1000, seed=sp["seed"])
    return p, media, sources, pts


def pct(x, q):
    return float(np.percentile(np.asarray(x, dtype=np.float64), q)) if len(x) else None


def run_serve(args):
    print(json.dumps(serve_stream(args.serve_requests, args.serve_nst_scale, args.serve_load, args.serve_active,
                                  args.serve_policy, args.serve_fill)))
    return 0


def serve_stream(n_requests, nst_scale, load, active, policy, fill):
    """Serial solves (one at a time) give the service times; the same requests
    then arrive as a Poisson stream at `load` times the serial service rate
    and go through the continuous-batching server.  Latency = completion
    minus arrival.  The serial latencies are those of a FIFO single server fed
    the same arrival times with the measured service times."""
    import queue
    import awpsgt
    specs = serve_requests(n_requests, 1, nst_scale)
    work = [sp["nx"] * sp["ny"] * sp["nz"] * len(sp["igreen"]) * (sp["nst"] + 1) for sp in specs]

    def producer(out_q):
        for sp in specs:
            out_q.put(build_request(sp))

    # serial solves
    q1 = queue.Queue(maxsize=2)
    th = threading.Thread(target=producer, args=(q1,), daemon=True)
    th.start()
    service = []
    for sp in specs:
        p, media, sources, pts = q1.get()
        t0 = time.perf_counter()
        with awpsgt.Solver(p) as s:
            s.load_media(media)
            for qq, (xyz, stf) in enumerate(sources):
                s.set_source(qq, xyz, stf)
            s.set_points(pts)
            s.run(p.nt, with_sgt=True)
        service.append(time.perf_counter() - t0)
    th.join()
    total_serial = float(sum(service))
    rate = load * len(specs) / total_serial
    arr = np.cumsum(np.random.default_rng(1).exponential(1.0 / rate, size=len(specs)))
    arr -= arr[0]
    free_at, serial_lat = 0.0, []
    for a, sv in zip(arr, service):
        start = max(a, free_at)
        free_at = start + sv
        serial_lat.append(free_at - a)

    # served stream: every request's host inputs are built before the stream
    # starts (about 10 GB for 64 requests), as the serial pass excludes their
    # building from its service times; built on the fly they made the
    # submitter fall behind the arrival schedule
    reqs = [build_request(sp) for sp in specs]
    lat, ids, late = [], [], []
    with awpsgt.Server(device=0, max_active=active, chunk_steps=10) as sv:
        sv.configure(policy, fill, 0.0)
        t_start = sv.time()
        for k, sp in enumerate(specs):
            req = reqs[k]
            while sv.time() - t_start < arr[k]:
                time.sleep(0.0005)
            ids.append(sv.submit(*req))
            late.append(sv.time() - t_start - arr[k])
        t_sub = {}
        for rid in ids:
            info, _ = sv.wait(rid, timeout=7200)
            if awpsgt.REQ_STATE[info["state"]] != "done":
                raise RuntimeError("request %d: %s" % (rid, info))
            t_sub[rid] = info
        t_end = max(i["t_done"] for i in t_sub.values())
    del reqs
    for k, rid in enumerate(ids):
        lat.append(t_sub[rid]["t_done"] - (t_start + arr[k]))
    span = t_end - t_start
    line = {
        "metric": "served-solve latency p50/p99", "value": pct(lat, 50), "unit": "s", "higher_is_better": False,
        "n_gpus": 1, "p50_s": pct(lat, 50), "p99_s": pct(lat, 99),
        "throughput": {"value": sum(work) / span * 1e-9, "unit": METRIC, "span_s": span},
        "serial": {"p50_s": pct(serial_lat, 50), "p99_s": pct(serial_lat, 99),
                   "throughput": {"value": sum(work) / total_serial * 1e-9, "unit": METRIC,
                                  "busy_s": total_serial}},
        "offered_load": load, "arrival_rate_per_s": rate, "requests": len(specs),
        "max_submit_lateness_s": float(max(late)),
        "max_active": active, "policy": policy, "dtype": "f32", "data": "synthetic (seeded layered media, seeded arrivals)",
        "config": {"workload": "serving stream: %d requests, sizes 100x100x50..500x500x250, NST 1000-4000 x %g"
                               % (len(specs), nst_scale), "cell_updates": int(sum(work))},
    }
    return line


def synth_workload():
    """The synthesis benchmark case: one site, one rupture of 64 x 32 points
    at 1 km (2048 points, 5 % of them off the SGT grid), 64 rupture
    variations, two SGT components of 2000 samples at 0.1 s, 3000 output
    samples, slip rates of 20-80 samples."""
    return ai.synth_case(seed=1, nx_f=64, nz_f=32, nt=2000, nv=64, ntout=3000, ncomp=2, nstf=(20, 80),
                         drop_frac=0.05)


def fp32_mac_peak(sm_mhz):
    """FP32 multiply-add pairs per second without FMA contraction: 148 SMs x
    128 lanes, one FMUL and one FADD per multiply-add, at the sampled clock."""
    return 148 * 128 * (sm_mhz or 1965.0) * 1e6 / 2.0


def run_synth(args):
    """Reciprocity synthesis (DirectSynth's worker step): rupture variations
    per second for one site.  A step synthesises every variation of the
    rupture against the SGT set resident in HBM (host set-up of the terms
    included); an e2e step adds the variations' hand-over from host memory
    and the seismogram read-back through the C ABI, and the SGT upload (once
    per site) is reported beside it."""
    import awpsgt
    c = synth_workload()
    nv, npts = len(c.variations), len(c.variations[0][0])
    with awpsgt.Synth(c.slon, c.slat, c.dtout, ntout=c.ntout) as s:
        s.set_sgt(c.master, c.index, c.headers, c.comps)
        for i, (p, q) in enumerate(c.variations):
            s.add_variation(i, p, q)
        for _ in range(max(3, args.warmup)):
            s.run()
        dev, conv, plan, wall, gf = [], [], [], [], []
        with ClockSampler(0) as clk:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                awpsgt._check(s.lib.awp_synth_run(s.h))
                wall.append(time.perf_counter() - t0)
                i = s.info()
                dev.append(i.seconds_device)
                conv.append(i.seconds_conv)
                gf.append(i.seconds_gf)
                plan.append(i.seconds_plan)
        info = s.info()
    clocks = clk.summary()
    t_step = statistics.median(wall)
    macs = info.macs
    e2e = None
    if not args.no_e2e:
        # a site's SGT set is uploaded once and serves every rupture of the
        # site (DirectSynth reads it once per site); an e2e step is one
        # rupture through the C ABI: its variations in from host memory, the
        # synthesis, the seismograms out to host memory
        t0 = time.perf_counter()
        s2 = awpsgt.Synth(c.slon, c.slat, c.dtout, ntout=c.ntout)
        s2.set_sgt(c.master, c.index, c.headers, c.comps)
        site_s = time.perf_counter() - t0
        ts = []
        for it in range(1 + max(3, args.steps // 2)):
            t0 = time.perf_counter()
            s2.clear_variations()
            for i2, (p, q) in enumerate(c.variations):
                s2.add_variation(i2, p, q, borrow=True)
            out = s2.run()
            if it:
                ts.append(time.perf_counter() - t0)
        s2.close()
        sgt_bytes = sum(x.nbytes for x in c.comps) + c.headers.nbytes + c.index.nbytes
        e2e = {"value": nv / statistics.median(ts), "unit": "rupture variations/s",
               "h2d_bytes_per_step": int(sum(p.nbytes + q.nbytes for p, q in c.variations)),
               "d2h_bytes_per_step": int(out.nbytes),
               "step": "one rupture: %d variations host->device, synthesis, seismograms device->host; "
                       "SGT set resident" % nv,
               "site_setup": {"seconds": site_s, "sgt_bytes_h2d": int(sgt_bytes),
                              "note": "SGT set upload, once per site"}}
    cpu = None
    if not args.no_cpu:
        # DirectSynth's own synthesis functions (built from the reference
        # sources into oracle/_ref by oracle/Makefile.ref) where present,
        # else the oracle's restatement of them; one host thread, as one
        # DirectSynth worker rank runs
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        sample = c.variations[:2]
        t0 = time.perf_counter()
        ref = oracle.synth_reference(c.master, c.index, c.headers, c.comps, c.slon, c.slat, c.dtout, c.ntout, 0.0,
                                     sample)
        kind = "reference"
        if ref is None:
            t0 = time.perf_counter()
            oracle.synth(c.master, c.index, c.headers, c.comps, c.slon, c.slat, c.dtout, c.ntout, 0.0, sample)
            kind = "port"
        dt_cpu = time.perf_counter() - t0
        cpu = {"value": len(sample) / dt_cpu, "unit": "rupture variations/s", "cores": 1, "kind": kind,
               "sample": "2 of the 64 variations, all 2048 points, one host thread (one DirectSynth worker)"}
    conv_s = statistics.median(conv)
    peak = fp32_mac_peak(clocks.get("sm_mhz"))
    line = {
        "metric": "rupture variations/s", "value": nv / t_step, "unit": "rupture variations/s",
        "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": max(3, args.warmup),
        "ms_per_step": t_step * 1e3, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded SGTs and rupture variations)",
        "config": {"workload": "reciprocity synthesis: 1 site, %d-point rupture, %d variations, 2-component SGT "
                               "nt=2000, ntout=3000" % (npts, nv), "terms": int(info.terms),
                   "non_exact_points": int(info.non_exact), "sgt_points": int(info.nsgt_points)},
        "device_ms_per_step": statistics.median(dev) * 1e3, "plan_ms_per_step": statistics.median(plan) * 1e3,
        "k_synth_gf_ms": statistics.median(gf) * 1e3, "k_synth_conv_ms": conv_s * 1e3,
        "roofline": {"bound": "fp32", "kernel": "k_synth_conv", "achieved": macs / conv_s * 1e-9, "peak": peak * 1e-9,
                     "unit": "GMAC/s", "frac": macs / conv_s / peak, "traffic": None,
                     "note": "peak = 148 SMs x 128 lanes x sampled SM clock / 2 (FMUL + FADD per multiply-add)"},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(info.gpu_launches), "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


def window_rate(w, media, pts, stfs, device, precision, kernel, tuning, prefill, warm_ts, timed_ts):
    """Device-resident rate of one stepper / storage mode over the same window
    of the job as the headline measurement: Gcell-updates/s, the dominant
    kernel's roofline fraction and the clocks seen."""
    import awpsgt
    s = make_solver(w, media, pts, stfs, device, precision, kernel, tuning if kernel == "auto" else None)
    s.run(prefill + warm_ts)
    with ClockSampler(device) as clk:
        st0 = s.stats()
        s.run(timed_ts)
        st1 = s.stats()
    prof = s.profile(w.ntiskp_sgt)
    bpcu = awpsgt.bytes_per_cell_update(s.p)
    s.close()
    peak, _ = peaks()
    dom = max((k for k in prof if prof[k]["launches"] and prof[k]["bytes"] > 0),
              key=lambda k: prof[k]["ms"] * prof[k]["launches"])
    cells = w.nx * w.ny * w.nz * len(w.igreen)
    return {"value": cells * timed_ts / (st1.seconds_loop - st0.seconds_loop) * 1e-9, "unit": METRIC,
            "precision": precision, "kernel": kernel, "bytes_per_cell_update": bpcu,
            "dominant_kernel": dom, "frac": prof[dom]["bytes"] / (prof[dom]["ms"] * 1e-3) / 1e9 / peak,
            "clocks": clk.summary()}


def precision_study():
    """Measured SGT errors of the storage modes against the FP64 oracle
    (profiles/precision.json, written by tests/test_precision_study.py)."""
    try:
        with open(os.path.join(ROOT, "profiles", "precision.json")) as f:
            return json.load(f)
    except Exception:
        return None


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
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the plain-FP32 and block-floating-point windows, the error check and the short "
                         "serving stream of the 1-GPU line")
    ap.add_argument("--config", type=int, default=0, help="workload 1..4 (default 2: 400x400x200 fx+fy+fz)")
    ap.add_argument("--grid", default="", help="nx,ny,nz: reduced grid for profiling captures")
    ap.add_argument("--components", type=int, default=0, help="first n of the fx, fy, fz components")
    ap.add_argument("--npc", type=int, default=0, choices=[0, 1], help="absorbing boundary: 0 Cerjan, 1 PML")
    ap.add_argument("--serve", action="store_true", help="serving stream: p50/p99 latency against serial solves")
    ap.add_argument("--serve-requests", type=int, default=64)
    ap.add_argument("--serve-load", type=float, default=1.2, help="offered load / serial service rate")
    ap.add_argument("--serve-active", type=int, default=4, help="requests on the GPU at once")
    ap.add_argument("--serve-nst-scale", type=float, default=1.0, help="scales every request's NST")
    ap.add_argument("--serve-policy", default="fifo", choices=["fifo", "sjf", "fifo_srpt"],
                    help="admission order (fifo_srpt: arrival order, double SM share for the least remaining work)")
    ap.add_argument("--serve-fill", type=float, default=0.0, help="resident cells x components that fill the GPU")
    ap.add_argument("--synth", action="store_true", help="reciprocity synthesis: rupture variations per second")
    ap.add_argument("--autotune", action="store_true", help="time launch shapes on this grid first (untimed)")
    ap.add_argument("--prefill", type=int, default=-1, metavar="STEPS",
                    help="untimed time steps before the warm-up (default: half the job; 0 for short profiling runs)")
    ap.add_argument("--job-profile", type=int, default=0, metavar="STEPS",
                    help="one complete job in chunks of STEPS time steps: step time, SM clock and power per chunk")
    ap.add_argument("--tune-cache", default="", help="autotuner cache file")
    ap.add_argument("--tune-steps", type=int, default=20, help="time steps per autotuner trial")
    args = ap.parse_args()
    if args.serve:
        return run_serve(args)
    if args.synth:
        return run_synth(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.job_profile:
        return run_job_profile(args)

    dist, rank, world, local = dist_setup(args.gpus)
    import awpsgt
    w = workload(args)
    # one complete SGT job per site; the sites are dealt to the ranks (one
    # each here: weak scaling, no data-path collective).  Site k differs from
    # the others by its seeded SGT points.
    sites = shard_jobs(list(range(world)), rank, world)
    site = sites[0]
    media = w.media()
    zmax = min(w.nz, max(1, int(round(10000.0 / w.dh)) + 1))
    pts = ai.sgt_points(w.nx, w.ny, zmax, w.npts, seed=site)
    stfs = [w.stf(q) for q in range(len(w.igreen))]
    ncomp = len(w.igreen)
    cells = w.nx * w.ny * w.nz
    per_step_ts = w.ntiskp_sgt                      # time steps per bench step
    steps_needed = (args.warmup + args.steps) * per_step_ts + 40
    assert steps_needed <= w.nt, "too many bench steps for one solve"
    # The timed window sits in the middle of the job, where the wavefield has
    # spread over the grid: a mostly-zero early wavefield draws less power, so
    # under the 1 kW cap its clocks (and step rate) run about 13 % above the
    # rest of the job.
    prefill = min(w.nt // 2, w.nt - steps_needed) // per_step_ts * per_step_ts
    if args.prefill >= 0:
        prefill = min(args.prefill, w.nt - steps_needed) // per_step_ts * per_step_ts

    # ---------------- launch shapes (untimed) ----------------
    tuning, tune_info = None, None
    if args.autotune:
        t0 = time.perf_counter()
        tuning, trial_rate = awpsgt.autotune(solver_params(w, local, args.precision, args.kernel), media,
                                             trial_steps=args.tune_steps, cache=args.tune_cache or None)
        tune_info = {"trial_gcell_per_s": trial_rate, "seconds": time.perf_counter() - t0,
                     "trial_steps": args.tune_steps}

    # ---------------- device-resident throughput ----------------
    s = make_solver(w, media, pts, stfs, local, args.precision, args.kernel, tuning)
    used_tuning = s.tuning().as_dict()
    s.run(prefill)
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
    e2e_vals, job_dev, h2d, d2h = [], [], 0, 0
    media_pinned = media
    if not args.no_e2e:
        try:
            import torch
            mt = torch.from_numpy(media).pin_memory()
            media_pinned = mt.numpy()
        except Exception:
            pass
    for it in range(0 if args.no_e2e else 1 + args.e2e_solves):
        barrier(dist)
        t0 = time.perf_counter()
        s = make_solver(w, media_pinned, pts, stfs, local, args.precision, args.kernel, tuning)
        out = s.run(w.nt, with_sgt=True)
        job_dev.append(s.stats().seconds_loop)
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
               "step": "one complete SGT job: %d time steps x %d components" % (w.nt, ncomp),
               "whole_job_device": cells * ncomp * w.nt / statistics.median(job_dev[1:]) * 1e-9}

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

    launches_per_ts = (2 if "k_fused" in prof else 4) + 2 * boundary(w)   # stepper kernel(s) + k_post (+ PML)
    gpu_launches = args.steps * (per_step_ts * launches_per_ts + 1)

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision == "f32" else "f32+%s" % args.precision,
        "data": "synthetic (seeded layered medium + 5% correlated perturbation, splitmix64 points)",
        "config": {"workload": w.name, "grid": [w.nx, w.ny, w.nz], "components": list(w.igreen),
                   "time_steps_per_bench_step": per_step_ts, "sgt_points": int(pts.shape[0]),
                   "timed_window": "time steps %d-%d of the %d-step job (untimed advance to there)" % (
                       prefill + args.warmup * per_step_ts, prefill + (args.warmup + args.steps) * per_step_ts,
                       w.nt),
                   "precision": args.precision, "l2": "inputs larger than L2 (%.1f GB state)" % (
                       s.p.nx * s.p.ny * s.p.nz * 4 * (15 * ncomp + 5) / 1e9),
                   "parallelism": "independent SGT jobs (sites) dealt to the GPUs" if world > 1 else "single GPU",
                   "site": site,
                   "tuning": used_tuning, "autotune": tune_info},
        "roofline": roofline,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "kernels": prof,
    }
    if world == 1 and not args.no_extras and not args.grid:
        # the plain FP32 two-sweep stepper (the comparison point of the batched
        # stepper's speed-up), block floating point memory variables and the
        # contracted stepper on the same window
        warm_ts, timed_ts = args.warmup * per_step_ts, min(args.steps, 10) * per_step_ts
        plain = window_rate(w, media, pts, stfs, local, "f32", "two_sweep", None, prefill, warm_ts, timed_ts)
        line["plain_fp32"] = plain
        line["vs_plain_fp32"] = value / plain["value"]
        if args.precision != "bfp":
            b = window_rate(w, media, pts, stfs, local, "bfp", "auto", None, prefill, warm_ts, timed_ts)
            b["vs_plain_fp32"] = b["value"] / plain["value"]
            study = precision_study()
            if study:
                b["sgt_rel_l2_vs_fp64"] = {k: v.get("bfp") for k, v in study.get("cases", {}).items()}
                b["error_source"] = study.get("source")
            line["bfp"] = b
        if args.kernel == "auto" and args.precision == "f32":
            f = window_rate(w, media, pts, stfs, local, "f32", "staged_fma", None, prefill, warm_ts, timed_ts)
            f["vs_plain_fp32"] = f["value"] / plain["value"]
            study = precision_study()
            if study:
                f["sgt_rel_l2_vs_fp64"] = {k: v.get("f32/staged_fma") for k, v in study.get("cases", {}).items()}
            line["staged_fma"] = f
        line["serving"] = serve_stream(16, 0.1, 1.2, 4, "fifo", 0.0)
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
