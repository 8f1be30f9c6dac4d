"""FP64 reference SGTs of a benchmark workload for the precision study
(tests/test_precision_study.py, AWP_PRECISION_STUDY=cfg3): the FP64 oracle on
the host runs the workload's solve component by component (hours of CPU for
the 640x640x256, 3000-step workload; about 17 GB of host memory per
component) and keeps the SGT file image of the first POINTS SGT points (the
wavefield does not depend on the points, so these records equal those of the
full solve), rounded to float32.  The output is too large to commit; pass its
directory to the study through AWP_PRECISION_REF.

    python tests/golden/make_precision_ref.py --config 3 --points 1000 --out REF [--steps N] [--components 2]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "cybershake-core_b200"), os.path.join(ROOT, "oracle")]
import awp_inputs as ai  # noqa: E402
import oracle  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--points", type=int, default=1000)
    ap.add_argument("--steps", type=int, default=0, help="time steps - 1 (default: the workload's NST)")
    ap.add_argument("--out", required=True)
    ap.add_argument("--components", default="", help="IGREEN values to make, e.g. 2 (default: all of the workload's)")
    args = ap.parse_args()
    w = ai.config(args.config)
    nst = args.steps or w.nst
    nt = nst + 1
    write_step = w.nst // w.ntiskp_sgt
    os.makedirs(args.out, exist_ok=True)
    media = w.media()
    pts = w.points()[:args.points]
    t0 = time.time()
    want = [int(c) for c in args.components.split(",")] if args.components else list(w.igreen)
    for q, g in enumerate(w.igreen):
        if g not in want:
            continue
        o = oracle.Oracle(nx=w.nx, ny=w.ny, nz=w.nz, dh=w.dh, dt=w.dt, nt=nt, nst=w.nst, nd=20, arbc=0.92, fl=w.fl,
                          fh=w.fh, fp=w.fp, socalq=w.socalq, ntiskp_sgt=w.ntiskp_sgt, write_step=write_step,
                          igreen=g, precision="f64")
        o.load_media(media)
        o.set_source([w.src_xyz], w.stf(q))
        o.set_points(pts)
        o.run(nt)
        np.save(os.path.join(args.out, "c%d.npy" % g), o.sgt().astype(np.float32))
        o.close()
        print("component %d done after %.0f s" % (g, time.time() - t0), flush=True)
    meta = {"config": args.config, "workload": w.name, "steps": nst, "points": args.points,
            "write_step": write_step, "note": "%d time steps, first %d of %d points, %.0f s on %d host threads" % (
                nt, args.points, w.npts, time.time() - t0, oracle.threads())}
    with open(os.path.join(args.out, "meta.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
