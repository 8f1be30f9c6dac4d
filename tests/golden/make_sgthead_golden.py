"""Generates the SgtHead golden fixtures under tests/golden/sgthead/ by running
the reference's own write_head and reformat_awp, built from the reference
sources by oracle/Makefile.ref (`make -f oracle/Makefile.ref`), on seeded
synthetic inputs.  Run from the repository root where the reference sources
are present:

    make -s -f oracle/Makefile.ref && python tests/golden/make_sgthead_golden.py

The fixtures (inputs and the reference outputs) are small and committed, so the
tests can check the header writer and the RWG reordering without the reference.
"""
import json
import os
import shutil
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "cybershake-core_b200"))
import awp_inputs as ai  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "sgthead")
REF = os.path.join(ROOT, "oracle", "_ref")

# (name, grid, spacing km, points, seed, rotation, write_head arguments after the media file)
HEADERS = [
    ("hdr_x", (24, 20, 12), 0.1, 60, 1, -55.0, dict(nt=4000, dt=0.005, tinc=10, comp="x", moment=1.0e20, flo=1.0,
                                                     corr=False)),
    ("hdr_z_corr", (17, 23, 9), 0.2, 40, 3, 12.5, dict(nt=3000, dt=0.01, tinc=5, comp="z", moment=2.5e19, flo=0.5,
                                                        corr=True)),
]
REFORMAT = [("sgt_x", 30, 37, 0, False), ("sgt_z", 30, 37, 1, True)]   # name, points, nt, seed, -z
VELOCITY = [("vel_20x17x9", 20, 17, 9, 5), ("vel_33x8x5", 33, 8, 5, 6)]   # name, nx, ny, nz, seed


def main():
    os.makedirs(OUT, exist_ok=True)
    meta = {"headers": [], "reformat": []}
    for name, (nx, ny, nz), h, npts, seed, rot, a in HEADERS:
        d = os.path.join(OUT, name)
        if os.path.isdir(d):
            shutil.rmtree(d)
        p = ai.write_sgthead_inputs(d, nx, ny, nz, h, npts, seed=seed, mrot=rot)
        args = [os.path.basename(p[k]) for k in ("modelbox", "coordfile", "fdloc", "gridout")]
        args += [str(h), str(a["nt"]), str(a["dt"]), str(a["tinc"]), a["comp"], "%g" % a["moment"], str(a["flo"]),
                 os.path.basename(p["media"]), "expected.sgthead"] + (["-c"] if a["corr"] else [])
        subprocess.run([os.path.join(REF, "write_head")] + args, cwd=d, check=True, capture_output=True)
        meta["headers"].append({"name": name, "args": args})
    for name, npts, nt, seed, z in REFORMAT:
        d = os.path.join(OUT, name)
        os.makedirs(d, exist_ok=True)
        np.random.default_rng(seed).standard_normal(npts * 6 * nt).astype(np.float32).tofile(os.path.join(d, "in.sgt"))
        subprocess.run([os.path.join(REF, "reformat_awp"), "in.sgt", str(nt), "expected.sgt"] + (["-z"] if z else []),
                       cwd=d, check=True, capture_output=True)
        meta["reformat"].append({"name": name, "nt": nt, "z": z})
    meta["velocity"] = []
    for name, nx, ny, nz, seed in VELOCITY:
        d = os.path.join(OUT, name)
        os.makedirs(d, exist_ok=True)
        rng = np.random.default_rng(seed)
        vs = (0.4 + 3.6 * rng.random(ny * nz * nx)).astype(np.float32)          # km/s, RWG order y, z, x
        (1.73 * vs).astype(np.float32).tofile(os.path.join(d, "v.p"))
        vs.tofile(os.path.join(d, "v.s"))
        (1.6 + rng.random(ny * nz * nx)).astype(np.float32).tofile(os.path.join(d, "v.d"))   # g/cm^3
        subprocess.run([os.path.join(REF, "reformat_velocity"), str(nx), str(ny), str(nz), "v", "expected.media"],
                       cwd=d, check=True, capture_output=True)
        meta["velocity"].append({"name": name, "nx": nx, "ny": ny, "nz": nz})
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
