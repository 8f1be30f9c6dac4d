"""Generates the set-up golden fixtures under tests/golden/setup/ by running
the reference CUDA stepper's own host set-up on one rank (AWP-GPU-SGT/src
mesh.c inimesh and tausub, cerjan.c inicrj), built from the reference sources
by oracle/Makefile.ref into oracle/_ref/libsetup_ref.so.  Run from the
repository root where the reference sources are present:

    make -s -f oracle/Makefile.ref && python tests/golden/make_setup_golden.py

The cases use SoCalQ = 1 and the viscoelastic scheme: the C set-up applies the
Q dispersion correction whatever SoCalQ says (the Fortran, which the oracle
follows, only with SoCalQ = 1), and it reads the Q arrays it does not allocate
when NVE = 0.  Media come from awp_inputs.layered_media with the listed
arguments; cases.json records a checksum of each input next to its fixture.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "cybershake-core_b200"), os.path.join(ROOT, "oracle")]
import awp_inputs as ai  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "setup")

# name, grid (nx, ny, nz), media seed, nvar, nd, arbc, fp, fl, fh
CASES = [
    ("nvar3_nd6", (20, 16, 12), 3, 3, 6, 0.92, 0.5, 0.01, 25.0),
    ("nvar5_nd4", (18, 14, 11), 7, 5, 4, 0.95, 1.0, 0.02, 10.0),
    ("nvar8_nd5", (16, 18, 10), 11, 8, 5, 0.90, 0.5, 0.01, 25.0),
]


def media_for(grid, seed, nvar):
    nx, ny, nz = grid
    m = ai.layered_media(nx, ny, nz, 200.0, seed=seed, pert_std=0.05, corr_len=1000.0)
    if nvar == 3:
        return m
    full = np.zeros((nz, ny, nx, nvar), np.float32)
    off = 3 if nvar == 8 else 0
    full[..., off:off + 3] = m
    full[..., off + 4] = 0.08 * m[..., 1]
    full[..., off + 3] = 1.7 * full[..., off + 4]
    return full


def main():
    os.makedirs(OUT, exist_ok=True)
    meta = []
    for name, grid, seed, nvar, nd, arbc, fp, fl, fh in CASES:
        m = media_for(grid, seed, nvar)
        r = oracle.setup_reference(m, nvar=nvar, nve=1, socalq=1, fp=fp, fl=fl, fh=fh, arbc=arbc, nd=nd)
        if r is None:
            raise SystemExit("oracle/_ref/libsetup_ref.so is not built: make -f oracle/Makefile.ref")
        np.savez(os.path.join(OUT, name + ".npz"), **{k: np.asarray(v) for k, v in r.items()})
        meta.append({"name": name, "grid": list(grid), "seed": seed, "nvar": nvar, "nd": nd, "arbc": arbc, "fp": fp,
                     "fl": fl, "fh": fh, "media_sha256": hashlib.sha256(m.tobytes()).hexdigest()})
        print(name)
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
