"""Generates the synthesis golden fixtures under tests/golden/synth/ by running
DirectSynth's own synthesis functions (find_sgt, mech_sgt, sum_sgt,
timeshift_sgt, get_srfpars, srf_stf, do_cnvlv and the geoproj-1 projection),
built from the reference sources by oracle/Makefile.ref into
oracle/_ref/libsynth_ref.so, on seeded synthetic cases.  Run from the
repository root where the reference sources are present:

    make -s -f oracle/Makefile.ref && python tests/golden/make_synth_golden.py

The cases' inputs come from awp_inputs.synth_case with the listed arguments;
cases.json records a checksum of those inputs next to each fixture, so a test
can tell a changed generator from a changed synthesis.  The fixtures are the
reference's seismograms, [nvar][3][ntout] float32.
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

OUT = os.path.join(ROOT, "tests", "golden", "synth")

# name, synth_case arguments, ntout, tstart
CASES = [
    ("small_2comp", dict(seed=2, nx_f=8, nz_f=4, nt=200, nv=3), 400, 0.0),
    ("x_only_mech23", dict(seed=11, ncomp=1, nv=3, mech2_frac=0.2, mech3_frac=0.1), 700, 1.3),
    ("two_comp_short", dict(seed=12, ncomp=2, nv=3), 150, -2.0),
    ("three_comp", dict(seed=13, ncomp=3, nv=2, mech3_frac=0.3), 600, 0.0),
    ("all_off_grid", dict(seed=21, nv=2, zero_frac=0.3, drop_frac=1.0, nstf=(1, 100), nt=120), 100, 0.0),
    ("default_ntout", dict(seed=3, nx_f=6, nz_f=3, nt=100, nv=2), 0, 0.5),
]


def input_digest(c):
    h = hashlib.sha256()
    for a in [c.master, c.index, c.headers] + list(c.comps):
        h.update(np.ascontiguousarray(a).tobytes())
    for p, q in c.variations:
        h.update(np.ascontiguousarray(p).tobytes())
        h.update(np.ascontiguousarray(q).tobytes())
    h.update(np.float32([c.slon, c.slat, c.dtout]).tobytes())
    return h.hexdigest()


def main():
    os.makedirs(OUT, exist_ok=True)
    meta = []
    for name, kw, ntout, tstart in CASES:
        c = ai.synth_case(**kw)
        seis = oracle.synth_reference(c.master, c.index, c.headers, c.comps, c.slon, c.slat, c.dtout, ntout, tstart,
                                      c.variations)
        if seis is None:
            raise SystemExit("oracle/_ref/libsynth_ref.so is not built: make -f oracle/Makefile.ref")
        np.save(os.path.join(OUT, name + ".npy"), seis)
        meta.append({"name": name, "case": kw, "ntout": ntout, "tstart": tstart, "inputs_sha256": input_digest(c),
                     "shape": list(seis.shape)})
        print(name, seis.shape)
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
