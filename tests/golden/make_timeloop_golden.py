"""Generates the time-loop golden fixtures under tests/golden/timeloop/ by running
the reference CUDA stepper's own velocity and stress kernels (dvelcx and
dstrqc of AWP-GPU-SGT/src/kernel_kp1_fix_havg_ifault5.cu) on the host CPU.
oracle/Makefile.ref cuts them out of the reference file and builds them with
oracle/gpusgt_step_driver.cpp into oracle/_ref/libgpusgt_step_ref.so.  Run
from the repository root where the reference sources are present:

    make -s -f oracle/Makefile.ref && python tests/golden/make_timeloop_golden.py

Each case starts from a seeded state of bounded noise (every wavefield and
memory-variable cell of the interior; ghost cells zero) on a seeded layered
medium.  The medium as the steppers read it (compliances, density, Q terms),
the relaxation coefficients of each cell (by the Fortran's parity rule,
viscoop.f:93-101) and the Cerjan factors are the oracle's own -- the set-up
stage is pinned to the reference separately (tests/golden/setup) -- so both
stepper implementations integrate exactly the same problem.  The fixture holds
every state field after NSTEPS steps in the cells below the free surface's
reach (k <= nz - 4*NSTEPS - 3): the reference's free-surface treatment differs
from the Fortran's by design (its averaged-moduli w image), and each step
carries a difference at most four cells further down.
"""
import ctypes as C
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "cybershake-core_b200"), os.path.join(ROOT, "oracle")]
import awp_inputs as ai  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "timeloop")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libgpusgt_step_ref.so")

# name, (nx, ny, nz), steps, dh, dt, medium ("layered" seed / "homogeneous"), noise seed
CASES = [
    ("layered_20x16x40_5steps", (20, 16, 40), 5, 100.0, 0.005, ("layered", 5), 0),
]
# further cases the tests run against the live library where it is built
LIVE_CASES = [
    ("homog_24x22x44_5steps", (24, 22, 44), 5, 200.0, 0.01, ("homogeneous", 0), 1),
    ("layered_26x18x52_7steps", (26, 18, 52), 7, 100.0, 0.005, ("layered", 9), 2),
]
# noise magnitude per state field: velocities, stresses, memory variables
SCALE = [1e-2] * 3 + [1e6] * 6 + [1e3] * 6
KW = dict(nd=6, arbc=0.92, fl=0.01, fh=25.0, fp=0.5, socalq=1, ntiskp_sgt=5, write_step=1)


def kmax(case):
    _, (nx, ny, nz), n, *_ = case
    return nz - 4 * n - 3


def make_oracle(case, precision="f32"):
    """The oracle on the case's medium with a zero source (so that the state
    alone drives the solve), its state set to the case's noise."""
    _, (nx, ny, nz), n, dh, dt, (kind, mseed), nseed = case
    media = (ai.homogeneous_media(nx, ny, nz) if kind == "homogeneous"
             else ai.layered_media(nx, ny, nz, dh, seed=mseed, pert_std=0.05, corr_len=1000.0))
    o = oracle.Oracle(nx=nx, ny=ny, nz=nz, dh=dh, dt=dt, nt=n, nst=n, igreen=1, precision=precision, **KW)
    o.load_media(media)
    o.set_source([(nx // 2, ny // 2, nz // 2)], np.zeros((n, 6), np.float32))
    o.set_points(np.array([[1, 1, 1]], np.int32))
    for f, a in enumerate(noise_state(case)):
        o.set_field(oracle.FIELDS[f], a)
    return o


def noise_state(case):
    _, (nx, ny, nz), _, _, _, _, nseed = case
    rng = np.random.default_rng(nseed)
    out = []
    for f in range(15):
        a = np.zeros((nz + 4, ny + 4, nx + 4), np.float32)
        a[2:-2, 2:-2, 2:-2] = (rng.uniform(-1.0, 1.0, (nz, ny, nx)) * SCALE[f]).astype(np.float32)
        out.append(a)
    return out


def load_ref():
    lib = C.CDLL(REF_LIB)
    lib.gsr_create.restype = C.c_void_p
    lib.gsr_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float]
    lib.gsr_destroy.argtypes = [C.c_void_p]
    lib.gsr_set.argtypes = lib.gsr_get.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    lib.gsr_set_tau.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.gsr_set_sponge.argtypes = [C.c_void_p] * 4
    lib.gsr_run.argtypes = [C.c_void_p, C.c_int]
    return lib


def run_reference(lib, case, tau_override=None):
    """The reference kernels on the case: every state field after the steps,
    padded host layout [nz+4][ny+4][nx+4].  tau_override replaces the
    (tau1, tau2) tables."""
    _, (nx, ny, nz), n, dh, dt, _, _ = case
    p = lambda a: a.ctypes.data_as(C.c_void_p)   # noqa: E731
    o = make_oracle(case)
    h = lib.gsr_create(nx, ny, nz, dh, dt)
    try:
        for f, a in enumerate(noise_state(case)):
            lib.gsr_set(h, f, p(a))
        for f in range(15, 20):
            m = np.ascontiguousarray(o.field(oracle.FIELDS[f]), dtype=np.float32)
            lib.gsr_set(h, f, p(m))
        t1, t2 = o.tau12() if tau_override is None else tau_override
        t1, t2 = np.ascontiguousarray(t1, np.float32), np.ascontiguousarray(t2, np.float32)
        lib.gsr_set_tau(h, p(t1), p(t2))
        cx, cy, cz = o.sponge()
        lib.gsr_set_sponge(h, p(cx), p(cy), p(cz))
        lib.gsr_run(h, n)
        out = []
        for f in range(15):
            g = np.zeros((nz + 4, ny + 4, nx + 4), np.float32)
            lib.gsr_get(h, f, p(g))
            out.append(g)
        return out
    finally:
        lib.gsr_destroy(h)
        o.close()


def region(case, a):
    """The compared cells: interior in x and y, k = 1 .. kmax."""
    _, (nx, ny, nz), *_ = case
    return a[2:kmax(case) + 2, 2:ny + 2, 2:nx + 2]


def main():
    lib = load_ref()
    os.makedirs(OUT, exist_ok=True)
    meta = []
    for case in CASES:
        fields = run_reference(lib, case)
        np.savez_compressed(os.path.join(OUT, case[0] + ".npz"),
                            **{oracle.FIELDS[f]: region(case, fields[f]) for f in range(15)})
        meta.append({"name": case[0], "grid": case[1], "steps": case[2], "dh": case[3], "dt": case[4],
                     "medium": case[5], "noise_seed": case[6], "kmax": kmax(case)})
    with open(os.path.join(OUT, "cases.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", len(meta), "case(s) to", OUT)


if __name__ == "__main__":
    main()
