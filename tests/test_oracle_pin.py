"""The oracle's set-up stage pinned to the reference's own code.

The reference CUDA stepper's host set-up (AWP-GPU-SGT/src mesh.c inimesh and
tausub, cerjan.c inicrj) was built from the reference sources and run on one
rank to make the fixtures in tests/golden/setup (tests/golden/make_setup_golden.py).
The oracle follows the Fortran of AWP-ODC-SGT (structure.f, relax.f,
cerjan.f), which evaluates in single precision where the C promotes some steps
to double (its 1./(...) and log/exp of doubles), so the bar is:

* the layout, the ghost-free interior and the density: bit for bit;
* the Cerjan factors: bit for bit;
* the compliances lam, mu, the Q terms qp, qs and the relaxation times: within
  32 units in the last place (measured: 19 for lam, whose vp^2 - 2 vs^2 cancels;
  6 for mu; 4 for the Q terms and tau).

Two differences between the codes are known and left out: the C applies the Q
dispersion correction of the velocities whatever SoCalQ says (structure.f:482-487
applies it only with SoCalQ = 1), and it reads Q arrays it never allocates when
NVE = 0.  The device path equals the FP32 oracle bit for bit
(tests/test_gpu_parity.py), so these bounds hold for it too.
"""
import json
import os

import numpy as np
import pytest

import oracle
from tests.golden.make_setup_golden import CASES, OUT, media_for

MAX_ULP = 32


def ulps(a, b):
    a = np.asarray(a, np.float32).ravel().view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).ravel().view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(2 ** 31) - a, a)
    b = np.where(b < 0, -(2 ** 31) - b, b)
    return np.abs(a - b)


def oracle_setup(grid, m, nvar, nd, arbc, fp, fl, fh):
    nx, ny, nz = grid
    o = oracle.Oracle(nx=nx, ny=ny, nz=nz, dh=200.0, dt=0.01, nt=20, nd=nd, arbc=arbc, fp=fp, fl=fl, fh=fh, socalq=1,
                      nvar=nvar, nve=1, igreen=1)
    o.load_media(m)
    out = {}
    for f in ("lam", "mu", "d1", "qp", "qs"):
        a = o.field(f)
        out[f] = np.stack([a[nz + 1 - k, 2:ny + 2, 2:nx + 2] for k in range(nz)])
    out["tau"] = o.tau().transpose(2, 1, 0)            # [itz][ity][itx] -> [idx][idy][idz]
    out["cx"], out["cy"], out["cz"] = o.sponge()
    e = o.extremes()                                    # vp, vs, rho (min, max)
    out["extremes"] = np.array([e[2], e[3], e[0], e[1], e[4], e[5]], np.float32)
    o.close()
    return out


def check(got, ref):
    for f in ("d1", "cx", "cy", "cz"):
        assert np.array_equal(got[f].view(np.uint32), np.asarray(ref[f], np.float32).view(np.uint32)), f
    for f in ("lam", "mu", "qp", "qs", "tau"):
        d = ulps(got[f], ref[f])
        assert d.max() <= MAX_ULP, (f, int(d.max()))
    np.testing.assert_allclose(got["extremes"], ref["extremes"], rtol=4e-6)


def test_fixtures_match_their_inputs():
    meta = json.load(open(os.path.join(OUT, "cases.json")))
    assert [c["name"] for c in meta] == [c[0] for c in CASES]
    import hashlib
    for (name, grid, seed, nvar, *_), c in zip(CASES, meta):
        assert hashlib.sha256(media_for(grid, seed, nvar).tobytes()).hexdigest() == c["media_sha256"], name


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_setup_matches_reference_fixtures(case):
    name, grid, seed, nvar, nd, arbc, fp, fl, fh = case
    ref = dict(np.load(os.path.join(OUT, name + ".npz")))
    check(oracle_setup(grid, media_for(grid, seed, nvar), nvar, nd, arbc, fp, fl, fh), ref)


def test_oracle_setup_matches_live_reference():
    """Another grid and medium through the reference set-up built here (skipped
    where the reference sources were not there to build it)."""
    grid, nvar, nd, arbc = (26, 22, 14), 5, 7, 0.93
    m = media_for(grid, 23, nvar)
    ref = oracle.setup_reference(m, nvar=nvar, nve=1, socalq=1, arbc=arbc, nd=nd)
    if ref is None:
        pytest.skip("oracle/_ref/libsetup_ref.so not built (reference sources absent)")
    check(oracle_setup(grid, m, nvar, nd, arbc, 0.5, 0.01, 25.0), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_device_media_match_reference_fixtures(case):
    """The media the device holds (awp_get_field) against the same fixtures,
    and bit for bit against the oracle."""
    import awpsgt
    name, grid, seed, nvar, nd, arbc, fp, fl, fh = case
    nx, ny, nz = grid
    m = media_for(grid, seed, nvar)
    p = awpsgt.make_params(nx, ny, nz, 200.0, 0.01, 20, nd=nd, arbc=arbc, fp=fp, fl=fl, fh=fh, socalq=1, nvar=nvar,
                           nve=1, ntiskp_sgt=10, write_step=2)
    with awpsgt.Solver(p) as s:
        s.load_media(m)
        dev = {f: np.stack([s.field(f, 0)[nz + 1 - k, 2:ny + 2, 2:nx + 2] for k in range(nz)])
               for f in ("lam", "mu", "d1", "qp", "qs")}
    orc = oracle_setup(grid, m, nvar, nd, arbc, fp, fl, fh)
    for f in dev:
        assert np.array_equal(dev[f].view(np.uint32), orc[f].view(np.uint32)), f
    ref = dict(np.load(os.path.join(OUT, name + ".npz")))
    assert np.array_equal(dev["d1"].view(np.uint32), ref["d1"].view(np.uint32))
    for f in ("lam", "mu", "qp", "qs"):
        assert ulps(dev[f], ref[f]).max() <= MAX_ULP, f


# ---------------------------------------------------------------------------
# The time loop pinned to the reference's own stencil kernels.
#
# The reference CUDA stepper's dvelcx and dstrqc (AWP-GPU-SGT/src/
# kernel_kp1_fix_havg_ifault5.cu:420-504, 726-973), run on the host from the
# reference sources (oracle/Makefile.ref, oracle/gpusgt_step_driver.cpp), made
# the fixtures in tests/golden/timeloop (tests/golden/make_timeloop_golden.py).
# Their dstrqc is an algebraic regrouping of the Fortran allq (the two
# dt * r terms folded into one coefficient, double-precision literals, other
# association orders), so the bar is a relative L2 difference per field of
# at most 2e-6 (measured: 1.6e-7 to 2.1e-7, the FP32 rounding level; the FP32
# oracle lies as far from its FP64 build).  Every state field is compared,
# the memory variables included, in the cells below the free surface's reach.
# ---------------------------------------------------------------------------

from tests.golden import make_timeloop_golden as tl

TL_TOL = 2e-6


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("case", tl.CASES, ids=[c[0] for c in tl.CASES])
def test_timeloop_oracle_matches_reference_kernels_fixture(case):
    got = np.load(os.path.join(tl.OUT, case[0] + ".npz"))
    for precision in ("f32", "f64"):
        o = tl.make_oracle(case, precision)
        o.run(case[2])
        for f in oracle.FIELDS[:15]:
            want = got[f]
            assert want.shape == (tl.kmax(case), case[1][1], case[1][0])
            assert np.abs(want).max() > 0
            err = rel_l2(tl.region(case, o.field(f)), want)
            assert err <= TL_TOL, (case[0], precision, f, err)
        o.close()


needs_ref = pytest.mark.skipif(not os.path.exists(tl.REF_LIB), reason="reference kernels not built here")


@needs_ref
@pytest.mark.parametrize("case", tl.CASES + tl.LIVE_CASES, ids=[c[0] for c in tl.CASES + tl.LIVE_CASES])
def test_timeloop_oracle_matches_reference_kernels_live(case):
    ref = tl.run_reference(tl.load_ref(), case)
    o = tl.make_oracle(case)
    o.run(case[2])
    for f in range(15):
        err = rel_l2(tl.region(case, o.field(oracle.FIELDS[f])), tl.region(case, ref[f]))
        assert err <= TL_TOL, (case[0], oracle.FIELDS[f], err)
    o.close()


@needs_ref
def test_timeloop_comparison_detects_a_misplaced_coefficient():
    """The comparison has the power to see a wrong coefficient: the reference
    kernels given the relaxation coefficients with the x parity swapped (the
    kind of divergence the reference's own texture set-up has, by starting
    its parity from ghost indices) disagree with the oracle by orders of
    magnitude more than the bar, in the memory variables and the stresses."""
    case = tl.CASES[0]
    o = tl.make_oracle(case)
    t1, t2 = o.tau12()
    swap = lambda t: t.reshape(2, 2, 2)[:, :, ::-1].ravel().copy()   # noqa: E731
    ref = tl.run_reference(tl.load_ref(), case, tau_override=(swap(t1), swap(t2)))
    o.run(case[2])
    for f in ("r1", "r4", "xx"):
        err = rel_l2(tl.region(case, o.field(f)), tl.region(case, ref[oracle.FIELDS.index(f)]))
        assert err > 100 * TL_TOL, (f, err)
    o.close()
