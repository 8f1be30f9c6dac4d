"""Launch shapes and the autotuner (awp_get_tuning / awp_set_tuning /
awp_autotune).

A launch shape changes how the grid is cut into work items, never the
arithmetic of a cell update, so every solve must stay bit-identical to the
FP32 oracle whatever tuning it runs with, including a tuning switched between
two steps of one solve.
"""
import os

import pytest

import awpsgt
from test_gpu_parity import Case, assert_same_state, bits_equal

pytestmark = pytest.mark.gpu


def solver_for(c, kernel, tuning=None):
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel=kernel, **c.kw())
    s = awpsgt.Solver(p)
    if tuning is not None:
        s.set_tuning(tuning)
    s.load_media(c.media)
    for q in range(len(c.igreen)):
        s.set_source(q, c.srcs[q], c.stfs[q])
    s.set_points(c.pts)
    return s


def variant(t, **kw):
    u = awpsgt.Tuning()
    for n, _ in awpsgt.Tuning._fields_:
        setattr(u, n, kw.get(n, getattr(t, n)))
    return u


# shape 2 is one work item over the whole depth (nz = 30)
SHAPES = {
    "staged": [dict(kchunk_staged=9, staged_rpt=2, staged_rpt_vel=2, unroll=1, staged_qslow=0),
               dict(kchunk_staged=16, staged_rpt=1, staged_rpt_vel=1, unroll=2, staged_qslow=1, staged_batch=3),
               dict(kchunk_staged=30)],
    "fused": [dict(ty=4, kchunk=16), dict(ty=16, kchunk=8), dict(ty=8, kchunk=30)],
    "two_sweep": [dict(ty=4, kchunk_sweep=8, unroll=2), dict(ty=16, kchunk_sweep=12, unroll=1),
                  dict(ty=8, kchunk_sweep=30)],
}


@pytest.mark.parametrize("kernel", ["staged", "fused", "two_sweep"])
@pytest.mark.parametrize("shape", [0, 1, 2])
def test_any_tuning_is_bit_exact(kernel, shape):
    c = Case(nx=44, ny=36, nz=30, nt=30, igreen=(1, 2), srcs=[[(20, 18, 6)], [(20, 18, 6)]])
    probe = solver_for(c, kernel)
    t = variant(probe.tuning(), **SHAPES[kernel][shape])
    probe.close()
    s = solver_for(c, kernel, t)
    got = s.tuning()
    assert got.as_dict() == t.as_dict()
    s.run(c.nt)
    for q in range(2):
        assert_same_state(s, c.oracle(q), q)


@pytest.mark.parametrize("kernel", ["staged", "fused", "two_sweep"])
def test_tuning_switched_mid_solve(kernel):
    c = Case(nx=40, ny=32, nz=26, nt=36, igreen=(3,), srcs=[[(18, 15, 9)]])
    ref = solver_for(c, kernel)
    ref.run(c.nt)
    s = solver_for(c, kernel)
    t0 = s.tuning()
    s.run(11)
    s.set_tuning(variant(t0, **SHAPES[kernel][0]))
    s.run(12)
    s.set_tuning(variant(t0, **SHAPES[kernel][1]))
    s.run(c.nt - 23)
    assert bits_equal(s.sgt(0), ref.sgt(0))
    assert bits_equal(s.chkj(0), ref.chkj(0))
    assert bits_equal(s.field("xy", 0), ref.field("xy", 0))


def test_set_tuning_rejects_bad_shapes():
    c = Case(nx=32, ny=24, nz=20, nt=10)
    s = solver_for(c, "staged")
    t = s.tuning()
    for bad in [dict(kchunk_staged=7), dict(kchunk_staged=21), dict(staged_rpt=3), dict(unroll=0),
                dict(ty=12), dict(staged_qslow=2), dict(kchunk=4), dict(kchunk_sweep=100), dict(staged_rpt_vel=0)]:
        with pytest.raises(awpsgt.AwpError):
            s.set_tuning(variant(t, **bad))
    assert s.tuning().as_dict() == t.as_dict()      # a rejected tuning changes nothing


@pytest.mark.parametrize("kernel", ["staged", "fused"])
def test_autotune_and_cache(kernel, tmp_path):
    c = Case(nx=96, ny=80, nz=72, nt=10, igreen=(1, 2))
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel=kernel, **c.kw())
    cache = str(tmp_path / "tune.txt")
    t, rate = awpsgt.autotune(p, c.media, trial_steps=4, cache=cache)
    assert rate > 0
    lines = open(cache).read().splitlines()
    assert len(lines) == 1
    # the second call reads the cache (same result, no new line)
    t2, rate2 = awpsgt.autotune(p, c.media, trial_steps=4, cache=cache)
    assert t2.as_dict() == t.as_dict() and rate2 == pytest.approx(rate, rel=1e-5)
    assert len(open(cache).read().splitlines()) == 1
    # a homogeneous trial of another grid is a new key
    p2 = awpsgt.make_params(c.nx, c.ny, 64, c.dh, c.dt, c.nt, igreen=c.igreen, kernel=kernel, **c.kw())
    t3, rate3 = awpsgt.autotune(p2, None, trial_steps=4, cache=cache)
    assert rate3 > 0 and len(open(cache).read().splitlines()) == 2
    # the tuned solve is the oracle's, bit for bit
    small = Case(nx=c.nx, ny=c.ny, nz=c.nz, nt=8, igreen=(1,), srcs=[[(40, 40, 10)]])
    s = solver_for(small, kernel, t)
    s.run(small.nt)
    assert_same_state(s, small.oracle(0), 0, fields=["u1", "xx", "xy"])
    assert os.path.getsize(cache) > 0


def test_autotune_rejects_bad_arguments():
    c = Case(nx=32, ny=24, nz=20, nt=10)
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, **c.kw())
    for bad in (0, -3, 100001):
        with pytest.raises(awpsgt.AwpError):
            awpsgt.autotune(p, c.media, trial_steps=bad)


STATE = awpsgt.FIELDS[:15]


@pytest.mark.parametrize("batch", [1, 2, 3])
@pytest.mark.parametrize("igreen", [(1, 2), (1, 2, 3), (-2, 4, 6)])
@pytest.mark.parametrize("precision", ["f32", "mixed"])
@pytest.mark.parametrize("nve", [1, 0])
def test_batched_sweeps_match_per_component(igreen, precision, nve, batch):
    """Components side by side in one work item (shared media tiles and cell
    coefficients; batch bit 0 the stress sweep, bit 1 the velocity sweep)
    against one component per work item: every state field, the CHKJ series
    and the SGTs bit for bit; FP32 also against the oracle."""
    n = len(igreen)
    c = Case(nx=45, ny=37, nz=29, nt=30, igreen=igreen, srcs=[[(20, 18, 6)]] * n, nve=nve)
    runs = []
    for batch in (0, batch):
        p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel="staged",
                               precision=precision, **c.kw())
        s = awpsgt.Solver(p)
        s.set_tuning(variant(s.tuning(), staged_batch=batch, kchunk_staged=11))
        s.load_media(c.media)
        for q in range(n):
            s.set_source(q, c.srcs[q], c.stfs[q])
        s.set_points(c.pts)
        s.run(c.nt)
        assert s.tuning().staged_batch == batch
        runs.append(s)
    a, b = runs
    for q in range(n):
        for f in STATE[:9] + (STATE[9:] if nve == 1 else []):
            assert bits_equal(a.field(f, q), b.field(f, q)), (q, f)
        assert bits_equal(a.chkj(q), b.chkj(q))
        assert bits_equal(a.sgt(q), b.sgt(q))
    if precision == "f32" and igreen[0] > 0:
        assert_same_state(b, c.oracle(0), 0, fields=STATE if nve == 1 else STATE[:9])


@pytest.mark.parametrize("batch", [0, 1, 3])
def test_single_level_chunk_all_batch_masks(batch):
    """nz = 33 in 8-level chunks leaves a one-level chunk at the bottom: the
    queues of the side-by-side sweeps are set up and rotated on the same
    level there."""
    c = Case(nx=40, ny=20, nz=33, nt=20, igreen=(1, 2, 3), srcs=[[(20, 10, 5)], [(21, 9, 6)], [(19, 11, 4)]])
    s = solver_for(c, "staged", None)
    s.close()
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel="staged", **c.kw())
    s = awpsgt.Solver(p)
    s.set_tuning(variant(s.tuning(), staged_batch=batch, kchunk_staged=8))
    s.load_media(c.media)
    for q in range(3):
        s.set_source(q, c.srcs[q], c.stfs[q])
    s.set_points(c.pts)
    s.run(c.nt)
    for q in range(3):
        assert_same_state(s, c.oracle(q), q)


@pytest.mark.parametrize("kernel", ["staged", "two_sweep", "fused"])
def test_sm_limit_is_bit_exact(kernel):
    """Persistent grids sized for a share of the SMs (as the server sizes
    solves that share a GPU), switched mid-solve: same results."""
    c = Case(nx=44, ny=36, nz=30, nt=40, igreen=(1, 2), srcs=[[(22, 18, 8)], [(20, 16, 12)]])
    s = solver_for(c, kernel)
    t0 = s.tuning()
    assert t0.sm_limit == 0
    s.set_tuning(variant(t0, sm_limit=5))
    s.run(17)
    s.set_tuning(variant(t0, sm_limit=37))
    s.run(c.nt)
    for q in range(2):
        assert_same_state(s, c.oracle(q), q)
    with pytest.raises(awpsgt.AwpError):
        s.set_tuning(variant(t0, sm_limit=-1))
    s.close()


@pytest.mark.parametrize("precision", ["f32", "mixed"])
def test_generic_ring_loads_are_bit_exact(monkeypatch, precision):
    """AWP_TUNE_GENERIC=1 (the default above 32 GiB of state) makes the
    one-component staged sweeps read their rings with generic loads: same
    arithmetic, so the same bits as the default sweeps and, in FP32, as the
    oracle."""
    c = Case(nx=45, ny=37, nz=29, nt=30, igreen=(1, 2), srcs=[[(20, 18, 6)], [(22, 16, 9)]])
    runs = []
    for gen in ("0", "1"):
        monkeypatch.setenv("AWP_TUNE_GENERIC", gen)
        p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel="staged",
                               precision=precision, **c.kw())
        s = awpsgt.Solver(p)
        s.set_tuning(variant(s.tuning(), staged_batch=0, kchunk_staged=11))
        s.load_media(c.media)
        for q in range(2):
            s.set_source(q, c.srcs[q], c.stfs[q])
        s.set_points(c.pts)
        s.run(c.nt)
        runs.append(s)
    a, b = runs
    for q in range(2):
        for f in STATE:
            assert bits_equal(a.field(f, q), b.field(f, q)), (q, f)
        assert bits_equal(a.sgt(q), b.sgt(q))
    if precision == "f32":
        assert_same_state(b, c.oracle(0), 0)
    for s in runs:
        s.close()
