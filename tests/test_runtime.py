"""Host runtime around the stepper: the device block cache that keeps freed
arrays for the next solver, and media uploads straight from page-locked host
memory.  Neither may change a result: a solver built on reused blocks, or fed
from pinned memory, must match a fresh one bit for bit.
"""
import numpy as np
import pytest

import awpsgt
from test_gpu_parity import Case, bits_equal

pytestmark = pytest.mark.gpu


def solve(c, media=None, kernel="auto"):
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel=kernel, **c.kw())
    s = awpsgt.Solver(p)
    s.load_media(c.media if media is None else media)
    for q in range(len(c.igreen)):
        s.set_source(q, c.srcs[q], c.stfs[q])
    s.set_points(c.pts)
    s.run(c.nt)
    out = [s.sgt(q) for q in range(len(c.igreen))] + [s.field("xy", 0), s.field("mu", 0), s.chkj(0)]
    s.close()
    return out


@pytest.mark.parametrize("kernel", ["staged", "fused"])
def test_reused_blocks_give_identical_results(kernel):
    awpsgt.release_cached_memory()
    a = Case(nx=48, ny=40, nz=32, nt=30, igreen=(1, 2), srcs=[[(20, 18, 6)], [(20, 18, 6)]], seed=3)
    b = Case(nx=48, ny=40, nz=32, nt=30, igreen=(1, 2), srcs=[[(30, 10, 12)], [(8, 30, 2)]], seed=9,
             stf_seed=11)
    first = solve(a, kernel=kernel)           # fresh blocks
    other = solve(b, kernel=kernel)           # a's blocks, other data left in them
    again = solve(a, kernel=kernel)           # b's blocks
    assert all(bits_equal(x, y) for x, y in zip(first, again))
    assert not bits_equal(first[0], other[0])
    awpsgt.release_cached_memory()
    fresh = solve(a, kernel=kernel)
    assert all(bits_equal(x, y) for x, y in zip(first, fresh))


def test_other_grid_after_cached_blocks():
    a = Case(nx=40, ny=32, nz=24, nt=20)
    b = Case(nx=56, ny=36, nz=28, nt=20)
    ra = solve(a)
    solve(b)
    assert all(bits_equal(x, y) for x, y in zip(ra, solve(a)))


def test_pinned_media_upload_matches_pageable():
    torch = pytest.importorskip("torch")
    c = Case(nx=52, ny=44, nz=36, nt=24, igreen=(3,), srcs=[[(25, 20, 9)]])
    pinned = torch.from_numpy(c.media.copy()).pin_memory().numpy()
    got = solve(c, media=pinned)
    ref = solve(c)
    assert all(bits_equal(x, y) for x, y in zip(got, ref))
    assert np.abs(ref[0]).max() > 0


def test_slightly_smaller_grid_reuses_blocks_and_matches():
    """A grid a few percent smaller takes the idle blocks of a larger one
    (their tails hold stale data) and still matches a fresh solve."""
    awpsgt.release_cached_memory()
    big = Case(nx=50, ny=40, nz=32, nt=20)
    small = Case(nx=48, ny=40, nz=31, nt=20, seed=5)
    fresh = solve(small)
    awpsgt.release_cached_memory()
    solve(big)
    reused = solve(small)
    assert all(bits_equal(x, y) for x, y in zip(fresh, reused))
