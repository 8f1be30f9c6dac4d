"""Failure detection without a GPU fault.

* A bounded barrier wait that runs out: with AWP_TEST_TMA_WITHHOLD the producer
  warp of block 0 in the staged stress sweep issues no copies (and no arrival)
  for one ring use, so the consumers waiting on that slot give up after the
  wait limit (AWP_TEST_WAIT_US, here 20 ms).  The block's other copies land
  before it exits; the solve reports AWP_ERR_TIMEOUT; the context stays usable
  and the next solve is bit-exact with the oracle.
* A device allocation that fails (AWP_TEST_FAIL_ALLOC = n: the n-th allocation
  of awp_create): AWP_ERR_OOM, everything allocated so far is released, and
  the next solver works.
Both knobs are read by awp_create; nothing here traps, faults or hangs a GPU.
"""
import gc

import numpy as np
import pytest

import awpsgt

from test_gpu_parity import Case, assert_same_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ncomp,kernel_name", [(3, "k_str_tmab"), (1, "k_str_tma")])
def test_withheld_tile_copy_times_out_then_next_solve_is_exact(monkeypatch, ncomp, kernel_name):
    c = Case(nt=30, igreen=(1, 2, 3)[:ncomp], srcs=[[(24, 20, 10)]] * ncomp)
    monkeypatch.setenv("AWP_TEST_TMA_WITHHOLD", "5")
    monkeypatch.setenv("AWP_TEST_WAIT_US", "20000")
    with pytest.raises(awpsgt.AwpError) as e:
        c.gpu(kernel="staged")
    assert awpsgt.STATUS[e.value.status] == "AWP_ERR_TIMEOUT"
    assert "barrier wait ran out" in str(e.value)
    monkeypatch.delenv("AWP_TEST_TMA_WITHHOLD")
    monkeypatch.delenv("AWP_TEST_WAIT_US")
    s = c.gpu(steps=5, kernel="staged")
    assert s.profile(1)[kernel_name]["launches"] == 1       # the stress sweep the injection exercised
    s.close()
    s = c.gpu(kernel="staged")
    for q in range(ncomp):
        assert_same_state(s, c.oracle(q), q)


@pytest.mark.parametrize("nth", [1, 7, 20])
def test_failed_allocation_is_oom_and_releases_everything(monkeypatch, nth):
    c = Case(nt=20)
    gc.collect()                                      # solvers of earlier tests released first
    live0, _ = awpsgt.device_memory(0)
    monkeypatch.setenv("AWP_TEST_FAIL_ALLOC", str(nth))
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, **c.kw())
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.Solver(p)
    assert awpsgt.STATUS[e.value.status] == "AWP_ERR_OOM"
    assert "AWP_TEST_FAIL_ALLOC" in str(e.value)
    assert awpsgt.device_memory(0)[0] == live0          # every block of the failed solver released
    monkeypatch.delenv("AWP_TEST_FAIL_ALLOC")
    s = c.gpu()
    assert awpsgt.device_memory(0)[0] > live0
    assert_same_state(s, c.oracle())
    assert np.abs(s.sgt()).max() > 0
    s.close()
    assert awpsgt.device_memory(0)[0] == live0
