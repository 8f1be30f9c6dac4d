"""FP64 stability monitor, asynchronous stepping and device views (GPU)."""
import numpy as np
import pytest

import awp_inputs as ai
import awpsgt

pytestmark = pytest.mark.gpu


def solver(nt=60, dt=0.01, monitor=0, kernel="auto", ncomp=1):
    nx, ny, nz = 48, 40, 32
    media = ai.layered_media(nx, ny, nz, 200.0, seed=2, pert_std=0.05, corr_len=1000.0)
    p = awpsgt.make_params(nx, ny, nz, 200.0, dt, nt, igreen=(1, 2, 3)[:ncomp], nd=8, socalq=1, ntiskp_sgt=5,
                           write_step=4, monitor_every=monitor, kernel=kernel)
    s = awpsgt.Solver(p)
    s.load_media(media)
    for q in range(ncomp):
        s.set_source(q, [(24, 20, 9)], ai.gaussian_derivative_stf(nt, dt, f0=1.0, column=q))
    s.set_points(ai.sgt_points(nx, ny, 20, 20))
    return s


def host_energy(s, q=0):
    tot = 0.0
    p = s.p
    for f in ("u1", "v1", "w1"):
        a = s.field(f, q)[2:p.nz + 2, 2:p.ny + 2, 2:p.nx + 2].astype(np.float64)
        tot += float((a * a).sum())
    return tot


@pytest.mark.parametrize("kernel", ["fused", "two_sweep"])
def test_energy_matches_host_sum(kernel):
    s = solver(kernel=kernel, ncomp=2)
    s.run(40)
    e = s.energy()
    for q in range(2):
        h = host_energy(s, q)
        assert h > 0
        assert abs(e[q] - h) <= 1e-12 * h


def test_field_energy_on_device_pointers():
    s = solver(ncomp=3)
    s.run(33)
    ptrs, L = [], None
    for q in range(3):
        for f in ("u1", "v1", "w1"):
            p, L = s.device_field(f, q)
            ptrs.append(p)
    a = awpsgt.field_energy(ptrs, L, 3)
    b = s.energy()
    assert np.array_equal(a, b)


def test_energy_is_deterministic():
    s = solver()
    s.run(30)
    a = s.energy()
    b = s.energy()
    assert np.array_equal(a, b)


def test_monitor_quiet_on_stable_run():
    s = solver(monitor=10)
    s.run(60)
    assert s.energy()[0] > 0


def test_monitor_reports_blow_up():
    """dt far beyond the CFL limit: the wavefield overflows to Inf/NaN and
    the monitor turns that into AWP_ERR_UNSTABLE (no device trap)."""
    s = solver(nt=400, dt=0.05, monitor=20)
    with pytest.raises(awpsgt.AwpError) as e:
        s.run(400)
    assert e.value.status == 5


def test_async_matches_sync():
    a = solver(kernel="fused")
    a.run(60)
    ref = a.sgt()
    b = solver(kernel="fused")
    b.run_async(23)
    b.run_async(37)
    while not b.query():
        pass
    b.sync()
    assert np.array_equal(b.sgt(), ref)
