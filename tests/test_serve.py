"""Continuous-batching server: every request's SGT is the same alone and in
the mix, admission respects the HBM budget, cancellation works (GPU)."""
import time

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt

pytestmark = pytest.mark.gpu


def make_request(seed, size, comps, nt, precision="f32", kernel="auto"):
    nx, ny, nz = size
    rng = np.random.default_rng(seed)
    dh = float(rng.choice([100.0, 200.0]))
    media = ai.layered_media(nx, ny, nz, dh, seed=seed, pert_std=0.05, corr_len=5 * dh)
    dt = ai.stable_dt(media, dh, 0.4)
    p = awpsgt.make_params(nx, ny, nz, dh, dt, nt, igreen=comps, nd=min(10, nx // 4), socalq=1, ntiskp_sgt=5,
                           write_step=(nt // 5), precision=precision, kernel=kernel)
    src = (nx // 2, ny // 2, max(1, nz // 4))
    sources = [([src], ai.gaussian_derivative_stf(nt, dt, f0=0.1 / dt / 20, column=c - 1)) for c in comps]
    pts = ai.sgt_points(nx, ny, min(nz, 10), 40, seed=seed)
    return p, media, sources, pts


def run_alone(p, media, sources, pts):
    with awpsgt.Solver(p) as s:
        s.load_media(media)
        for q, (xyz, stf) in enumerate(sources):
            s.set_source(q, xyz, stf)
        s.set_points(pts)
        return s.run(p.nt, with_sgt=True)


REQS = [(1, (64, 48, 40), (1,), 120), (2, (96, 80, 48), (1, 2), 90), (3, (40, 40, 32), (1, 2, 3), 150),
        (4, (128, 96, 64), (2,), 60), (5, (50, 60, 36), (3, 1), 100), (6, (72, 72, 40), (1,), 80)]


@pytest.mark.parametrize("policy,fill", [("fifo", 0.0), ("sjf", 1.0e6), ("fifo_srpt", 0.0)])
def test_mix_equals_alone(policy, fill):
    reqs = [make_request(*r) for r in REQS]
    alone = [run_alone(*r) for r in reqs]
    with awpsgt.Server(max_active=4, chunk_steps=20) as sv:
        sv.configure(policy, fill, 2.0e6)
        ids = []
        for r in reqs:
            ids.append(sv.submit(*r))
            time.sleep(0.01)
        for k, rid in enumerate(ids):
            info, out = sv.wait(rid, timeout=600)
            assert awpsgt.REQ_STATE[info["state"]] == "done", info
            assert info["t_done"] >= info["t_admit"] >= info["t_submit"]
            assert np.array_equal(out.view(np.uint32), alone[k].view(np.uint32)), k


def test_budget_serialises_admission():
    reqs = [make_request(*r) for r in REQS[:3]]
    biggest = max(awpsgt.footprint_bytes(r[0], 40) for r in reqs)
    with awpsgt.Server(hbm_budget=int(biggest * 1.05), max_active=8, chunk_steps=25) as sv:
        ids = [sv.submit(*r) for r in reqs]
        infos = [sv.wait(i, timeout=600)[0] for i in ids]
    for a, b in zip(infos, infos[1:]):
        assert b["t_admit"] >= a["t_done"] - 1e-6     # one request resident at a time
    assert all(awpsgt.REQ_STATE[i["state"]] == "done" for i in infos)


def test_oversized_request_rejected():
    r = make_request(*REQS[0])
    with awpsgt.Server(hbm_budget=1 << 20) as sv:
        with pytest.raises(awpsgt.AwpError) as e:
            sv.submit(*r)
        assert e.value.status == 8


def test_cancel_queued_and_running():
    big = make_request(7, (160, 160, 80), (1, 2, 3), 3000)
    small = make_request(8, (40, 40, 32), (1,), 40)
    with awpsgt.Server(max_active=1, chunk_steps=10) as sv:
        a = sv.submit(*big)
        b = sv.submit(*small)
        sv.cancel(b)
        time.sleep(0.5)
        sv.cancel(a)
        ia, _ = sv.wait(a, timeout=120)
        ib, _ = sv.wait(b, timeout=120)
    assert awpsgt.REQ_STATE[ia["state"]] == "cancelled"
    assert awpsgt.REQ_STATE[ib["state"]] == "cancelled"


def test_sjf_admits_least_work_first():
    blocker = make_request(9, (160, 160, 80), (1,), 1500)
    big = make_request(10, (96, 96, 64), (1, 2), 400)
    small = make_request(11, (40, 40, 32), (1,), 40)
    with awpsgt.Server(max_active=1, chunk_steps=10) as sv:
        sv.configure("sjf")
        ids = [sv.submit(*r) for r in (blocker, big, small)]
        infos = [sv.wait(i, timeout=600)[0] for i in ids]
    assert all(awpsgt.REQ_STATE[i["state"]] == "done" for i in infos)
    assert infos[2]["t_admit"] < infos[1]["t_admit"]       # the small one overtook the big one
    assert infos[2]["t_admit"] > infos[0]["t_admit"]


def test_configure_rejects_unknown_policy():
    with awpsgt.Server() as sv:
        with pytest.raises(awpsgt.AwpError) as e:
            sv.lib.awp_server_configure(sv.h, 7, 0.0, 0.0) and awpsgt._check(sv.lib.awp_server_configure(sv.h, 7, 0.0, 0.0))
        assert e.value.status == 2
