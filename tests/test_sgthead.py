"""SgtHead formats on either side of the stepper: the RWG header file, the RWG
component order of the SGTs, and AWP media built from RWG velocity volumes.

Golden fixtures (tests/golden/sgthead, made by the reference's own write_head,
reformat_awp and reformat_velocity, see make_sgthead_golden.py) pin the header
writer byte for byte and the oracle's restatements of the two transforms;
where the reference tools have been built into oracle/_ref, more header cases
are compared live.  The GPU tests check the device transforms (awp_get_sgt_rwg,
the reformat_awp and reformat_velocity tools, awp_load_media_rwg) against
those fixtures and restatements."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "sgthead")
REF = os.path.join(ROOT, "oracle", "_ref")
CASES = json.load(open(os.path.join(GOLD, "cases.json")))


def run_write_head(exe, cwd, args):
    return subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("case", CASES["headers"], ids=lambda c: c["name"])
def test_header_writer_matches_reference_bytes(case, tmp_path):
    src = os.path.join(GOLD, case["name"])
    for f in os.listdir(src):
        if f != "expected.sgthead":
            shutil.copy(os.path.join(src, f), tmp_path / f)
    r = run_write_head(awpsgt.WRITE_HEAD_PATH, tmp_path, case["args"])
    assert r.returncode == 0, r.stderr
    got = np.fromfile(tmp_path / "expected.sgthead", dtype=np.uint8)
    ref = np.fromfile(os.path.join(src, "expected.sgthead"), dtype=np.uint8)
    assert got.size == ref.size and np.array_equal(got, ref)
    m, ix, hd = awpsgt.read_sgt_header(str(tmp_path / "expected.sgthead"))
    assert m["globnp"] == len(ix) == len(hd) > 0 and m["geoproj"] == 1
    assert np.all(hd["lam"] > 0) and np.all(hd["mu"] > 0) and np.all(hd["rho"] > 0)


def test_header_through_c_abi(tmp_path):
    case = CASES["headers"][0]
    src = os.path.join(GOLD, case["name"])
    a = case["args"]
    awpsgt.write_sgt_header(str(tmp_path / "h"), *(os.path.join(src, x) for x in a[:4]), float(a[4]), int(a[5]),
                            float(a[6]), int(a[7]), a[8], float(a[9]), float(a[10]), os.path.join(src, a[11]),
                            mu_corr=len(a) > 13)
    assert np.array_equal(np.fromfile(tmp_path / "h", np.uint8),
                          np.fromfile(os.path.join(src, "expected.sgthead"), np.uint8))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "write_head")), reason="reference tools not built here")
@pytest.mark.parametrize("seed,grid,comp,corr,rot", [(11, (40, 30, 20), "y", True, -30.0),
                                                     (12, (64, 48, 30), "x", False, -55.0),
                                                     (13, (9, 70, 5), "z", False, 88.0)])
def test_header_writer_against_live_reference(seed, grid, comp, corr, rot, tmp_path):
    p = ai.write_sgthead_inputs(str(tmp_path), *grid, 0.15, 150, seed=seed, mrot=rot)
    args = [p["modelbox"], p["coordfile"], p["fdloc"], p["gridout"], "0.15", "5000", "0.004", "10", comp, "1e20",
            "0.75", p["media"]]
    extra = ["-c"] if corr else []
    r1 = run_write_head(os.path.join(REF, "write_head"), tmp_path, args + ["ref.h"] + extra)
    r2 = run_write_head(awpsgt.WRITE_HEAD_PATH, tmp_path, args + ["our.h"] + extra)
    assert r1.returncode == 0 and r2.returncode == 0, r2.stderr
    assert np.array_equal(np.fromfile(tmp_path / "ref.h", np.uint8), np.fromfile(tmp_path / "our.h", np.uint8))


def test_header_writer_reports_bad_inputs(tmp_path):
    case = CASES["headers"][0]
    src = os.path.join(GOLD, case["name"])
    for f in os.listdir(src):
        shutil.copy(os.path.join(src, f), tmp_path / f)
    os.remove(tmp_path / "media")
    r = run_write_head(awpsgt.WRITE_HEAD_PATH, tmp_path, case["args"])
    assert r.returncode != 0 and "media" in r.stderr
    shutil.copy(os.path.join(src, "media"), tmp_path / "media")
    lines = open(tmp_path / "coordfile").read().splitlines()
    lines[-1] = "999 0 0 1 0 0 0"                  # outside the grid
    open(tmp_path / "coordfile", "w").write("\n".join(lines) + "\n")
    r = run_write_head(awpsgt.WRITE_HEAD_PATH, tmp_path, case["args"])
    assert r.returncode != 0 and "point record" in r.stderr
    r = subprocess.run([awpsgt.WRITE_HEAD_PATH], capture_output=True, text=True)
    assert r.returncode != 0 and "Usage" in r.stdout


@pytest.mark.parametrize("case", CASES["reformat"], ids=lambda c: c["name"])
def test_oracle_reorder_matches_reference_tool(case):
    d = os.path.join(GOLD, case["name"])
    src = np.fromfile(os.path.join(d, "in.sgt"), np.float32)
    ref = np.fromfile(os.path.join(d, "expected.sgt"), np.float32)
    got = oracle.reorder_rwg(src, case["nt"], case["z"])
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES["reformat"], ids=lambda c: c["name"])
def test_reformat_tool_on_gpu_matches_reference(case, tmp_path):
    d = os.path.join(GOLD, case["name"])
    args = [os.path.join(d, "in.sgt"), str(case["nt"]), str(tmp_path / "out.sgt")] + (["-z"] if case["z"] else [])
    r = subprocess.run([awpsgt.REFORMAT_AWP_PATH] + args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(tmp_path / "out.sgt", np.float32)
    ref = np.fromfile(os.path.join(d, "expected.sgt"), np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("z", [False, True])
def test_device_rwg_image_matches_oracle_reorder(z):
    nx, ny, nz, nt = 48, 40, 32, 61
    media = ai.layered_media(nx, ny, nz, 200.0, seed=6, pert_std=0.05, corr_len=1000.0)
    p = awpsgt.make_params(nx, ny, nz, 200.0, 0.01, nt, igreen=(3 if z else 1,), nd=8, socalq=1, ntiskp_sgt=5,
                           write_step=4)
    with awpsgt.Solver(p) as s:
        s.load_media(media)
        s.set_source(0, [(24, 20, 9)], ai.gaussian_derivative_stf(nt, 0.01, f0=1.0, column=2 if z else 0))
        s.set_points(ai.sgt_points(nx, ny, 20, 30, seed=1))
        s.run(nt)
        awp = s.sgt(0)
        rwg = s.sgt_rwg(0, z_source=z)
    ntf = awp.size // (30 * 6)
    assert np.abs(awp).max() > 0
    assert np.array_equal(rwg.view(np.uint32), oracle.reorder_rwg(awp, ntf, z).view(np.uint32))
    host = awpsgt.sgt_reorder_rwg(awp, ntf, z)
    assert np.array_equal(host.view(np.uint32), rwg.view(np.uint32))


@pytest.mark.parametrize("case", CASES["velocity"], ids=lambda c: c["name"])
def test_oracle_velocity_reformat_matches_reference_tool(case):
    d = os.path.join(GOLD, case["name"])
    vol = [np.fromfile(os.path.join(d, "v." + c), np.float32) for c in "psd"]
    got = oracle.rwg_to_awp_media(*vol, case["nx"], case["ny"], case["nz"])
    ref = np.fromfile(os.path.join(d, "expected.media"), np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES["velocity"], ids=lambda c: c["name"])
def test_reformat_velocity_tool_on_gpu_matches_reference(case, tmp_path):
    d = os.path.join(GOLD, case["name"])
    r = subprocess.run([awpsgt.REFORMAT_VELOCITY_PATH, str(case["nx"]), str(case["ny"]), str(case["nz"]),
                        os.path.join(d, "v"), str(tmp_path / "m")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(tmp_path / "m", np.float32)
    ref = np.fromfile(os.path.join(d, "expected.media"), np.float32)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_solver_media_from_rwg_volumes_equals_awp_file():
    case = CASES["velocity"][0]
    d = os.path.join(GOLD, case["name"])
    nx, ny, nz = case["ny"], case["nx"], case["nz"]          # AWP x is RWG y
    p = awpsgt.make_params(nx, ny, nz, 100.0, 0.005, 10, igreen=(1,), nd=3, socalq=1, ntiskp_sgt=1, write_step=5)
    fields = ("lam", "mu", "d1", "qp", "qs")
    with awpsgt.Solver(p) as a, awpsgt.Solver(p) as b:
        awpsgt._check(a.lib.awp_load_media_file(a.h, os.path.join(d, "expected.media").encode()))
        b.load_media_rwg(os.path.join(d, "v"))
        for f in fields:
            fa, fb = a.field(f), b.field(f)
            assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32)), f
