"""Checkpoint / restart (AWP-ODC-SGT/src/pmcl3d.f:1018-1097 read, 1967-2045 write).

A solve interrupted after any step, written with awp_checkpoint_write and
continued by a fresh solver through awp_checkpoint_read, must end with the
same SGT file image, CHKJ series and wavefield as the uninterrupted solve,
bit for bit: every stepper, odd steps (the fused stepper's second buffer),
several components, and memory variables stored in 16 bits.  The drop-in
driver resumes from output_ckp/ when IN3D sets CHECKPOINT.
"""
import os
import subprocess

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt

from test_pmcl3d import NST, in3d, oracle_sgt, write_inputs

NX, NY, NZ, NT = 48, 40, 32, 47


def make_solver(kernel, precision, ncomp):
    media = ai.layered_media(NX, NY, NZ, 200.0, seed=6, pert_std=0.05, corr_len=1000.0)
    p = awpsgt.make_params(NX, NY, NZ, 200.0, 0.01, NT, igreen=(1, 2, 3)[:ncomp], nd=8, socalq=1, ntiskp_sgt=5,
                           write_step=3, precision=precision, kernel=kernel)
    s = awpsgt.Solver(p)
    s.load_media(media)
    for q in range(ncomp):
        s.set_source(q, [(24, 20, 9)], ai.gaussian_derivative_stf(NT, 0.01, f0=1.0, column=q))
    s.set_points(ai.sgt_points(NX, NY, 20, 40, seed=1))
    return s


def bf16_rn(a):
    b = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32)


def state(s, ncomp):
    out = []
    for q in range(ncomp):
        out.append(s.sgt(q).view(np.uint32).copy())
        out.append(s.chkj(q).view(np.uint32).copy())
        for f in awpsgt.FIELDS[:15]:
            out.append(s.field(f, q).view(np.uint32).copy())
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("kernel,precision,ncomp,stop", [
    ("staged", "f32", 3, 23), ("staged", "f32", 1, 10), ("fused", "f32", 2, 23), ("two_sweep", "f32", 1, 17),
    ("staged", "mixed", 2, 19), ("two_sweep", "bf16", 1, 31), ("staged", "bfp", 3, 29), ("fused", "bfp", 1, 13)])
def test_resume_is_bitwise_equal(tmp_path, kernel, precision, ncomp, stop):
    with make_solver(kernel, precision, ncomp) as s:
        s.run(NT)
        want = state(s, ncomp)
    with make_solver(kernel, precision, ncomp) as s:
        s.run(stop)
        s.checkpoint_write(str(tmp_path))
    assert int((tmp_path / "ckp0000000.hdr").read_text()) == stop
    for q in range(ncomp):
        for kind in ("ckp", "ckpdy", "ckpsgt"):
            assert (tmp_path / ("%s%07d%07d.bin" % (kind, q, stop))).exists()
    with make_solver(kernel, precision, ncomp) as s:
        assert s.checkpoint_read(str(tmp_path)) == stop
        s.run(NT)                                   # runs the remaining NT - stop steps
        got = state(s, ncomp)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_checkpoint_file_holds_the_reference_records(tmp_path):
    """ckp<rank><step>.bin: five records of three padded arrays (u1 v1 w1,
    xx yy zz, xy xz yz, r1 r2 r3, r4 r5 r6); ckpdy: u2, broken, mu."""
    with make_solver("staged", "f32", 1) as s:
        s.run(12)
        s.checkpoint_write(str(tmp_path))
        nvol = (NX + 4) * (NY + 4) * (NZ + 4)
        raw = np.fromfile(tmp_path / "ckp00000000000012.bin", dtype=np.float32)
        assert raw.size == 15 * nvol
        for n, f in enumerate(awpsgt.FIELDS[:15]):
            assert np.array_equal(raw[n * nvol:(n + 1) * nvol].view(np.uint32), s.field(f).ravel().view(np.uint32))
        dy = np.fromfile(tmp_path / "ckpdy00000000000012.bin", dtype=np.float32)
        assert dy.size == 3 * nvol and not dy[:2 * nvol].any()
        assert np.array_equal(dy[2 * nvol:], s.field("mu").ravel())


@pytest.mark.gpu
def test_no_checkpoint_means_step_zero(tmp_path):
    with make_solver("staged", "f32", 1) as s:
        assert s.checkpoint_read(str(tmp_path)) == 0
        s.run(NT)


@pytest.mark.gpu
def test_checkpoint_of_another_solve_is_refused(tmp_path):
    with make_solver("staged", "f32", 1) as s:
        s.run(10)
        s.checkpoint_write(str(tmp_path))
    media = ai.layered_media(NX, NY, NZ, 200.0, seed=6)
    p = awpsgt.make_params(NX, NY, NZ, 200.0, 0.01, NT, igreen=(1,), nd=8, socalq=1, ntiskp_sgt=5, write_step=3)
    with awpsgt.Solver(p) as s:
        s.load_media(media)
        s.set_source(0, [(24, 20, 9)], ai.gaussian_derivative_stf(NT, 0.01))
        s.set_points(ai.sgt_points(NX, NY, 20, 7, seed=1))           # other points: another SGT image
        with pytest.raises(awpsgt.AwpError) as e:
            s.checkpoint_read(str(tmp_path))
        assert awpsgt.STATUS[e.value.status] == "AWP_ERR_IO"


@pytest.mark.gpu
def test_pmcl3d_resumes_from_output_ckp(tmp_path):
    """CHECKPOINT 20: the run writes output_ckp/ after steps 20 and 40; pointed
    back at step 20 and started again it resumes there and writes the same
    SGT file and CHKJ as the uninterrupted run and the oracle."""
    media, stf, pts = write_inputs(tmp_path)
    w = in3d(tmp_path)
    w.checkpoint = 20
    w.write(str(tmp_path / "IN3D"))
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    ck = tmp_path / "output_ckp"
    assert int((ck / "ckp0000000.hdr").read_text()) == 60
    for step in (20, 40, 60):
        assert (ck / ("ckp0000000%07d.bin" % step)).exists()
    first = (tmp_path / "out" / "sgt" / "awp-strain").read_bytes()
    chkj = (tmp_path / "out" / "CHKJ").read_text()
    os.remove(tmp_path / "out" / "sgt" / "awp-strain")
    (ck / "ckp0000000.hdr").write_text("          20\n")
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    assert "starting from step 20" in r.stdout
    assert (tmp_path / "out" / "sgt" / "awp-strain").read_bytes() == first
    assert (tmp_path / "out" / "CHKJ").read_text() == chkj
    ref = oracle_sgt(media, stf, pts).sgt()
    assert np.array_equal(np.frombuffer(first, np.uint32), ref.view(np.uint32))
    assert NST == 60


@pytest.mark.gpu
def test_set_field_round_trip():
    with make_solver("staged", "mixed", 1) as s:
        rng = np.random.default_rng(3)
        a = np.zeros((NZ + 4, NY + 4, NX + 4), np.float32)
        a[2:-2, 2:-2, 2:-2] = rng.uniform(-1, 1, (NZ, NY, NX)).astype(np.float32)
        s.set_field("xy", a)
        assert np.array_equal(s.field("xy"), a)
        s.set_field("r4", a)                         # bf16 storage: rounded to nearest even
        assert np.array_equal(s.field("r4"), bf16_rn(a))
        with pytest.raises(awpsgt.AwpError):
            s.set_field("mu", a)                     # media are not state


@pytest.mark.gpu
def test_set_field_block_floating_point():
    """Memory variables in block floating point: a value set comes back within
    2^-14 of its group's largest magnitude; setting what was read back leaves
    the stored words unchanged (checkpoint restore is exact)."""
    with make_solver("staged", "bfp", 1) as s:
        rng = np.random.default_rng(4)
        shape = (NZ + 4, NY + 4, NX + 4)
        vals = []
        for n, f in enumerate(("r1", "r2", "r3", "r4", "r5", "r6")):
            a = np.zeros(shape, np.float32)
            a[2:-2, 2:-2, 2:-2] = (rng.standard_normal((NZ, NY, NX)) * 10.0 ** (n - 2)).astype(np.float32)
            s.set_field(f, a)
            vals.append(a)
        got = [s.field(f) for f in ("r1", "r2", "r3", "r4", "r5", "r6")]
        for g0 in (0, 3):
            mx = np.maximum.reduce([np.abs(vals[g0 + a]) for a in range(3)])
            for a in range(3):
                assert np.all(np.abs(got[g0 + a] - vals[g0 + a]) <= mx * 2.0 ** -14)
        for f, a in zip(("r1", "r2", "r3", "r4", "r5", "r6"), got):
            s.set_field(f, a)
        for f, a in zip(("r1", "r2", "r3", "r4", "r5", "r6"), got):
            assert np.array_equal(s.field(f).view(np.uint32), a.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["staged", "fused"])
def test_get_plane_equals_the_field_level(kernel):
    """awp_get_plane returns level k of a wavefield or stress as it stands
    after the steps done so far: the fused stepper alternates between two
    buffers, so the level must come from the current one (odd and even step
    counts); memory variables and out-of-range levels are refused."""
    with make_solver(kernel, "f32", 2) as s:
        for steps in (7, 6):
            s.run(steps)
            for q in range(2):
                for f in ("u1", "w1", "zz", "xy"):
                    full = s.field(f, q)
                    for k in (1, NZ // 2, NZ):
                        assert np.array_equal(s.plane(f, k, q).view(np.uint32),
                                              full[k + 1, 2:NY + 2, 2:NX + 2].view(np.uint32))
            assert np.abs(s.plane("u1", NZ - 9, 0)).max() > 0
        for bad in (("r1", 1), ("u1", 0), ("u1", NZ + 1)):
            with pytest.raises(awpsgt.AwpError):
                s.plane(*bad)
