"""The PML absorbing boundary (NPC = 1; AWP-ODC-SGT/src/pml.f).

CPU, the oracle's restatement of pml.f (no reference run can pin it: the
Fortran cannot be built here and the CUDA variant has no PML):
* a wave leaving a homogeneous box is absorbed and the solve stays stable;
* the restatements of opposite faces agree: the split of a source's energy
  between the west and east layers (and south and north) follows that of the
  Cerjan run, whose sponge treats the faces alike (a wrong coefficient,
  profile or difference in one face's routines shows as a changed split or a
  blow-up);
* before the wave reaches the layers the interior matches the Cerjan run.

GPU: the two-sweep and staged steppers with the PML kernels equal the FP32
oracle bit for bit -- every wavefield and stress everywhere, the memory
variables in the interior zone (in the PML zones the sweeps leave values
there that nothing reads; the oracle leaves zeros), CHKJ and the SGT image;
a checkpointed PML solve resumes bit for bit; the drop-in driver runs an
IN3D with NPC 1.
"""
import os
import subprocess

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt
import oracle

from test_gpu_parity import Case, bits_equal, first_diff, rel_l2

STATE = oracle.FIELDS[:15]


def box_energy(o, nd):
    u, v, w = (o.field(f)[2:-2, 2:-2, 2:-2].astype(np.float64) for f in ("u1", "v1", "w1"))
    e = u * u + v * v + w * w          # [z][y][x]
    return e.sum(), e[:, :, :nd].sum(), e[:, :, -nd:].sum(), e[:, :nd, :].sum(), e[:, -nd:, :].sum()


def pml_oracle(n=40, nz=36, nd=8, nt=400, igreen=1, pht=0.1):
    media = ai.homogeneous_media(n, n, nz)
    o = oracle.Oracle(nx=n, ny=n, nz=nz, dh=200.0, dt=0.01, nt=nt, nst=nt, nd=nd, arbc=0.92, socalq=1,
                      ntiskp_sgt=10, write_step=nt // 10, igreen=igreen, npc=1, pht=pht)
    o.load_media(media)
    o.set_source([(n // 2, n // 2, nz // 2)], ai.gaussian_derivative_stf(nt, 0.01, f0=2.0, column=igreen - 1))
    o.set_points(np.array([[5, 5, 5]], np.int32))
    return o


@pytest.mark.parametrize("igreen", [1, 3])
def test_oracle_pml_absorbs_and_stays_stable(igreen):
    nd = 8
    o = pml_oracle(igreen=igreen, nd=nd)
    hist = []
    for _ in range(20):
        o.run(20)
        hist.append(box_energy(o, nd))
    o.close()
    tot = np.array([h[0] for h in hist])
    assert np.isfinite(tot).all()
    peak = tot.argmax()
    assert peak < len(tot) - 5
    assert tot[-1] < 2e-2 * tot[peak]                   # the wave has left through the layers
    assert np.all(np.diff(tot[peak + 2:]) < 0)           # and nothing comes back


def layer_ratios(npc, igreen, n=40, nz=36, nd=8, steps=(80, 120, 160)):
    """South/north and west/east energy ratios of u, v, w in the layers."""
    media = ai.homogeneous_media(n, n, nz)
    o = oracle.Oracle(nx=n, ny=n, nz=nz, dh=200.0, dt=0.01, nt=200, nst=200, nd=nd, arbc=0.92, socalq=1,
                      ntiskp_sgt=10, write_step=20, igreen=igreen, npc=npc, pht=0.1)
    o.load_media(media)
    o.set_source([(n // 2, n // 2, nz // 2)], ai.gaussian_derivative_stf(200, 0.01, f0=2.0, column=igreen - 1))
    o.set_points(np.array([[5, 5, 5]], np.int32))
    out, done = [], 0
    for t in steps:
        o.run(t - done)
        done = t
        _, w, e, s_, n_ = box_energy(o, nd)
        out += [s_ / n_, w / e]
    o.close()
    return np.array(out)


@pytest.mark.parametrize("igreen", [1, 2, 3])
def test_oracle_pml_treats_opposite_faces_alike(igreen):
    """The energy a source sends into the south against the north layer (and
    west against east) depends on where it sits on the staggered grid; the
    PML must not change that split: its ratios follow the Cerjan run's,
    whose sponge treats the faces alike by construction.  A wrong
    coefficient, profile or difference in one face's routines breaks this."""
    pml, crj = layer_ratios(1, igreen), layer_ratios(0, igreen)
    assert np.all((pml / crj > 0.8) & (pml / crj < 1.25)), (pml, crj)


def test_oracle_pml_interior_matches_cerjan_early():
    """Before the wave reaches the layers, PML and Cerjan runs agree in the
    interior to FP32 rounding (the interior operators are the same; the
    boundaries differ only below the signal)."""
    n, nz, nd, nt = 40, 36, 8, 30
    media = ai.homogeneous_media(n, n, nz)
    outs = []
    for npc in (0, 1):
        o = oracle.Oracle(nx=n, ny=n, nz=nz, dh=200.0, dt=0.01, nt=nt, nst=nt, nd=nd, arbc=0.92, socalq=1,
                          ntiskp_sgt=10, write_step=1, igreen=1, npc=npc)
        o.load_media(media)
        o.set_source([(n // 2, n // 2, nz // 2)], ai.gaussian_derivative_stf(nt, 0.01, f0=2.0))
        o.set_points(np.array([[5, 5, 5]], np.int32))
        o.run(nt)
        outs.append(o.field("u1")[nd + 6:-nd - 6, nd + 6:-nd - 6, nd + 6:-nd - 6].copy())
        o.close()
    assert np.abs(outs[0]).max() > 0
    assert rel_l2(outs[1], outs[0]) <= 1e-6


# --------------------------------------------------------------------------- GPU

class PmlCase(Case):
    def __init__(self, **kw):
        kw.setdefault("nd", 6)
        super().__init__(**kw)

    def kw(self):
        k = super().kw()
        k.update(npc=1, pht=0.1)
        return k


def assert_same_state_pml(s, o, c, q=0):
    nd = c.nd
    bad = []
    for f in STATE:
        a, b = s.field(f, q), o.field(f)
        if f.startswith("r"):          # the memory variables of the interior zone
            a = a[nd + 2:c.nz + 2, nd + 2:c.ny + 2 - nd, nd + 2:c.nx + 2 - nd]
            b = b[nd + 2:c.nz + 2, nd + 2:c.ny + 2 - nd, nd + 2:c.nx + 2 - nd]
        if not bits_equal(a, b):
            bad.append((f, first_diff(a, b), rel_l2(a, b)))
    assert not bad, bad
    assert bits_equal(s.chkj(q), o.chkj())
    assert bits_equal(s.sgt(q), o.sgt())


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["staged", "two_sweep", "staged_fma"])
@pytest.mark.parametrize("igreen", [(1,), (1, 2, 3)])
def test_pml_bit_exact_with_oracle(kernel, igreen):
    c = PmlCase(nx=44, ny=36, nz=30, nt=60, igreen=igreen, srcs=[[(22, 18, 12)]] * len(igreen))
    s = c.gpu(kernel=kernel)
    for q in range(len(igreen)):
        o = c.oracle(q)
        if kernel == "staged_fma":     # contraction: within FP32 rounding, not bit for bit
            assert rel_l2(s.sgt(q), o.sgt()) <= 1e-5
            continue
        assert_same_state_pml(s, o, c, q)
        assert np.abs(o.sgt()).max() > 0
    s.close()


@pytest.mark.gpu
def test_pml_odd_sizes_and_sources_in_the_layers():
    c = PmlCase(nx=37, ny=29, nz=23, nt=45, nd=5, srcs=[[(3, 4, 2)]], ntiskp=3, write_step=7,
                pts=[(1, 1, 1), (37, 29, 23), (3, 4, 2), (20, 15, 1)])
    s = c.gpu(kernel="staged")
    assert_same_state_pml(s, c.oracle(), c)
    s.close()


@pytest.mark.gpu
def test_pml_rejected_with_fused_stepper_and_16bit_media():
    c = PmlCase(nt=10)
    with pytest.raises(awpsgt.AwpError) as e:
        c.gpu(kernel="fused")
    assert awpsgt.STATUS[e.value.status] == "AWP_ERR_PARAM"
    with pytest.raises(awpsgt.AwpError):
        c.gpu(precision="bf16", kernel="two_sweep")


@pytest.mark.gpu
def test_pml_checkpoint_resume(tmp_path):
    c = PmlCase(nx=40, ny=34, nz=28, nt=40, igreen=(1, 2), srcs=[[(20, 17, 10)]] * 2)
    full = c.gpu(kernel="staged")
    want = [full.sgt(q).view(np.uint32).copy() for q in range(2)]
    full.close()
    s = c.gpu(steps=17, kernel="staged")
    s.checkpoint_write(str(tmp_path))
    s.close()
    for q in range(2):
        for kind in ("ckpew", "ckpns", "ckpb"):
            assert (tmp_path / ("%s%07d%07d.bin" % (kind, q, 17))).exists()
    p = awpsgt.make_params(c.nx, c.ny, c.nz, c.dh, c.dt, c.nt, igreen=c.igreen, kernel="staged", **c.kw())
    with awpsgt.Solver(p) as s:
        s.load_media(c.media)
        for q in range(2):
            s.set_source(q, c.srcs[q], c.stfs[q])
        s.set_points(c.pts)
        assert s.checkpoint_read(str(tmp_path)) == 17
        s.run(c.nt)
        for q in range(2):
            assert np.array_equal(s.sgt(q).view(np.uint32), want[q])


@pytest.mark.gpu
def test_pmcl3d_runs_npc1(tmp_path):
    from test_pmcl3d import NST, in3d, write_inputs
    media, stf, pts = write_inputs(tmp_path)
    w = in3d(tmp_path)
    w.npc = 1
    w.pht = 0.1
    w.write(str(tmp_path / "IN3D"))
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    got = np.fromfile(tmp_path / "out" / "sgt" / "awp-strain", dtype=np.float32)
    o = oracle.Oracle(nx=48, ny=40, nz=32, dh=200.0, dt=0.01, nt=NST + 1, nst=NST, nd=8, fl=0.01, fh=25.0, fp=0.5,
                      socalq=1, ntiskp_sgt=5, write_step=3, igreen=1, npc=1, pht=0.1)
    o.load_media(media)
    o.set_source([(24, 20, 9)], stf)
    o.set_points(pts)
    o.run(NST + 1)
    assert np.array_equal(got.view(np.uint32), o.sgt().view(np.uint32))
    assert "PML=1 OR CERJAN=0:    1" in (tmp_path / "out" / "CHKP").read_text()
