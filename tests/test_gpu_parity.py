"""Parity of the sm_100a stepper (through the C ABI) with the CPU oracle.

The FP32 stepper evaluates the Fortran expressions in the same order with one
rounding per operation, so the bar is bit-exactness: every field, the CHKJ
series and the raw SGT file image must equal the FP32 oracle's bit for bit.
Against the FP64 oracle the SGT relative-L2 error must stay <= 1e-4.
"""
import numpy as np
import pytest

import awp_inputs as ai
import awpsgt
import oracle

pytestmark = pytest.mark.gpu

ALL_FIELDS = oracle.FIELDS


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def first_diff(a, b):
    d = np.argwhere(np.asarray(a, np.float32).view(np.uint32) != np.asarray(b, np.float32).view(np.uint32))
    return d[0].tolist() if len(d) else None


class Case:
    def __init__(self, nx=48, ny=40, nz=32, nt=50, dh=200.0, dt=0.01, igreen=(1,), srcs=None, npts=50,
                 media="layered", nvar=3, nve=1, mediastart=1, socalq=1, nd=8, ntiskp=5, write_step=4,
                 seed=3, pts=None, stf_seed=None):
        self.nx, self.ny, self.nz, self.nt = nx, ny, nz, nt
        self.dh, self.dt = dh, dt
        self.igreen = tuple(igreen)
        self.nvar, self.nve, self.mediastart, self.socalq, self.nd = nvar, nve, mediastart, socalq, nd
        self.ntiskp, self.write_step = ntiskp, write_step
        if media == "layered":
            m = ai.layered_media(nx, ny, nz, dh, seed=seed, pert_std=0.05, corr_len=1000.0)
        else:
            m = ai.homogeneous_media(nx, ny, nz)
        if nvar > 3:
            full = np.zeros((nz, ny, nx, nvar), np.float32)
            off = 3 if nvar == 8 else 0
            full[..., off:off + 3] = m
            full[..., off + 4] = 0.08 * m[..., 1]
            full[..., off + 3] = 1.7 * full[..., off + 4]
            m = full
        self.media = m
        if srcs is None:
            srcs = [[(nx // 2, ny // 2, nz // 3)] for _ in self.igreen]
        self.srcs = srcs
        rng = np.random.default_rng(7 if stf_seed is None else stf_seed)
        self.stfs = [rng.standard_normal((len(s), nt, 6)).astype(np.float32) * np.float32(1e12) for s in srcs]
        self.pts = ai.sgt_points(nx, ny, min(nz, 20), npts, seed=0) if pts is None else np.asarray(pts, np.int32)

    def kw(self):
        return dict(nd=self.nd, socalq=self.socalq, nve=self.nve, mediastart=self.mediastart, nvar=self.nvar,
                    ntiskp_sgt=self.ntiskp, write_step=self.write_step, fl=0.01, fh=25.0, fp=0.5)

    def gpu(self, steps=None, precision="f32", split=None, kernel="auto"):
        p = awpsgt.make_params(self.nx, self.ny, self.nz, self.dh, self.dt, self.nt, igreen=self.igreen,
                               precision=precision, kernel=kernel, **self.kw())
        s = awpsgt.Solver(p)
        s.load_media(self.media if self.mediastart else None)
        for q in range(len(self.igreen)):
            s.set_source(q, self.srcs[q], self.stfs[q])
        s.set_points(self.pts)
        n = self.nt if steps is None else steps
        if split:
            done = 0
            for c in split:
                s.run(c)
                done += c
            s.run(n - done)
        else:
            s.run(n)
        return s

    def oracle(self, q=0, steps=None, precision="f32", rstore="f32"):
        o = oracle.Oracle(nx=self.nx, ny=self.ny, nz=self.nz, dh=self.dh, dt=self.dt, nt=self.nt,
                          igreen=self.igreen[q], precision=precision, rstore=rstore, **self.kw())
        o.load_media(self.media if self.mediastart else None)
        o.set_source(self.srcs[q], self.stfs[q])
        o.set_points(self.pts)
        o.run(self.nt if steps is None else steps)
        return o


def assert_same_state(s, o, q=0, fields=ALL_FIELDS):
    bad = []
    for f in fields:
        a, b = s.field(f, q), o.field(f)
        if not bits_equal(a, b):
            bad.append((f, first_diff(a, b), rel_l2(a, b)))
    assert not bad, bad
    assert bits_equal(s.chkj(q), o.chkj())
    assert bits_equal(s.sgt(q), o.sgt())


KERNELS = ["fused", "two_sweep", "staged"]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("igreen,src", [
    (1, (20, 22, 10)), (2, (28, 22, 1)), (3, (5, 5, 31)), (-2, (30, 20, 2)),
    (-1, (30, 20, 2)), (-1, (10, 11, 17)), (4, (10, 12, 1)), (5, (40, 30, 1)), (6, (28, 22, 1)),
])
def test_bit_exact_every_igreen(igreen, src, kernel):
    c = Case(igreen=(igreen,), srcs=[[src]])
    s = c.gpu(kernel=kernel)
    o = c.oracle()
    assert_same_state(s, o)
    if igreen != -1:
        assert np.abs(o.sgt()).max() > 0
    else:   # no SGT output for moment sources (pmcl3d.f:1536)
        assert np.abs(s.sgt()).max() == 0


@pytest.mark.parametrize("kernel", KERNELS)
def test_batched_components_match_individual_oracles(kernel):
    c = Case(nx=44, ny=36, nz=30, nt=40, igreen=(1, 2, 3),
             srcs=[[(22, 18, 8)], [(22, 18, 8)], [(22, 18, 8)]])
    s = c.gpu(kernel=kernel)
    for q in range(3):
        assert_same_state(s, c.oracle(q), q)


@pytest.mark.parametrize("kernel", KERNELS)
def test_odd_sizes_and_boundary_points(kernel):
    nx, ny, nz = 37, 19, 23
    pts = [(1, 1, 1), (nx, ny, nz), (1, ny, 1), (nx, 1, nz), (18, 9, 1), (18, 9, 1), (5, 7, 12)]
    c = Case(nx=nx, ny=ny, nz=nz, nt=45, nd=5, srcs=[[(18, 9, 6)]], pts=pts, ntiskp=3, write_step=7)
    assert_same_state(c.gpu(kernel=kernel), c.oracle())


@pytest.mark.parametrize("kernel,kstage,unroll,rpt", [("fused", None, None, None), ("staged", None, None, None),
                                                      ("staged", "8", "1", "1"), ("staged", "9", "2", "2"),
                                                      ("staged", "16", "1", "2"), ("staged", "9", "2", "2v"),
                                                      ("staged", "16", "1", "1v")])
def test_multi_tile_multi_chunk_grid(kernel, kstage, unroll, rpt, monkeypatch):
    """Several x/y tiles (partial ones at the high edges) and z chunks: halo
    recompute at the fused stepper's tile seams and redundant levels at its
    chunk seams; the staged stepper's tile halos, chunk prologues and ring
    reuse across many work items per block."""
    if kstage:
        monkeypatch.setenv("AWP_TUNE_KSTAGE", kstage)
    if unroll:
        monkeypatch.setenv("AWP_TUNE_UNROLL", unroll)
    if rpt:                               # "2v": two rows per thread in the velocity sweep too
        monkeypatch.setenv("AWP_TUNE_RPT", rpt[0])
        if rpt.endswith("v"):
            monkeypatch.setenv("AWP_TUNE_RPTV", "2")
    c = Case(nx=100, ny=30, nz=80, nt=25, nd=6, srcs=[[(50, 15, 40)]], ntiskp=5, write_step=5)
    assert_same_state(c.gpu(kernel=kernel), c.oracle())


@pytest.mark.parametrize("qslow,batch", [("0", "0"), ("1", "0"), ("1", "1"), ("1", "3")])
def test_staged_batched_components_many_items(qslow, batch, monkeypatch):
    """Three components as neighbouring work items (or one component over
    all tiles at a time, or side by side in one item of the stress sweep),
    8-level chunks, two tile rows per thread in both sweeps."""
    monkeypatch.setenv("AWP_TUNE_BATCH", batch)
    monkeypatch.setenv("AWP_TUNE_KSTAGE", "8")
    monkeypatch.setenv("AWP_TUNE_RPT", "2")
    monkeypatch.setenv("AWP_TUNE_RPTV", "2")
    monkeypatch.setenv("AWP_TUNE_QSLOW", qslow)
    c = Case(nx=70, ny=20, nz=41, nt=30, igreen=(1, 2, 3),
             srcs=[[(35, 10, 20)], [(34, 9, 20)], [(36, 11, 21)]])
    s = c.gpu(kernel="staged")
    for q in range(3):
        assert_same_state(s, c.oracle(q), q)


@pytest.mark.parametrize("kernel", KERNELS)
def test_elastic_scheme(kernel):
    c = Case(nve=0, nt=40)
    s, o = c.gpu(kernel=kernel), c.oracle()
    assert_same_state(s, o, fields=ALL_FIELDS[:9] + ALL_FIELDS[15:18])


def test_homogeneous_mediastart0():
    c = Case(mediastart=0, media="homogeneous", nt=40)
    assert_same_state(c.gpu(), c.oracle())


@pytest.mark.parametrize("nvar", [5, 8])
def test_media_with_q_columns(nvar):
    c = Case(nvar=nvar, nt=30)
    assert_same_state(c.gpu(), c.oracle())


def test_several_sources_same_cell_keep_order():
    srcs = [[(20, 20, 10), (20, 20, 10), (21, 20, 10)]]
    c = Case(igreen=(-2,), srcs=srcs, nt=30)
    assert_same_state(c.gpu(), c.oracle())


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("ntiskp", [5, 4])
def test_split_runs_and_partial_sgt_chunk(kernel, ntiskp):
    # 53 steps, NTISKP 5 -> 10 samples, WRITE_STEP 4 -> 2 full chunks written;
    # an odd period makes the graphs alternate buffer parity
    c = Case(nt=53, ntiskp=ntiskp, write_step=4)
    s = c.gpu(split=[3, 11, 20], kernel=kernel)
    assert_same_state(s, c.oracle())


def test_reset_reproduces_run():
    c = Case(nt=35)
    s = c.gpu()
    a = s.sgt().copy()
    s.reset()
    s.run(c.nt)
    assert bits_equal(s.sgt(), a)


def test_fp64_error_budget():
    c = Case(nt=80, stf_seed=11)
    s = c.gpu()
    o64 = c.oracle(precision="f64")
    err = rel_l2(s.sgt(), o64.sgt())
    assert err <= 1e-4, err


@pytest.mark.parametrize("precision", ["bf16", "f16", "mixed"])
@pytest.mark.parametrize("kernel", KERNELS)
def test_mixed_precision_runs_close_to_fp64(precision, kernel):
    """Media and memory variables in 16 bits, wavefields and arithmetic FP32:
    the SGT stays close to the FP64 oracle (the bound here is loose; the
    measured errors are reported by the error study)."""
    c = Case(nt=80, stf_seed=11)
    if kernel == "staged" and precision != "mixed":
        # the staged stepper reads FP32 media: asking for it with 16-bit media
        # is a parameter error, not a silent switch to another stepper
        with pytest.raises(awpsgt.AwpError) as e:
            c.gpu(precision=precision, kernel=kernel)
        assert awpsgt.STATUS[e.value.status] == "AWP_ERR_PARAM"
        return
    s = c.gpu(precision=precision, kernel=kernel)
    o64 = c.oracle(precision="f64")
    g = s.sgt()
    assert np.isfinite(g).all()
    err = rel_l2(g, o64.sgt())
    assert err <= 2e-2, err


# storage of r1..r6 in the device modes with FP32 media -> the oracle's emulation of it
RSTORE = {"mixed": "bf16", "bfp": "bfp33"}


@pytest.mark.parametrize("precision", ["mixed", "bfp"])
@pytest.mark.parametrize("kernel", KERNELS)
def test_16bit_memory_variables_bit_exact(precision, kernel):
    """FP32 media with r1..r6 in 16 bits (bf16, or block floating point) are
    bit-exact with the FP32 oracle storing r1..r6 in the same format: every
    field (memory variables decoded), CHKJ and the SGT image."""
    c = Case(nx=44, ny=36, nz=30, nt=40, igreen=(1, 2, 3), srcs=[[(22, 18, 8)], [(22, 18, 8)], [(22, 18, 8)]])
    s = c.gpu(kernel=kernel, precision=precision)
    for q in range(3):
        assert_same_state(s, c.oracle(q, rstore=RSTORE[precision]), q)


@pytest.mark.parametrize("qslow,batch,rpt", [("0", "0", "1"), ("1", "0", "2"), ("1", "1", "1")])
def test_bfp_staged_shapes_bit_exact(qslow, batch, rpt, monkeypatch):
    monkeypatch.setenv("AWP_TUNE_QSLOW", qslow)
    monkeypatch.setenv("AWP_TUNE_BATCH", batch)
    monkeypatch.setenv("AWP_TUNE_RPT", rpt)
    monkeypatch.setenv("AWP_TUNE_KSTAGE", "9")
    c = Case(nx=70, ny=20, nz=41, nt=30, igreen=(1, 2), srcs=[[(35, 10, 20)], [(30, 12, 33)]], ntiskp=3,
             write_step=5)
    s = c.gpu(kernel="staged", precision="bfp")
    for q in range(2):
        assert_same_state(s, c.oracle(q, rstore="bfp33"), q)


def test_bfp_error_budget():
    """Block floating point r1..r6 stays within the 1e-4 SGT budget of FP64."""
    c = Case(nt=80, stf_seed=11)
    err = rel_l2(c.gpu(precision="bfp").sgt(), c.oracle(precision="f64").sgt())
    assert err <= 1e-4, err


def test_mixed_mode_same_result_staged_and_two_sweep():
    c = Case(nt=40)
    a = c.gpu(precision="mixed", kernel="staged").sgt()
    b = c.gpu(precision="mixed", kernel="two_sweep").sgt()
    assert bits_equal(a, b)


def test_mixed_precision_same_result_both_kernels():
    c = Case(nt=40)
    a = c.gpu(precision="f16", kernel="fused").sgt()
    b = c.gpu(precision="f16", kernel="two_sweep").sgt()
    assert bits_equal(a, b)


def test_config1_full_run_bit_exact():
    """Workload 1 (160x160x80, h=200 m, dt=0.01 s, 1000 steps,
    homogeneous half-space, fx at the centre 2 km deep, 1000 SGT points,
    every 10 steps) against the FP32 oracle, and its FP64 error."""
    w = ai.config(1)
    media = w.media()
    pts = w.points()
    stf = w.stf(0)
    kw = dict(nd=20, arbc=0.92, fl=0.01, fh=25.0, fp=0.5, socalq=1, ntiskp_sgt=10, write_step=100)
    p = awpsgt.make_params(w.nx, w.ny, w.nz, w.dh, w.dt, w.nt, igreen=(1,), nst=w.nst, **kw)
    with awpsgt.Solver(p) as s:
        s.load_media(media)
        s.set_source(0, [w.src_xyz], stf)
        s.set_points(pts)
        gpu = s.run(w.nt, with_sgt=True)[0]
        chkj = s.chkj()
    o = oracle.Oracle(nx=w.nx, ny=w.ny, nz=w.nz, dh=w.dh, dt=w.dt, nt=w.nt, nst=w.nst, igreen=1, **kw)
    o.load_media(media)
    o.set_source([w.src_xyz], stf)
    o.set_points(pts)
    o.run(w.nt)
    ref = o.sgt()
    assert gpu.size == 1000 * 6 * 100
    assert np.abs(ref).max() > 0
    assert bits_equal(gpu, ref), rel_l2(gpu, ref)
    assert bits_equal(chkj, o.chkj())


def kinematic_rupture(n, seed=5, dt=0.01):
    """n subfaults: rows [type slip t_rupture t_rise area 0] [strike dip rake 0 0 0],
    the three slip-rate functions in turn."""
    rng = np.random.default_rng(seed)
    t = np.zeros((n, 2, 6), np.float32)
    t[:, 0, 0] = 1 + np.arange(n) % 3
    t[:, 0, 1] = rng.uniform(0.5, 2.0, n)                 # slip (m)
    t[:, 0, 2] = rng.uniform(0.0, 15 * dt, n)             # rupture time (s)
    t[:, 0, 3] = rng.uniform(5 * dt, 20 * dt, n)          # rise time (s)
    t[:, 0, 4] = rng.uniform(1e4, 4e4, n)                 # area (m^2)
    t[:, 1, 0] = rng.uniform(0.0, 360.0, n)               # strike, dip, rake (degrees)
    t[:, 1, 1] = rng.uniform(10.0, 90.0, n)
    t[:, 1, 2] = rng.uniform(-180.0, 180.0, n)
    return t


@pytest.mark.parametrize("kernel", ["staged", "two_sweep"])
def test_kinematic_source_matches_oracle(kernel):
    """IFAULT=5: subfault moment rates inserted after every stress update.  The
    CUDA and C-library sinf/cosf/expf/powf differ in the last bits, so the
    bar is a tolerance (rel-L2 <= 1e-5 against the FP32 oracle, <= 1e-4
    against FP64), not bit equality."""
    nx, ny, nz, nt, dt = 48, 40, 32, 60, 0.01
    xyz = [(16 + 2 * k, 20 + (k % 3), 12 + (k % 4)) for k in range(12)] + [(20, 20, 12)]   # one shared cell
    tab = kinematic_rupture(len(xyz), dt=dt)
    media = ai.layered_media(nx, ny, nz, 200.0, seed=3, pert_std=0.05, corr_len=1000.0)
    pts = ai.sgt_points(nx, ny, 20, 50, seed=0)
    kw = dict(nd=8, socalq=1, ntiskp_sgt=5, write_step=4, fl=0.01, fh=25.0, fp=0.5)
    p = awpsgt.make_params(nx, ny, nz, 200.0, dt, nt, nst=2, igreen=(1,), kernel=kernel, kinematic=1, **kw)
    with awpsgt.Solver(p) as s:
        s.load_media(media)
        s.set_source(0, xyz, tab)
        s.set_points(pts)
        s.run(nt)
        g = s.sgt(0)
        gxx = s.field("xx")
    refs = {}
    for prec in ("f32", "f64"):
        o = oracle.Oracle(nx=nx, ny=ny, nz=nz, dh=200.0, dt=dt, nt=nt, nst=2, igreen=1, kinematic=1,
                          precision=prec, **kw)
        o.load_media(media)
        o.set_source(xyz, tab)
        o.set_points(pts)
        o.run(nt)
        refs[prec] = (o.sgt(), o.field("xx"))
    assert np.abs(g).max() > 0
    assert rel_l2(g, refs["f32"][0]) <= 1e-5
    assert rel_l2(gxx, refs["f32"][1]) <= 1e-5
    assert rel_l2(g, refs["f64"][0]) <= 1e-4



@pytest.mark.parametrize("precision", ["f32", "bfp"])
def test_staged_fma_within_fp32_rounding_of_oracle(precision):
    """The staged sweeps compiled with multiply-add contraction: every field
    and the SGT image within 1e-5 relative L2 of the FP32 oracle (the memory
    variables within 1e-4: a block-floating-point rounding can land one
    quantum apart), the SGT point layout unchanged, and the FP64 budget of
    1e-4 met."""
    c = Case(nx=44, ny=36, nz=30, nt=60, igreen=(1, 2, 3), srcs=[[(22, 18, 8)], [(20, 16, 12)], [(24, 19, 9)]],
             stf_seed=11)
    s = c.gpu(kernel="staged_fma", precision=precision)
    for q in range(3):
        o = c.oracle(q, rstore=RSTORE.get(precision, "f32"))
        for f in ALL_FIELDS[:15]:
            err = rel_l2(s.field(f, q), o.field(f))
            assert err <= (1e-4 if f.startswith("r") else 1e-5), (q, f, err)
        g, ref = s.sgt(q), o.sgt()
        assert g.shape == ref.shape and np.array_equal(g == 0, ref == 0)
        assert rel_l2(g, ref) <= 1e-5
        assert rel_l2(g, c.oracle(q, precision="f64").sgt()) <= 1e-4
