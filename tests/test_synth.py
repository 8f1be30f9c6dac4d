"""Reciprocity seismogram synthesis (DirectSynth's worker step) on the GPU
against the CPU oracle (oracle/synth_oracle.c), plus the SRF reader, the
oracle's own known-answer checks and the file paths.

The oracle restates jbsim3d_synth's loop (find_sgt, mech_sgt, sum_sgt /
timeshift_sgt, srf_stf / do_cnvlv) in the reference's order; the device path
must equal it bit for bit.  Both are pinned to DirectSynth's own functions:
tests/golden/synth holds seismograms those functions produced
(tests/golden/make_synth_golden.py, via oracle/_ref/libsynth_ref.so built by
oracle/Makefile.ref), and where that library is built the oracle is also
compared with it live."""
import hashlib
import json
import os

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt
import oracle


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "synth")
GOLD_CASES = json.load(open(os.path.join(GOLD, "cases.json")))


def golden_case(g):
    kw = dict(g["case"])
    if "nstf" in kw:
        kw["nstf"] = tuple(kw["nstf"])
    c = ai.synth_case(**kw)
    h = hashlib.sha256()
    for a in [c.master, c.index, c.headers] + list(c.comps):
        h.update(np.ascontiguousarray(a).tobytes())
    for p, q in c.variations:
        h.update(np.ascontiguousarray(p).tobytes())
        h.update(np.ascontiguousarray(q).tobytes())
    h.update(np.float32([c.slon, c.slat, c.dtout]).tobytes())
    assert h.hexdigest() == g["inputs_sha256"], "synth_case no longer makes the inputs the fixture was made from"
    return c, np.load(os.path.join(GOLD, g["name"] + ".npy"))


def case_seis(c, ntout=0, tstart=0.0):
    return oracle.synth(c.master, c.index, c.headers, c.comps, c.slon, c.slat, c.dtout, ntout, tstart,
                        c.variations)


# ---- pinning: the reference's own synthesis functions -----------------------

@pytest.mark.parametrize("g", GOLD_CASES, ids=lambda g: g["name"])
def test_oracle_matches_reference_fixtures(g):
    c, want = golden_case(g)
    got, _ = case_seis(c, g["ntout"], g["tstart"])
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsynth_ref.so")),
                    reason="reference synthesis functions not built here")
@pytest.mark.parametrize("seed,kw,ntout,tstart", [
    (31, dict(nv=4, mech2_frac=0.3, mech3_frac=0.2, jitter=0.45), 900, 0.7),
    (32, dict(ncomp=3, nv=2, drop_frac=0.5, nstf=(3, 200), nt=350), 0, -1.0),
    (33, dict(ncomp=1, nv=3, zero_frac=0.5, nx_f=16, nz_f=10), 300, 3.0)])
def test_oracle_matches_live_reference(seed, kw, ntout, tstart):
    c = ai.synth_case(seed=seed, **kw)
    got, _ = case_seis(c, ntout, tstart)
    want = oracle.synth_reference(c.master, c.index, c.headers, c.comps, c.slon, c.slat, c.dtout, ntout, tstart,
                                  c.variations)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


# ---- host side: SRF reader, grid lookup, the oracle's known answers ----------

@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("plane", [False, True])
def test_srf_reader_round_trip(tmp_path, binary, plane):
    c = ai.synth_case(seed=3, nv=1, mech2_frac=0.3, mech3_frac=0.2, zero_frac=0.1)
    pts, pool = c.variations[0]
    path = str(tmp_path / "r.srf")
    ai.write_srf(path, pts, pool, binary=binary, plane=plane)
    got, gpool = awpsgt.read_srf(path, binary=binary)
    assert len(got) == len(pts)
    for f in ("lon", "lat", "dep", "stk", "dip", "area", "tinit", "dt", "rake", "slip1", "slip2", "slip3",
              "nt1", "nt2", "nt3"):
        assert np.array_equal(got[f], pts[f]), f
    for c_ in (1, 2, 3):
        for a, b in zip(got, pts):
            n = int(a["nt%d" % c_])
            assert np.array_equal(gpool[a["stf%d" % c_]:a["stf%d" % c_] + n], pool[b["stf%d" % c_]:b["stf%d" % c_] + n])


def test_srf_reader_errors(tmp_path):
    with pytest.raises(awpsgt.AwpError, match="cannot open"):
        awpsgt.read_srf(str(tmp_path / "missing.srf"))
    c = ai.synth_case(seed=4, nv=1)
    path = str(tmp_path / "cut.srf")
    ai.write_srf(path, *c.variations[0])
    text = open(path).read()
    open(path, "w").write(text[: len(text) // 2])
    with pytest.raises(awpsgt.AwpError, match="cut short"):
        awpsgt.read_srf(path)
    open(path, "w").write("1.0\nNOTPOINTS 3\n")
    with pytest.raises(awpsgt.AwpError, match="POINTS"):
        awpsgt.read_srf(path)


def test_oracle_grid_lookup_inverts_the_projection():
    c = ai.synth_case(seed=5, jitter=0.0)
    assert oracle.synth_get_indx(c.master, c.h_km, c.slon, c.slat, 0.0)[1] == (8, 10, 1)
    lon, lat = ai.model_xy_to_lonlat(c.master, np.array([0.0, 17.0, 33.0]), np.array([0.0, 5.0, 41.0]))
    for (x, y), lo, la in zip([(0, 0), (17, 5), (33, 41)], lon, lat):
        indx, xyz = oracle.synth_get_indx(c.master, c.h_km, lo, la, 2.0)
        assert xyz == (x, y, 3) and indx == x * 10**12 + y * 10**6 + 3


def test_oracle_delta_slip_rate_gives_shifted_rotated_sgt():
    """One exact SGT point, one slip component, stf * dt = 1 at a single
    sample: the seismogram is the mechanism-weighted, rotated, tapered SGT
    shifted by the rupture time (sgt3d_subs.c:1121-1422), computed here in
    float64 numpy."""
    c = ai.synth_case(seed=6, nx_f=1, nz_f=1, nv=1, drop_frac=0.0, mech2_frac=0.0, mech3_frac=0.0,
                      zero_frac=0.0, jitter=0.0, ncomp=3)
    pts, _ = c.variations[0]
    pts = pts.copy()
    pts["nt1"], pts["stf1"], pts["tinit"] = 1, 0, 2.5
    pool = np.array([1.0 / c.dtout], np.float32)
    v = [(pts, pool)]
    seis, ntout = oracle.synth(c.master, c.index, c.headers, c.comps, c.slon, c.slat, c.dtout, 0, 0.0, v)
    a = pts[0]
    indx, xyz = oracle.synth_get_indx(c.master, c.h_km, a["lon"], a["lat"], a["dep"])
    ip = int(np.searchsorted(c.index["indx"], indx))
    assert c.index["indx"][ip] == indx
    h = c.headers[ip]
    r = np.radians
    dip, rak, stk, az = float(a["dip"]), float(a["rake"]), float(a["stk"]), float(h["xazim"])
    vx, vy, vz = -np.sin(r(dip)) * np.sin(r(stk - az)), np.sin(r(dip)) * np.cos(r(stk - az)), -np.cos(r(dip))
    us, ud = np.cos(r(rak)), np.sin(r(rak))
    ux = ud * np.cos(r(dip)) * np.sin(r(stk - az)) + us * np.cos(r(stk - az))
    uy = -ud * np.cos(r(dip)) * np.cos(r(stk - az)) + us * np.sin(r(stk - az))
    uz = -ud * np.sin(r(dip))
    lam, mu = float(h["lam"]), float(h["mu"])
    m = np.array([(lam + 2 * mu) * vx * ux + lam * vy * uy + lam * vz * uz,
                  lam * vx * ux + (lam + 2 * mu) * vy * uy + lam * vz * uz,
                  lam * vx * ux + lam * vy * uy + (lam + 2 * mu) * vz * uz,
                  mu * (vx * uy + vy * ux), mu * (vx * uz + vz * ux), mu * (vy * uz + vz * uy)])
    amp = float(a["area"]) / float(h["xmom"])
    s = [amp * np.einsum("k,kt->t", m, c.comps[q][ip].astype(np.float64)) for q in range(3)]
    nt = int(h["nt"])
    fac = np.ones(nt)
    fac[nt - 9:] = 0.5 * (1 + np.cos(np.pi / 10 * np.arange(1, 10)))
    ge = (s[0] * np.sin(r(az)) + s[1] * np.cos(r(az))) * fac
    gn = (s[0] * np.cos(r(az)) - s[1] * np.sin(r(az))) * fac
    gv = -s[2] * fac
    x = np.float32(np.float32(h["tst"]) + np.float32(2.5)) / np.float32(c.dtout)
    shift = int(x + 0.5) if x >= 0 else int(x - 0.5)       # truncation, sgt3d_subs.c:1215-1219
    want = np.zeros((3, ntout))
    lo, hi = max(shift, 0), min(nt + shift, ntout)
    for k, g in enumerate((gv, gn, ge)):
        want[k, lo:hi] = g[lo - shift:hi - shift]
    scale = np.abs(want).max()
    assert scale > 0
    np.testing.assert_allclose(seis[0], want, rtol=0, atol=2e-5 * scale)


def test_oracle_is_linear_in_a_power_of_two():
    c = ai.synth_case(seed=7, nv=2)
    s1, _ = case_seis(c)
    c.variations = [(p, q * np.float32(4.0)) for p, q in c.variations]
    s4, _ = case_seis(c)
    np.testing.assert_allclose(s4, s1 * np.float32(4.0), rtol=1e-6, atol=1e-36)     # subnormals round


def test_oracle_refuses_resampling():
    c = ai.synth_case(seed=8, nv=1)
    pts, pool = c.variations[0]
    pts = pts.copy()
    pts["dt"] = c.dtout * 0.5
    c.variations = [(pts, pool)]
    with pytest.raises(ValueError):
        case_seis(c)


# ---- device path ---------------------------------------------------------------

def run_device(c, ntout=0, tstart=0.0, rv_batch=0, ubuf_mb=None):
    if ubuf_mb is not None:
        os.environ["AWP_SYNTH_UBUF_MB"] = str(ubuf_mb)
    try:
        with awpsgt.Synth(c.slon, c.slat, c.dtout, ntout=ntout, tstart=tstart, rv_batch=rv_batch) as s:
            s.set_sgt(c.master, c.index, c.headers, c.comps)
            for i, (p, q) in enumerate(c.variations):
                s.add_variation(100 + i, p, q)
            out = s.run()
            return out, s.info()
    finally:
        os.environ.pop("AWP_SYNTH_UBUF_MB", None)


@pytest.mark.gpu
@pytest.mark.parametrize("ncomp", [1, 2, 3])
@pytest.mark.parametrize("ntout,tstart", [(0, 0.0), (700, 1.3), (150, -2.0)])
def test_device_matches_oracle_bitwise(ncomp, ntout, tstart):
    c = ai.synth_case(seed=10 + ncomp, ncomp=ncomp, nv=3, mech2_frac=0.2, mech3_frac=0.1)
    want, nout = case_seis(c, ntout, tstart)
    got, info = run_device(c, ntout, tstart)
    assert got.shape == want.shape and info.ntout == nout
    assert info.non_exact > 0 and info.terms > len(c.variations[0][0]) and info.gpu_launches >= 2
    assert np.abs(got).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("rv_batch,ubuf_mb", [(1, None), (2, 1), (0, 1), (3, 2)])
def test_device_batches_and_chunks_match_oracle(rv_batch, ubuf_mb):
    """Several variation batches and term-buffer chunks (1 MiB holds a few
    points' terms) accumulate in the same order as one pass."""
    c = ai.synth_case(seed=20, nx_f=20, nz_f=8, nt=400, nv=5, ntout=1200, nstf=(5, 120))
    want, _ = case_seis(c, 1200)
    got, info = run_device(c, 1200, rv_batch=rv_batch, ubuf_mb=ubuf_mb)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    if ubuf_mb:
        assert info.gpu_launches > 2 * ((5 + (rv_batch or 5) - 1) // (rv_batch or 5))


@pytest.mark.gpu
def test_device_edge_cases_match_oracle():
    """Points without slip, slip rates as long as the output, every rupture
    point off the SGT grid (four-point brackets)."""
    c = ai.synth_case(seed=21, nv=2, zero_frac=0.3, drop_frac=1.0, nstf=(1, 100), nt=120)
    want, nout = case_seis(c, 100)
    got, info = run_device(c, 100)
    assert info.non_exact == len(c.variations[0][0])
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_device_files_and_grm_output(tmp_path):
    c = ai.synth_case(seed=22, ncomp=2, nv=2)
    paths = {}
    for q, comp in enumerate("xy"):
        hd = c.headers.copy()
        if comp == "y":
            hd["ymom"], hd["xmom"] = hd["xmom"], 0.0
        head = str(tmp_path / ("s_%s.sgthead" % comp))
        with open(head, "wb") as f:
            f.write(c.master.tobytes() + c.index.tobytes() + hd.tobytes())
        data = str(tmp_path / ("s_%s.sgt" % comp))
        c.comps[q].tofile(data)
        paths[comp] = (head, data)
    srfs = []
    for i, (p, q) in enumerate(c.variations):
        srfs.append(str(tmp_path / ("v%d.srf" % i)))
        ai.write_srf(srfs[-1], p, q, binary=bool(i % 2))
    want, nout = case_seis(c)
    with awpsgt.Synth(c.slon, c.slat, c.dtout) as s:
        s.load_sgt_files(paths["x"][0], paths["x"][1], paths["y"][0], paths["y"][1])
        for i, f in enumerate(srfs):
            s.add_srf_file(7 + i, f, binary=bool(i % 2))
        got = s.run()
        grm = str(tmp_path / "Seismogram_TEST_1_2_3.grm")
        s.write_grm(grm, site="TEST", source_id=2, rupture_id=3, det_max_freq=1.0)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    hd, data = awpsgt.read_grm(grm, 2, nout)
    assert list(hd["rup_var_id"]) == [7, 8] and all(hd["comps"] == 3) and all(hd["nt"] == nout)
    assert all(hd["source_id"] == 2) and hd[0]["site_name"] == b"TEST"
    assert np.array_equal(data, got[:, 1:3])                # north, east (jbsim3d.c:626-629)


@pytest.mark.gpu
def test_device_errors(tmp_path):
    c = ai.synth_case(seed=23, nv=1)
    with awpsgt.Synth(c.slon, c.slat, c.dtout) as s:
        with pytest.raises(awpsgt.AwpError, match="no SGT"):
            s.run()
        s.set_sgt(c.master, c.index, c.headers, c.comps)
        with pytest.raises(awpsgt.AwpError, match="no rupture"):
            s.run()
        p, q = c.variations[0]
        bad = p.copy()
        bad["dt"] = c.dtout * 2
        s.add_variation(0, bad, q)
        with pytest.raises(awpsgt.AwpError, match="resampling"):
            s.run()
        s.clear_variations()
        with pytest.raises(awpsgt.AwpError, match="points"):
            s.add_variation(0, p, q)
            s.add_variation(1, p[:-1], q)
        bad = p.copy()
        bad["nt1"][0], bad["stf1"][0] = 3, len(q) + 5
        with pytest.raises(awpsgt.AwpError, match="pool"):
            s.add_variation(2, bad, q)
    head = str(tmp_path / "x.sgthead")
    hd = c.headers.copy()
    with open(head, "wb") as f:
        f.write(c.master.tobytes() + c.index.tobytes() + hd.tobytes())
    data = str(tmp_path / "x.sgt")
    c.comps[0].tofile(data)
    with awpsgt.Synth(c.slon, c.slat, c.dtout) as s:
        with pytest.raises(awpsgt.AwpError, match="Y-moment"):
            s.load_sgt_files(head, data, head, data)


@pytest.mark.gpu
def test_device_large_case_properties():
    """At a size the oracle would take minutes on: batch split and chunking
    change nothing, a variation's seismogram does not depend on its place in
    the batch, and doubling every slip rate doubles the seismograms (exactly
    but for products that round in the subnormal range)."""
    c = ai.synth_case(seed=30, nx_f=48, nz_f=16, nt=1000, nv=8, ntout=1500, nstf=(20, 80))
    a, _ = run_device(c, 1500)
    b, _ = run_device(c, 1500, rv_batch=3, ubuf_mb=8)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    c.variations = c.variations[::-1]
    r, _ = run_device(c, 1500, rv_batch=5)
    assert np.array_equal(r[::-1].view(np.uint32), a.view(np.uint32))
    c.variations = [(p, q * np.float32(2.0)) for p, q in c.variations[::-1]]
    d, _ = run_device(c, 1500)
    np.testing.assert_allclose(d, a * np.float32(2.0), rtol=1e-6, atol=1e-36)


@pytest.mark.gpu
def test_device_zero_slip_long_slip_rate_and_reuse():
    """A rupture without slip gives zero seismograms; a slip rate longer than
    ntout is refused; clearing the variations keeps the SGT set for the next
    rupture, whose results equal a fresh object's."""
    c = ai.synth_case(seed=24, nv=2)
    with awpsgt.Synth(c.slon, c.slat, c.dtout, ntout=500) as s:
        s.set_sgt(c.master, c.index, c.headers, c.comps)
        p, q = c.variations[0]
        quiet = p.copy()
        quiet["nt1"] = quiet["nt2"] = quiet["nt3"] = 0
        s.add_variation(0, quiet, q)
        z = s.run()
        assert z.shape == (1, 3, 500) and not np.any(z.view(np.uint32))
        assert s.info().terms == 0
        s.clear_variations()
        longer = p.copy()
        i = int(np.argmax(longer["nt1"]))
        longer["nt1"][i], longer["stf1"][i] = 501, len(q)
        s.add_variation(1, longer, np.concatenate([q, np.ones(501, np.float32)]))
        with pytest.raises(awpsgt.AwpError, match="longer than ntout"):
            s.run()
        s.clear_variations()
        for k, (pp, qq) in enumerate(c.variations):
            s.add_variation(k, pp, qq)
        again = s.run()
    want, _ = case_seis(c, 500)
    assert np.array_equal(again.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_device_empty_rupture():
    c = ai.synth_case(seed=25, nv=1)
    with awpsgt.Synth(c.slon, c.slat, c.dtout, ntout=300) as s:
        s.set_sgt(c.master, c.index, c.headers, c.comps)
        s.add_variation(0, np.zeros(0, awpsgt.SRFPOINT), np.zeros(0, np.float32))
        out = s.run()
    assert out.shape == (1, 3, 300) and not np.any(out)


@pytest.mark.gpu
def test_device_borrowed_variations_equal_copied():
    c = ai.synth_case(seed=26, nv=4)
    a, _ = run_device(c, 600)
    with awpsgt.Synth(c.slon, c.slat, c.dtout, ntout=600) as s:
        s.set_sgt(c.master, c.index, c.headers, c.comps)
        for i, (p, q) in enumerate(c.variations):
            s.add_variation(100 + i, p, q, borrow=True)
        b = s.run()
        again = s.run()                      # still listed: read in place again
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert np.array_equal(a.view(np.uint32), again.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("g", GOLD_CASES, ids=lambda g: g["name"])
def test_device_matches_reference_fixtures(g):
    """The device path against seismograms of DirectSynth's own functions."""
    c, want = golden_case(g)
    got, _ = run_device(c, g["ntout"], g["tstart"])
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
