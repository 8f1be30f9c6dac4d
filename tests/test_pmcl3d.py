"""The pmcl3d drop-in driver end to end: reference-format inputs on disk, both
reference command lines, reference-format outputs compared with the oracle."""
import os
import subprocess

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt
import fortran_format as ff
import oracle

NX, NY, NZ, NST = 48, 40, 32, 60


def write_inputs(d, igreen=1, ifault=0, write_step=3, ntiskp=5):
    media = ai.layered_media(NX, NY, NZ, 200.0, seed=4, pert_std=0.05, corr_len=1000.0)
    stf = ai.gaussian_derivative_stf(NST, 0.01, f0=1.0, column=max(igreen, 1) - 1 if igreen in (1, 2, 3) else 0)
    pts = ai.sgt_points(NX, NY, 20, 30, seed=0)
    os.makedirs(d / "input", exist_ok=True)
    ai.write_media(str(d / "input" / "media"), media)
    if ifault == 0:
        ai.write_source_text(str(d / "input" / "src"), (24, 20, 9), stf)
    else:
        ai.write_source_binary(str(d / "input" / "src"), (24, 20, 9), stf)
    ai.write_cordfile(str(d / "input" / "cord"), pts, comment="test points")
    return media, stf, pts


def oracle_sgt(media, stf, pts, igreen=1, write_step=3, ntiskp=5, nt=None):
    nt = NST + 1 if nt is None else nt
    o = oracle.Oracle(nx=NX, ny=NY, nz=NZ, dh=200.0, dt=0.01, nt=nt, nst=NST, nd=8, fl=0.01, fh=25.0, fp=0.5,
                      socalq=1, ntiskp_sgt=ntiskp, write_step=write_step, igreen=igreen)
    o.load_media(media)
    o.set_source([(24, 20, 9)], stf)
    o.set_points(pts)
    o.run(nt)
    return o


def in3d(d, igreen=1, ifault=0, write_step=3, ntiskp=5):
    w = ai.In3d(igreen=igreen, tmax=0.6, dh=200.0, dt=0.01, nd=8, nst=NST, nx=NX, ny=NY, nz=NZ, ifault=ifault,
                mediarestart=1, nvar=3, socalq=1, nve=1, fl=0.01, fh=25.0, fp=0.5, read_step=NST,
                write_step=write_step, write_step2=write_step, ntiskp_sgt=ntiskp,
                chkp="out/CHKP", chkj="out/CHKJ", insrc="input/src", invel="input/media", insgt="input/cord",
                sgtgro="out/sgt/awp-strain")
    w.write(str(d / "IN3D"))
    return w


@pytest.mark.gpu
@pytest.mark.parametrize("ifault", [0, 1])
def test_fortran_command_line(tmp_path, ifault):
    media, stf, pts = write_inputs(tmp_path, ifault=ifault)
    w = in3d(tmp_path, ifault=ifault)
    assert w.nt == NST + 1
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    got = np.fromfile(tmp_path / "out" / "sgt" / "awp-strain", dtype=np.float32)
    o = oracle_sgt(media, stf, pts)
    ref = o.sgt()
    assert got.size == ref.size == 30 * 6 * 12       # NT = int(int(61/3)*3/5) = 12
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    # CHKJ: (I6,3E10.3) per step, u1 v1 w1 at (ND+2, ND+2, ND+2)
    lines = (tmp_path / "out" / "CHKJ").read_text().splitlines()
    assert len(lines) == NST + 1
    assert all(len(l) == 36 for l in lines)
    cj = o.chkj()
    last = lines[-1]
    assert int(last[:6]) == NST + 1
    np.testing.assert_allclose([float(last[6 + 10 * q:16 + 10 * q]) for q in range(3)], cj[-1], rtol=6e-3, atol=1e-30)
    chkp = (tmp_path / "out" / "CHKP").read_text()
    assert "STABILITY CRITERIA .5 > CMAX*DT/DX" in chkp and "# OF TIME STEPS   61" in chkp   # I5


@pytest.mark.gpu
def test_positional_overrides(tmp_path):
    media, stf, pts = write_inputs(tmp_path)
    in3d(tmp_path)
    os.rename(tmp_path / "input" / "media", tmp_path / "other_media")
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D", "input/src", "other_media", "out/C1", "out/C2"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "out" / "C1").exists() and (tmp_path / "out" / "C2").exists()


@pytest.mark.gpu
def test_gpu_command_line_chunk_files(tmp_path):
    """The argument list gpu_wrapper.py builds; one SGT%07d file per
    WRITE_STEP chunk, each [point][6][WRITE_STEP] (FAST-T layout)."""
    media, stf, pts = write_inputs(tmp_path, ifault=1)
    argv = [awpsgt.PMCL3D_PATH, "-T", "0.6", "--IGREEN", "1", "--DH", "200.0", "--DT", "0.01", "--NSRC", "1",
            "--NST", str(NST), "-X", str(NX), "-Y", str(NY), "-Z", str(NZ), "-x", "1", "-y", "1", "--NPC", "0",
            "--ARBC", "0.92", "--ND", "8", "--IFAULT", "1", "--MEDIASTART", "1", "--FL", "0.01", "--FH", "25.0",
            "--FP", "0.5", "--READ_STEP", str(NST), "--WRITE_STEP", "4", "-o", "out_sgt", "--INSGT", "input/cord",
            "-c", "out_sgt/CHKP", "--INSRC", "input/src", "--INVEL", "input/media", "--NTISKP_SGT", "5",
            "--NTISKP", "10"]
    r = subprocess.run(argv, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    # nt = (int)(0.6/0.01) + 1 = 60 or 61 depending on rounding of 0.6f/0.01f
    nt = int(np.float32(0.6) / np.float32(0.01)) + 1
    o = oracle_sgt(media, stf, pts, write_step=4, ntiskp=5, nt=nt)
    ref = o.sgt().reshape(30, 6, -1)
    nchunk = (nt // 5) // 4
    assert nchunk >= 2
    for c in range(nchunk):
        f = tmp_path / "out_sgt" / ("SGT%07d" % ((c + 1) * 4 * 5))
        got = np.fromfile(f, dtype=np.float32).reshape(30, 6, 4)
        assert np.array_equal(got, ref[:, :, c * 4:(c + 1) * 4])
    assert (tmp_path / "out_sgt" / "CHKP").exists()


def test_driver_reports_missing_input(tmp_path):
    """Errors come back as a message and a nonzero exit, never a crash."""
    in3d(tmp_path)
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    assert "source" in r.stderr


def test_driver_rejects_unknown_boundary(tmp_path):
    """NPC is 0 (Cerjan) or 1 (PML); anything else is refused before the
    solver touches a device."""
    write_inputs(tmp_path)
    w = in3d(tmp_path)
    w.npc = 2
    w.write(str(tmp_path / "IN3D"))
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "NPC" in r.stderr, r.stderr


@pytest.mark.gpu
def test_rwg_order_output(tmp_path):
    """AWP_RWG_SGT=x: the SGT file comes out in RWG component order, as
    SgtHead's reformat_awp would write it."""
    media, stf, pts = write_inputs(tmp_path)
    in3d(tmp_path)
    env = dict(os.environ, AWP_RWG_SGT="x")
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300,
                       env=env)
    assert r.returncode == 0, r.stderr + r.stdout
    got = np.fromfile(tmp_path / "out" / "sgt" / "awp-strain", dtype=np.float32)
    ref = oracle.reorder_rwg(oracle_sgt(media, stf, pts).sgt(), 12)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.gpu
def test_gpu_command_line_kinematic_source(tmp_path):
    """IFAULT=5 with the GPU command line: a binary subfault table (two rows of
    six per subfault, NST = READ_STEP = 2) drives the run; the SGT chunk files
    match the oracle within the tolerance of the kinematic tests."""
    from test_gpu_parity import kinematic_rupture, rel_l2
    media, _, pts = write_inputs(tmp_path)
    xyz = [(18 + k, 20, 10 + k % 3) for k in range(8)]
    tab = kinematic_rupture(len(xyz), seed=9)
    with open(tmp_path / "input" / "kin", "wb") as f:
        for k, (x, y, z) in enumerate(xyz):
            np.asarray((x, y, z), np.int32).tofile(f)
            tab[k].astype(np.float32).tofile(f)
    argv = [awpsgt.PMCL3D_PATH, "-T", "0.6", "--IGREEN", "1", "--DH", "200.0", "--DT", "0.01", "--NSRC", str(len(xyz)),
            "--NST", "2", "-X", str(NX), "-Y", str(NY), "-Z", str(NZ), "-x", "1", "-y", "1", "--NPC", "0",
            "--ARBC", "0.92", "--ND", "8", "--IFAULT", "5", "--MEDIASTART", "1", "--FL", "0.01", "--FH", "25.0",
            "--FP", "0.5", "--READ_STEP", "2", "--WRITE_STEP", "4", "-o", "out_kin", "--INSGT", "input/cord",
            "-c", "out_kin/CHKP", "--INSRC", "input/kin", "--INVEL", "input/media", "--NTISKP_SGT", "5",
            "--NTISKP", "10"]
    r = subprocess.run(argv, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    nt = int(np.float32(0.6) / np.float32(0.01)) + 1
    o = oracle.Oracle(nx=NX, ny=NY, nz=NZ, dh=200.0, dt=0.01, nt=nt, nst=2, nd=8, fl=0.01, fh=25.0, fp=0.5,
                      socalq=1, ntiskp_sgt=5, write_step=4, igreen=1, kinematic=1)
    o.load_media(media)
    o.set_source(xyz, tab)
    o.set_points(pts)
    o.run(nt)
    ref = o.sgt().reshape(30, 6, -1)
    got = np.concatenate([np.fromfile(tmp_path / "out_kin" / ("SGT%07d" % ((c + 1) * 20)), np.float32).reshape(30, 6, 4)
                          for c in range((nt // 5) // 4)], axis=2)
    assert np.abs(got).max() > 0
    assert rel_l2(got, ref[:, :, :got.shape[2]]) <= 1e-5
    bad = argv[:]
    bad[bad.index("--NST") + 1] = "3"
    r = subprocess.run(bad, cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "NST" in r.stderr


@pytest.mark.gpu
def test_autotuned_drop_in_run(tmp_path):
    """AWP_AUTOTUNE_CACHE: the driver tunes the launch shapes for the grid
    first, keeps them in the file, reuses them on the next run, and the SGT
    file stays bit-identical to the oracle's."""
    media, stf, pts = write_inputs(tmp_path)
    in3d(tmp_path)
    cache = tmp_path / "tune.txt"
    env = dict(os.environ, AWP_AUTOTUNE_CACHE=str(cache))
    ref = oracle_sgt(media, stf, pts).sgt()
    for run in range(2):
        r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300,
                           env=env)
        assert r.returncode == 0, r.stderr + r.stdout
        assert "Launch shapes tuned" in r.stdout
        got = np.fromfile(tmp_path / "out" / "sgt" / "awp-strain", dtype=np.float32)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
        assert len(cache.read_text().splitlines()) == 1      # the second run reads it back


def test_fortran_format_helper():
    """The edit-descriptor helper the CHKP / CHKJ comparisons use, on values
    whose Fortran output follows from the standard's rules by hand."""
    assert ff.e(0.5, 15, 7) == "  0.5000000E+00"
    assert ff.e(-1.234e-5, 10, 3) == "-0.123E-04"
    assert ff.e(0.0, 10, 3) == " 0.000E+00"
    assert ff.e(9.9996, 10, 3) == " 0.100E+02"        # rounding carries into the exponent
    assert ff.g(0.92, 13, 4) == "   0.9200    "
    assert ff.g(0.01, 14, 5) == "   0.10000E-01"
    assert ff.g(25.0, 14, 5) == "    25.000    "
    assert ff.g(0.5, 14, 5) == "   0.50000    "
    assert ff.g(99999.9, 13, 4) == "   0.1000E+06"
    assert ff.f(200.0, 10, 4) == "  200.0000"
    assert ff.i(61, 5) == "   61"
    assert ff.i(100000, 5) == "*****"                 # CyberShake's NTISKP in an I5 field
    assert ff.list_directed("igreen = ", 1) == " igreen =            1"


def expected_chkp_fortran(w, ext):
    """io.f:486-531 (wrpm3d) for one rank, every REAL in single precision;
    ext = the oracle's extremes (vp min/max, vs min/max, rho min/max) of the
    SoCalQ-corrected media (structure.f:469-530)."""
    f32 = np.float32
    vpmin, vpmax, vsmin, vsmax, dmin, dmax = (f32(v) for v in ext)
    cfl = f32(vpmax * f32(w.dt)) / f32(w.dh)
    lines = [ff.list_directed("igreen = ", w.igreen),
             "STABILITY CRITERIA .5 > CMAX*DT/DX = " + ff.e(cfl, 15, 7),
             "# OF X NODES PER PROC" + ff.i(w.nx // w.npx, 5),
             "# OF Y NODES PER PROC" + ff.i(w.ny // w.npy, 5),
             "# OF Z NODES PER PROC" + ff.i(w.nz // w.npz, 5),
             "# OF TIME STEPS" + ff.i(w.nt, 5),
             "DISCRETIZATION IN SPACE" + ff.f(f32(w.dh), 10, 4),
             "DISCRETIZATION IN TIME" + ff.f(f32(w.dt), 10, 4),
             "PML REFLECTION COEFFICIENT" + ff.g(f32(w.arbc), 13, 4),
             "HIGHEST P-VELOCITY ENCOUNTERED" + ff.f(vpmax, 10, 2),
             "LOWEST P-VELOCITY ENCOUNTERED" + ff.f(vpmin, 10, 2),
             "HIGHEST S-VELOCITY ENCOUNTERED" + ff.f(vsmax, 10, 2),
             "LOWEST S-VELOCITY ENCOUNTERED" + ff.f(vsmin, 10, 2),
             "HIGHEST DENSITY ENCOUNTERED" + ff.f(dmax, 15, 2),
             "LOWEST  DENSITY ENCOUNTERED" + ff.f(dmin, 15, 2),
             "SKIP OF SEISMOGRAMS IN TIME (LOOP COUNTER)" + ff.i(w.ntiskp, 5),
             "ABC CONDITION, PML=1 OR CERJAN=0:" + ff.i(w.npc, 5),
             "FD SCHEME, VISCO=1 OR ELASTIC=0:" + ff.i(w.nve, 5),
             "Q, FL,FP,FH:" + ff.g(f32(w.fl), 14, 5) + ff.g(f32(w.fp), 14, 5) + ff.g(f32(w.fh), 14, 5)]
    return "\n".join(lines) + "\n"


@pytest.mark.gpu
def test_chkp_and_chkj_text_match_the_fortran_writes(tmp_path):
    """CHKP line for line as wrpm3d writes it (io.f:481-536: the stability
    number vpe(2)*dt/dh, the media extremes, the parameters, each in its
    edit descriptor) and CHKJ as (I6,3E10.3) of the oracle's probe values
    (pmcl3d.f:1478-1479), character for character.  The first CHKP line is
    list-directed output, whose spacing the standard leaves to the compiler:
    gfortran's."""
    media, stf, pts = write_inputs(tmp_path)
    w = in3d(tmp_path)
    r = subprocess.run([awpsgt.PMCL3D_PATH, "IN3D"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    o = oracle_sgt(media, stf, pts)
    got = (tmp_path / "out" / "CHKP").read_text()
    want = expected_chkp_fortran(w, o.extremes())
    assert got == want, "\n".join(a + " | " + b for a, b in zip(got.splitlines(), want.splitlines()) if a != b)
    cj = o.chkj()
    want_j = "".join(ff.i(n + 1, 6) + "".join(ff.e(v, 10, 3) for v in cj[n]) + "\n" for n in range(len(cj)))
    assert (tmp_path / "out" / "CHKJ").read_text() == want_j
    assert np.abs(cj).max() > 0


@pytest.mark.gpu
def test_gpu_command_line_surface_records_and_chkfile(tmp_path):
    """The GPU command line with NTISKP < NT (AWP-GPU-SGT/src/pmcl3d.c:962-1031,
    1172-1174): every NTISKP steps u1 v1 w1 on the NBG*:NSKP*:NED* window
    (z in depth from the surface) fill a WRITE_STEP-sample buffer, written to
    OUT/SX%07d, SY, SZ when full; the CHKFILE, after the parameter lines of
    io.c:16-31, gets "step :\tu\tv\tw" at x = y = ND+1, depth ND, and "END"."""
    media, stf, pts = write_inputs(tmp_path, ifault=1)
    ntiskp, ws = 4, 3
    argv = [awpsgt.PMCL3D_PATH, "-T", "0.6", "--IGREEN", "1", "--DH", "200.0", "--DT", "0.01", "--NSRC", "1",
            "--NST", str(NST), "-X", str(NX), "-Y", str(NY), "-Z", str(NZ), "-x", "1", "-y", "1", "--NPC", "0",
            "--ARBC", "0.92", "--ND", "8", "--IFAULT", "1", "--MEDIASTART", "1", "--FL", "0.01", "--FH", "25.0",
            "--FP", "0.5", "--READ_STEP", str(NST), "--WRITE_STEP", str(ws), "-o", "out", "--INSGT", "input/cord",
            "-c", "out/CHKP", "--INSRC", "input/src", "--INVEL", "input/media", "--NTISKP_SGT", "5",
            "--NTISKP", str(ntiskp), "--NBGX", "2", "--NEDX", "40", "--NSKPX", "3", "--NBGY", "1", "--NEDY", "-1",
            "--NSKPY", "2", "--NBGZ", "1", "--NEDZ", "3", "--NSKPZ", "2"]
    r = subprocess.run(argv, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    nt = int(np.float32(0.6) / np.float32(0.01)) + 1
    # the window by hand from pmcl3d.c:300-320 and calcRecordingPoints for one
    # rank: NEDX 40 -> 38 (a record point), x = 2, 5, .., 38; NEDY -1 -> 40 ->
    # 39, and since NY <= 39 fails, y = 1, 3, .., 39; depth 0 and 2 (z = NZ, NZ-2)
    xs, ys, ks = np.arange(1, 38, 3), np.arange(0, 39, 2), [NZ, NZ - 2]
    o = oracle.Oracle(nx=NX, ny=NY, nz=NZ, dh=200.0, dt=0.01, nt=nt, nst=NST, nd=8, fl=0.01, fh=25.0, fp=0.5,
                      socalq=1, ntiskp_sgt=5, write_step=ws, igreen=1)
    o.load_media(media)
    o.set_source([(24, 20, 9)], stf)
    o.set_points(pts)
    bufs = {c: np.zeros((ws, len(ks), len(ys), len(xs)), np.float32) for c in ("u1", "v1", "w1")}
    lines, done, nfiles = [], 0, 0
    for t in range(ntiskp, nt + 1, ntiskp):
        o.run(t - done)
        done = t
        sample = (t // ntiskp + ws - 1) % ws
        probe = []
        for c in ("u1", "v1", "w1"):
            fld = o.field(c)
            for dz, k in enumerate(ks):
                bufs[c][sample, dz] = fld[k + 1, 2:NY + 2, 2:NX + 2][np.ix_(ys, xs)]
            probe.append(fld[NZ - 8 + 1, 8 + 2, 8 + 2])
        lines.append("%d :\t%e\t%e\t%e" % (t, *probe))
        if (t // ntiskp) % ws == 0:
            nfiles += 1
            for c, name in (("u1", "SX"), ("v1", "SY"), ("w1", "SZ")):
                got = np.fromfile(tmp_path / "out" / ("%s%07d" % (name, t)), dtype=np.float32)
                assert got.size == bufs[c].size
                assert np.array_equal(got.view(np.uint32), bufs[c].ravel().view(np.uint32)), (name, t)
    assert nfiles >= 4 and np.abs(bufs["u1"]).max() > 0
    chk = (tmp_path / "out" / "CHKP").read_text().splitlines()
    f32 = np.float32
    ext = o.extremes()
    head = ["STABILITY CRITERIA .5 > CMAX*DT/DX:\t%f" % (f32(f32(ext[1]) * f32(0.01)) / f32(200.0)),
            "# OF X,Y,Z NODES PER PROC:\t%d, %d, %d" % (NX, NY, NZ), "# OF TIME STEPS:\t%d" % nt,
            "DISCRETIZATION IN SPACE:\t%f" % f32(200.0), "DISCRETIZATION IN TIME:\t%f" % f32(0.01),
            "PML REFLECTION COEFFICIENT:\t%f" % f32(0.92),
            "HIGHEST P-VELOCITY ENCOUNTERED:\t%f" % ext[1], "LOWEST P-VELOCITY ENCOUNTERED:\t%f" % ext[0],
            "HIGHEST S-VELOCITY ENCOUNTERED:\t%f" % ext[3], "LOWEST S-VELOCITY ENCOUNTERED:\t%f" % ext[2],
            "HIGHEST DENSITY ENCOUNTERED:\t%f" % ext[5], "LOWEST  DENSITY ENCOUNTERED:\t%f" % ext[4],
            "SKIP OF SEISMOGRAMS IN TIME (LOOP COUNTER):\t%d" % ntiskp, "ABC CONDITION, PML=1 OR CERJAN=0:\t0",
            "FD SCHEME, VISCO=1 OR ELASTIC=0:\t1", "Q, FL,FP,FH:\t%f, %f, %f" % (f32(0.01), f32(0.5), f32(25.0))]
    assert chk == head + lines + ["END"]
