"""Input formats and command lines of the drop-in driver (no GPU): the C
readers of libawpsgt against files written in the reference formats."""
import os

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt

REF_IN3D_TEXT = """        2 igreen        = SGT Parameters
    200.0 TMAX          = propagation time

    200.0 DH            = spatial step for x, y, z (meters)
    0.005 DT            = time step (seconds)

        0 NPC           = PML or Cerjan ABC (1=PML, 0=Cerjan)

       20 ND\t        = ABC thickness (grid-points) PML <= 20, Cerjan >= 20
     0.92 ARBC          = coefficient for PML (3-4), or Cerjan (0.90-0.96)
      0.1 PHT           =

        1 NSRC          = number of source nodes on fault
    40000 NST           = number of time steps in rupture functions

      800 NX            = x model dimension in nodes
      600 NY            = y model dimension in nodes
      400 NZ            = z model dimension in nodes

        8 NPX           = number of procs in the x direction
       10 NPY           = number of procs in the Y direction
        8 NPZ           = number of procs in the Z direction

        0 IFAULT
        0 CHECKPOINT
        1 ISFCVLM
        0 IMD5
        1 IVELOCITY
        1 MEDIARESTART
        3 NVAR
        1 IOST
        1 PARTDEG
        1 IO_OPT
        1 PERF_MEAS
        0 IDYNA
        1 SOCALQ

        1 NVE

    0.677 MU_S
    0.525 MU_D

     0.01 FL
     25.0 FH
      0.5 FP

    20000 READ_STEP
    2000 WRITE_STEP
    2000 WRITE_STEP2

       10 NBGX
      400 NEDX
       10 NSKPX
       10 NBGY
      300 NEDY
       10 NSKPY
       10 NBGZ
      200 NEDZ
       10 NSKPZ

   100000 NTISKP
       10 NTISKP_SGT

       10 NBGX2
      400 NEDX2
       10 NSKPX2
       10 NBGY2
      300 NEDY2
       10 NSKPY2
        1 NBGZ2
      200 NEDZ2
       10 NSKPZ2

       10 NTISKP2

'output_ckp/CHKP96PV' CHKP   = input and derived parameters for QC
'output_ckp/CHKJ96PV' CHKJ   = single location output for QC

'input/fy_src_100m'    INSRC  = mt based fault file
'/scratch/awp.100m.media' INVEL  = velocity structure file

'/scratch/awp.100m.cordfile' INSGT = sgt station lists

'output_sfc/XX96PS' SXRGO
'output_sfc/YY96PS' SYRGO
'output_sfc/ZZ96PS' SZRGO

'output_vlm/XY96PV' SXRGO2
'output_vlm/YZ96PV' SYRGO2
'output_vlm/XZ96PV' SZRGO2

'output_sfc/awp-strain' SGTGRO

'output_dyn/SGSN' SGSN       =  file to host 19 more variables for SGSN mode
"""


def test_splitmix64_published_sequence():
    # first outputs of splitmix64 seeded with 1234567 (Vigna's reference code)
    r = ai.SplitMix64(1234567)
    got = [r.next_u64() for _ in range(5)]
    assert got == [6457827717110365317, 3203168211198807973, 9817491932198370423,
                   4593380528125082431, 16408922859458223821]


def test_sgt_points_distinct_sorted_in_range():
    p = ai.sgt_points(160, 160, 51, 1000, seed=0)
    assert p.shape == (1000, 3)
    assert len({tuple(r) for r in p}) == 1000
    assert p[:, 0].min() >= 1 and p[:, 0].max() <= 160 and p[:, 2].min() >= 1 and p[:, 2].max() <= 51
    keys = [(y, x, z) for x, y, z in p]
    assert keys == sorted(keys)
    assert np.array_equal(p, ai.sgt_points(160, 160, 51, 1000, seed=0))


def test_reference_layout_in3d_parses(tmp_path):
    """The annotated reference IN3D (notes after each value, blank lines,
    tab characters, quoted paths) in the order of io.f:327-417."""
    f = tmp_path / "IN3D"
    f.write_text(REF_IN3D_TEXT)
    o = awpsgt.read_in3d(str(f))
    assert o.igreen == 2 and o.tmax == 200.0 and o.dh == 200.0 and abs(o.dt - 0.005) < 1e-9
    assert (o.nx, o.ny, o.nz) == (800, 600, 400)
    assert (o.npx, o.npy, o.npz) == (8, 10, 8)
    assert o.nve == 1 and o.socalq == 1 and o.nvar == 3
    assert abs(o.fl - 0.01) < 1e-9 and o.fh == 25.0 and o.fp == 0.5
    assert o.read_step == 20000 and o.write_step == 2000 and o.ntiskp_sgt == 10
    assert o.chkp == b"output_ckp/CHKP96PV" and o.invel == b"/scratch/awp.100m.media"
    assert o.sgtgro == b"output_sfc/awp-strain" and o.sgsn == b"output_dyn/SGSN"
    assert o.nt == 40001          # nint(200/0.005) + 1 (pmcl3d.f:287)
    p = awpsgt.params_from_in3d(o)
    assert p.nt == 40001 and p.igreen[0] == 2 and p.write_step == 2000


def test_in3d_writer_roundtrip(tmp_path):
    w = ai.In3d(igreen=1, tmax=10.0, nx=160, ny=160, nz=80, nst=1000, write_step=100, ntiskp_sgt=10,
                chkp="o/CHKP", chkj="o/CHKJ", insrc="in/src", invel="in/media", insgt="in/cord",
                sgtgro="out/sgt")
    w.write(str(tmp_path / "IN3D"))
    o = awpsgt.read_in3d(str(tmp_path / "IN3D"))
    assert o.nt == w.nt == 1001
    assert o.insgt == b"in/cord" and o.sgtgro == b"out/sgt"


def test_truncated_in3d_is_an_io_error(tmp_path):
    f = tmp_path / "IN3D"
    f.write_text("\n".join(REF_IN3D_TEXT.splitlines()[:20]))
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.read_in3d(str(f))
    assert e.value.status == 1


def test_positional_command_line_overrides(tmp_path):
    f = tmp_path / "IN3D"
    f.write_text(REF_IN3D_TEXT)
    o = awpsgt.parse_command_line(["pmcl3d", str(f), "my_src", "my_media", "my_chkp", "my_chkj"])
    assert o.insrc == b"my_src" and o.invel == b"my_media" and o.chkp == b"my_chkp" and o.chkj == b"my_chkj"
    assert o.gpu_cli == 0


def test_gpu_command_line_as_built_by_the_wrapper():
    # the argument list of AWP-GPU-SGT/gpu_wrapper.py
    argv = ["pmcl3d", "-T", "200.0", "--IGREEN", "1", "--DH", "100.0", "--DT", "0.005", "--NSRC", "1",
            "--NST", "40000", "-X", "400", "-Y", "300", "-Z", "200", "-x", "4", "-y", "3", "--NPC", "0",
            "--ARBC", "0.92", "--ND", "80", "--IFAULT", "1", "--MEDIASTART", "2", "--FL", "0.01", "--FH", "25.0",
            "--FP", "1.0", "--READ_STEP", "40000", "--WRITE_STEP", "4000", "-o", "comp_x/output_sgt",
            "--INSGT", "in/cord", "-c", "comp_x/CHKP", "--INSRC", "in/src", "--INVEL", "in/media",
            "--NTISKP_SGT", "10", "--NTISKP", "1000"]
    o = awpsgt.parse_command_line(argv)
    assert o.gpu_cli == 1
    assert (o.nx, o.ny, o.nz, o.npx, o.npy) == (400, 300, 200, 4, 3)
    assert o.igreen == 1 and o.nd == 80 and o.ifault == 1 and o.mediarestart == 2
    assert o.out_dir == b"comp_x/output_sgt" and o.chkp == b"comp_x/CHKP" and o.insgt == b"in/cord"
    assert o.write_step == 4000 and o.ntiskp_sgt == 10 and o.ntiskp == 1000
    assert o.nt == 40001          # (int)(TMAX/DT) + 1 (AWP-GPU-SGT/src/pmcl3d.c:265)
    assert o.nvar == 3 and o.socalq == 1 and o.nve == 1   # command.c defaults


def test_unknown_gpu_option_rejected():
    with pytest.raises(awpsgt.AwpError):
        awpsgt.parse_command_line(["pmcl3d", "--NOPE", "1"])


def test_source_text_roundtrip(tmp_path):
    stf = ai.gaussian_derivative_stf(50, 0.01, f0=1.0, column=1)
    stf[:, 4] = np.linspace(-1, 1, 50)
    ai.write_source_text(str(tmp_path / "src"), (80, 81, 11), stf)
    xyz, got = awpsgt.read_source(str(tmp_path / "src"), 0, 1, 50)
    assert tuple(xyz[0]) == (80, 81, 11)
    np.testing.assert_array_equal(got[0], stf)


def test_source_reference_table_format(tmp_path):
    """Rows "v, 0.0, 0.0, 0.0, 0.0, 0.0" as in AWP-*-SGT/utils/data/f?_src."""
    text = "3 4 1\n0.000000e+00, 0.0, 0.0, 0.0, 0.0, 0.0\n1.653250e+09, 0.0, 0.0, 0.0, 0.0, 0.0\n" \
           "2.267340e+09, 0.0, 0.0, 0.0, 0.0, 0.0\n"
    (tmp_path / "src").write_text(text)
    xyz, got = awpsgt.read_source(str(tmp_path / "src"), 0, 1, 3)
    assert tuple(xyz[0]) == (3, 4, 1)
    assert got[0, 1, 0] == np.float32(1.653250e+09) and got[0, 2, 0] == np.float32(2.267340e+09)


def test_source_binary_roundtrip_and_short_file(tmp_path):
    stf = np.random.default_rng(1).standard_normal((40, 6)).astype(np.float32)
    ai.write_source_binary(str(tmp_path / "src.bin"), (5, 6, 7), stf)
    xyz, got = awpsgt.read_source(str(tmp_path / "src.bin"), 1, 1, 40)
    assert tuple(xyz[0]) == (5, 6, 7)
    np.testing.assert_array_equal(got[0], stf)
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.read_source(str(tmp_path / "src.bin"), 1, 1, 41)
    assert e.value.status == 1


def test_cordfile_with_comments(tmp_path):
    pts = ai.sgt_points(50, 40, 10, 25, seed=2)
    ai.write_cordfile(str(tmp_path / "c"), pts, comment="generated")
    got = awpsgt.read_cordfile(str(tmp_path / "c"))
    np.testing.assert_array_equal(got, pts)


def test_short_cordfile_is_an_io_error(tmp_path):
    (tmp_path / "c").write_text("3\n1 2 3\n4 5 6\n")
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.read_cordfile(str(tmp_path / "c"))
    assert e.value.status == 1


def test_layered_media_recipe():
    m = ai.layered_media(64, 48, 40, 100.0, seed=0)
    vp, vs, rho = m[..., 0], m[..., 1], m[..., 2]
    np.testing.assert_allclose(vp / vs, 1.73, rtol=1e-6)
    np.testing.assert_allclose(rho, 310.0 * vp.astype(np.float64) ** 0.25, rtol=1e-6)
    # velocities increase with depth on average; 5 % perturbation
    assert vs[:5].mean() < vs[-5:].mean()
    base = vs / (1 + 0.0)
    layer_top = vs[0]
    assert abs(layer_top.std() / layer_top.mean() - 0.05) < 0.02
