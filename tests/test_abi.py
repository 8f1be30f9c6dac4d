"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares, reports errors as status codes, and its host-side helpers
(parameter defaults, algorithmic byte counts, footprints) are consistent."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import awpsgt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("awp_sgt.h", "awp_synth.h")]


def header_functions():
    src = "".join(open(h).read() for h in HEADERS)
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(awp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = awpsgt.load_library()
    decl = header_functions()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(awpsgt.EXPORTED + awpsgt.EXPORTED_SYNTH) == decl
    assert sorted(os.listdir(os.path.join(ROOT, "include"))) == sorted(os.path.basename(h) for h in HEADERS)


def test_exports_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", awpsgt.LIB_PATH], capture_output=True, text=True).stdout
    names = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    for n in header_functions():
        assert n in names, n


def test_param_defaults_match_gpu_command_defaults():
    lib = awpsgt.load_library()
    p = awpsgt.Params()
    lib.awp_params_default(C.byref(p))
    # AWP-GPU-SGT/src/command.c:60-115
    assert (p.nx, p.ny, p.nz) == (224, 224, 1024)
    assert p.dh == 200.0 and abs(p.dt - 0.01) < 1e-9
    assert p.nd == 20 and abs(p.arbc - 0.92) < 1e-7
    assert p.nst == 91 and p.write_step == 10 and p.ntiskp_sgt == 1
    assert p.socalq == 1 and p.nve == 1


@pytest.mark.parametrize("kernel,ncomp,prec,expect", [
    # two sweeps: velocity R 9 W 3, stress R 9 W 6, r1..r6 R+W, media shared
    ("two_sweep", 1, "f32", 176.0), ("two_sweep", 2, "f32", 166.0), ("two_sweep", 3, "f32", 156.0 + 20.0 / 3),
    ("two_sweep", 2, "bf16", 137.0), ("staged", 1, "f32", 176.0), ("staged", 3, "mixed", 132.0 + 20.0 / 3),
    # fused: u v w and 6 stresses read + written once, r1..r6 R+W, media once
    ("fused", 1, "f32", 140.0), ("fused", 2, "f16", 101.0), ("fused", 3, "f16", 96.0 + 10.0 / 3),
])
def test_algorithmic_bytes(kernel, ncomp, prec, expect):
    p = awpsgt.make_params(64, 64, 64, 100.0, 0.005, 10, igreen=(1, 2, 3)[:ncomp], precision=prec, ntiskp_sgt=1,
                           kernel=kernel)
    assert abs(awpsgt.bytes_per_cell_update(p) - expect) < 1e-9


def test_footprint_grows_with_components():
    p1 = awpsgt.make_params(400, 400, 200, 100.0, 0.005, 4001, igreen=(1,), ntiskp_sgt=10)
    p3 = awpsgt.make_params(400, 400, 200, 100.0, 0.005, 4001, igreen=(1, 2, 3), ntiskp_sgt=10)
    f1, f3 = awpsgt.footprint_bytes(p1, 5000), awpsgt.footprint_bytes(p3, 5000)
    cells = 400 * 400 * 200
    assert f1 > cells * 4 * 20
    assert f3 > f1 + 2 * cells * 4 * 15


def test_status_strings():
    lib = awpsgt.load_library()
    assert lib.awp_status_string(0) == b"AWP_OK"
    assert lib.awp_status_string(5) == b"AWP_ERR_UNSTABLE"


def test_bad_parameters_rejected_before_any_device_call():
    p = awpsgt.make_params(4, 64, 64, 100.0, 0.005, 10, ntiskp_sgt=1)
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.Solver(p)
    assert e.value.status == 2
    p = awpsgt.make_params(64, 64, 64, 100.0, 0.005, 10, ntiskp_sgt=1, igreen=(7,))
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.Solver(p)
    assert e.value.status == 2
    p = awpsgt.make_params(48, 40, 32, 200.0, 0.01, 10, nst=3, igreen=(1,), kinematic=1, ntiskp_sgt=1)
    with pytest.raises(awpsgt.AwpError) as e:   # IFAULT=5 subfaults are two rows each
        awpsgt.Solver(p)
    assert e.value.status == 2 and "NST = 2" in str(e.value)
    for prec in ("bf16", "f16"):           # the staged stepper reads FP32 media only
        p = awpsgt.make_params(64, 64, 64, 100.0, 0.005, 10, ntiskp_sgt=1, precision=prec, kernel="staged")
        with pytest.raises(awpsgt.AwpError) as e:
            awpsgt.Solver(p)
        assert e.value.status == 2 and "FP32 media" in str(e.value)


def test_create_without_gpu_fails_loudly():
    """On a machine without a GPU the CUDA path reports AWP_ERR_CUDA; there is
    no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = awpsgt.make_params(32, 32, 32, 100.0, 0.005, 10, ntiskp_sgt=1)
    with pytest.raises(awpsgt.AwpError) as e:
        awpsgt.Solver(p)
    assert e.value.status in (3, 4)


# ctypes mirror -> C type, for the layout check below
MIRRORS = [("Layout", "awp_layout"), ("Params", "awp_params"), ("Stats", "awp_stats"), ("Tuning", "awp_tuning"),
           ("KernelTimes", "awp_kernel_times"), ("In3dC", "awp_in3d"), ("SgtHeadArgs", "awp_sgthead_args"),
           ("Request", "awp_request"), ("RequestInfo", "awp_request_info"), ("SynthParams", "awp_synth_params"),
           ("SynthInfo", "awp_synth_info")]
# numpy record dtype -> C type
RECORDS = [("SRFPOINT", "awp_srf_point"), ("SEISHEADER", "awp_seisheader")]


def test_ctypes_mirrors_match_the_header_layouts(tmp_path):
    """Size and every field offset of each Python mirror (ctypes structures and
    numpy record dtypes) equal the C compiler's for the header's struct (gcc on
    this host)."""
    import ctypes
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "awp_sgt.h"', '#include "awp_synth.h"',
             'int main(void) {']
    for py, c in MIRRORS:
        cls = getattr(awpsgt, py)
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (py, c))
        for name, _ in cls._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (py, name, c, name))
    for py, c in RECORDS:
        dt = getattr(awpsgt, py)
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (py, c))
        for name in dt.names:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (py, name, c, name))
    lines.append('return 0; }')
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(tuple(l.rsplit(" ", 1)) for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                                 text=True).stdout.splitlines())
    for py, _ in MIRRORS:
        cls = getattr(awpsgt, py)
        assert int(got["%s size" % py]) == ctypes.sizeof(cls), py
        for name, _ in cls._fields_:
            assert int(got["%s %s" % (py, name)]) == getattr(cls, name).offset, (py, name)
    for py, _ in RECORDS:
        dt = getattr(awpsgt, py)
        assert int(got["%s size" % py]) == dt.itemsize, py
        for name in dt.names:
            assert int(got["%s %s" % (py, name)]) == dt.fields[name][1], (py, name)
