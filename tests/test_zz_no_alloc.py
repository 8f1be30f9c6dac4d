"""awp_field_energy_noalloc through the C ABI (GPU).

The entry point computes the same FP64 wavefield energy as awp_field_energy
but keeps its partial sums in a static device array instead of allocating
them, for callers that must not allocate device memory while solves run.
This file is collected last so that it runs both after the other GPU tests
and, with `pytest tests/test_zz_no_alloc.py`, alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

import awp_inputs as ai
import awpsgt

pytestmark = pytest.mark.gpu


def running_solver(ncomp, nt=60, dt=0.01):
    nx, ny, nz = 48, 40, 32
    media = ai.layered_media(nx, ny, nz, 200.0, seed=3, pert_std=0.05, corr_len=1000.0)
    p = awpsgt.make_params(nx, ny, nz, 200.0, dt, nt, igreen=(1, 2, 3)[:ncomp], nd=8, socalq=1, ntiskp_sgt=5,
                           write_step=4)
    s = awpsgt.Solver(p)
    s.load_media(media)
    for q in range(ncomp):
        s.set_source(q, [(24, 20, 9)], ai.gaussian_derivative_stf(nt, dt, f0=1.0, column=q))
    s.set_points(ai.sgt_points(nx, ny, 20, 20))
    s.run(35)
    return s


def field_pointers(s, ncomp):
    ptrs, L = [], None
    for q in range(ncomp):
        for f in ("u1", "v1", "w1"):
            p, L = s.device_field(f, q)
            ptrs.append(p)
    return ptrs, L


@pytest.mark.parametrize("ncomp", [1, 3])
def test_noalloc_energy_matches_allocating_call_twice(ncomp):
    import torch
    s = running_solver(ncomp)
    ptrs, L = field_pointers(s, ncomp)
    ref = awpsgt.field_energy(ptrs, L, ncomp)
    assert np.all(ref > 0)
    stream = torch.cuda.Stream()
    for _ in range(2):                                  # two calls in a row reuse the scratch
        out = torch.full((ncomp,), float("nan"), dtype=torch.float64, device="cuda")
        with torch.cuda.stream(stream):
            awpsgt.field_energy_noalloc(ptrs, L, ncomp, out, stream.cuda_stream)
        stream.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(got, ref)     # same passes, same order: bit-equal
    s.close()


def test_noalloc_energy_on_default_stream_after_a_step():
    import torch
    s = running_solver(2)
    ptrs, L = field_pointers(s, 2)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    awpsgt.field_energy_noalloc(ptrs, L, 2, out, 0)
    torch.cuda.synchronize()
    first = out.cpu().numpy()
    np.testing.assert_array_equal(first, awpsgt.field_energy(ptrs, L, 2))
    s.run(5)                                            # the wavefield moves on; so must the energy
    ptrs, L = field_pointers(s, 2)
    awpsgt.field_energy_noalloc(ptrs, L, 2, out, 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), awpsgt.field_energy(ptrs, L, 2))
    assert not np.array_equal(out.cpu().numpy(), first)
    s.close()


def test_noalloc_rejects_more_components_than_its_scratch_holds():
    import torch
    s = running_solver(1)
    ptrs, L = field_pointers(s, 1)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    lib = awpsgt.load_library()
    arr = (C.c_void_p * 12)(*(ptrs * 4))
    st = lib.awp_field_energy_noalloc(arr, 4, C.byref(L), C.c_void_p(out.data_ptr()), None)
    assert awpsgt.STATUS[st] == "AWP_ERR_PARAM"
    assert b"static scratch" in lib.awp_last_error()
    s.close()
