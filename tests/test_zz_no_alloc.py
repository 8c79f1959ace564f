"""sgh_dctn_noalloc: the DCT entry point that allocates nothing.

It exists for callers that hold device arrays but cannot allocate device
memory -- a plain ctypes host without a CUDA array library, or an application
whose memory manager owns the whole device -- so it keeps its scratch in a
fixed array inside the library instead of asking for a workspace. This file
is named to be collected last; it passes alone in a fresh process and after
the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

# same bound as the other DCT parity tests (FP64 dense contraction vs FFT)
TOL = 1e-14

SHAPES = [(16, 32, 64), (32, 64, 128), (5, 7), (37,), (3, 1, 7)]


def _dctn_with_workspace(L, kind, x, out):
    """The existing entry point, sgh_dctn, with a caller-allocated workspace."""
    import torch
    shape = (C.c_int32 * x.dim())(*x.shape)
    n = C.c_uint64()
    assert L.sgh_dctn_workspace_bytes(x.dim(), shape, C.byref(n)) == 0
    ws = torch.empty(n.value, dtype=torch.uint8, device=x.device)
    rc = L.sgh_dctn(kind, x.dim(), shape, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                    C.c_void_p(ws.data_ptr()), n.value, None)
    assert rc == 0, L.sgh_last_error()
    torch.cuda.synchronize()


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kind", [2, 3])
def test_noalloc_matches_workspace_entry_point_twice(shape, kind):
    import torch

    from spectral_galerkin_heat_b200 import _lib
    L = _lib.lib()
    x = torch.as_tensor(np.random.default_rng(sum(shape) + kind).standard_normal(shape),
                        device="cuda")
    ref = torch.empty_like(x)
    _dctn_with_workspace(L, kind, x, ref)
    cshape = (C.c_int32 * x.dim())(*x.shape)
    for _ in range(2):  # two calls in a row share the one scratch array
        got = torch.full_like(x, np.nan)
        rc = L.sgh_dctn_noalloc(kind, x.dim(), cshape, C.c_void_p(x.data_ptr()),
                                C.c_void_p(got.data_ptr()), None)
        assert rc == 0, L.sgh_last_error()
        torch.cuda.synchronize()
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < TOL


@pytest.mark.parametrize("shape", [(37,), (5, 7), (16, 32, 64)])
@pytest.mark.parametrize("kind", [2, 3])
def test_noalloc_in_place_matches_workspace_entry_point(shape, kind):
    """out aliasing in: the 1-D copy into scratch and the 2-D/3-D passes whose
    last pass writes over the input, against sgh_dctn on a copy."""
    import torch

    from spectral_galerkin_heat_b200 import _lib
    L = _lib.lib()
    x = torch.as_tensor(np.random.default_rng(7 * sum(shape) + kind).standard_normal(shape),
                        device="cuda")
    ref = torch.empty_like(x)
    _dctn_with_workspace(L, kind, x.clone(), ref)
    cshape = (C.c_int32 * x.dim())(*x.shape)
    got = x.clone()
    rc = L.sgh_dctn_noalloc(kind, x.dim(), cshape, C.c_void_p(got.data_ptr()),
                            C.c_void_p(got.data_ptr()), None)
    assert rc == 0, L.sgh_last_error()
    torch.cuda.synchronize()
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < TOL


def _largest_fitting_shape(L):
    """(64, 128, n) with the largest n whose scratch fits the built-in array."""
    limit = 16 << 20
    best = None
    for n in range(64, 200):
        shape = (C.c_int32 * 3)(64, 128, n)
        b = C.c_uint64()
        assert L.sgh_dctn_workspace_bytes(3, shape, C.byref(b)) == 0
        if b.value <= limit:
            best = (64, 128, n)
        else:
            return best, (64, 128, n)
    raise AssertionError("no shape crosses the scratch size")


def test_noalloc_at_the_scratch_boundary():
    """The largest shape that fits runs and matches sgh_dctn; one more plane is refused."""
    import torch

    from spectral_galerkin_heat_b200 import _lib
    L = _lib.lib()
    fits, over = _largest_fitting_shape(L)
    x = torch.as_tensor(np.random.default_rng(11).standard_normal(fits), device="cuda")
    ref = torch.empty_like(x)
    _dctn_with_workspace(L, 2, x, ref)
    got = torch.full_like(x, np.nan)
    rc = L.sgh_dctn_noalloc(2, 3, (C.c_int32 * 3)(*fits), C.c_void_p(x.data_ptr()),
                            C.c_void_p(got.data_ptr()), None)
    assert rc == 0, L.sgh_last_error()
    torch.cuda.synchronize()
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < TOL
    rc = L.sgh_dctn_noalloc(2, 3, (C.c_int32 * 3)(*over), C.c_void_p(x.data_ptr()),
                            C.c_void_p(got.data_ptr()), None)
    assert rc == -5


def test_noalloc_rejects_arrays_beyond_its_scratch():
    import torch

    from spectral_galerkin_heat_b200 import _lib
    L = _lib.lib()
    shape = (C.c_int32 * 3)(64, 256, 512)  # 8.4M elements: needs far more than 16 MiB
    x = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.sgh_dctn_noalloc(2, 3, shape, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), None)
    assert rc == -5  # SGH_ERR_WORKSPACE, nothing launched
    assert b"too large" in L.sgh_last_error()
