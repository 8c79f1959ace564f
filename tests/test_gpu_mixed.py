"""Split-BF16 tensor-core (tcgen05) face DCT against SciPy's FP64 DCT.

Three BF16 products per k-step with FP32 accumulation keep about 16
significant bits per operand: the stated bound for one 2-D transform is a
relative L2 error below 1e-4 (typically ~1e-5).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.fft

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL_BF16X3 = 1e-4


def _dct2_bf16x3(x, kind):
    import torch

    from spectral_galerkin_heat_b200 import _lib
    L = _lib.lib()
    ny, nx = x.shape
    n = C.c_uint64()
    assert L.sgh_dct2_bf16x3_workspace_bytes(ny, nx, C.byref(n)) == 0
    ws = torch.zeros(n.value, dtype=torch.uint8, device="cuda")
    xin = torch.as_tensor(x, device="cuda")
    out = torch.full_like(xin, np.nan)
    rc = L.sgh_dct2_bf16x3(kind, ny, nx, C.c_void_p(xin.data_ptr()), C.c_void_p(out.data_ptr()),
                           C.c_void_p(ws.data_ptr()), n.value, None)
    assert rc == 0, L.sgh_last_error()
    torch.cuda.synchronize()
    status = int(ws[:4].view(torch.int32).item())
    return out.cpu().numpy(), status


@pytest.mark.parametrize("shape", [(32, 64), (64, 128), (128, 256), (17, 40), (200, 96), (256, 512)])
@pytest.mark.parametrize("kind", [2, 3])
def test_bf16x3_face_dct_matches_scipy(shape, kind):
    rng = np.random.default_rng(sum(shape) + kind)
    x = 300.0 + 50.0 * rng.standard_normal(shape)
    got, status = _dct2_bf16x3(x, kind)
    assert status == 0
    ref = scipy.fft.dctn(x, type=kind, norm="ortho")
    err = rel_l2(got, ref)
    assert err < TOL_BF16X3, err
