"""Closure convolution kernels (tcgen05 forward and input gradient, FP32
weight gradient) against the numpy checker on the same BF16 inputs."""
import ctypes as C

import numpy as np
import pytest

from closure_oracle import conv3d_dw, conv3d_dx, conv3d_fwd
from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu

# FP32 accumulation of 27*CIN BF16 products in a different order, relative to max|out|
FWD_TOL = 2e-5
DW_TOL = 2e-5


def _bf16(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


# x periods of 128 and 256 (TMA rows); 64 and 32: a 128-point tile then spans
# several periods; 96, 24, 160 and 200: tiles that wrap part of a period
SHAPES = [((5, 6, 128), 16, 32), ((4, 3, 256), 32, 32), ((3, 5, 128), 32, 16),
          ((4, 6, 64), 16, 32), ((3, 4, 32), 32, 32), ((5, 3, 64), 32, 16),
          ((3, 4, 96), 16, 32), ((4, 3, 24), 32, 32), ((3, 3, 160), 32, 16), ((2, 3, 200), 32, 32)]


@pytest.mark.parametrize("shape,cin,cout", SHAPES)
def test_conv3d_forward_and_gradients(mhd3d, shape, cin, cout):
    _gpu_or_skip(mhd3d)
    torch = pytest.importorskip("torch")
    lib = mhd3d.gpu_lib()
    nz, ny, nx = shape
    rng = np.random.default_rng(cin * 100 + cout)
    x = _bf16(torch, rng.standard_normal(shape + (cin,)))
    w = _bf16(torch, rng.standard_normal((cout, 27 * cin)) / np.sqrt(27 * cin))
    b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32)).cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    yf = torch.zeros(shape + (cout,), dtype=torch.float32, device="cuda")
    yb = torch.zeros(shape + (cout,), dtype=torch.bfloat16, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for relu in (0, 1):
        assert lib.mhd3d_conv3d(cin, cout, _p(x), _p(w), _p(b), None, relu, _p(yb), _p(yf), nx, ny, nz, _p(err),
                                C.c_void_p(s)) == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        ref = conv3d_fwd(_np(x), _np(w), _np(b), relu=bool(relu))
        scale = np.abs(ref).max()
        assert np.abs(_np(yf) - ref).max() <= FWD_TOL * scale
        assert np.abs(_np(yb) - ref).max() <= 8e-3 * scale   # BF16 rounding of the output
    # input gradient: conv(dy, wt) masked by the ReLU of the layer input
    dy = _bf16(torch, rng.standard_normal(shape + (cout,)))
    wt = torch.zeros((cin, 27 * cout), dtype=torch.bfloat16, device="cuda")
    assert lib.mhd3d_conv3d_wtranspose(cin, cout, _p(w), _p(wt), C.c_void_p(s)) == 0
    if (cout, cin) in ((16, 32), (32, 32), (32, 16)):
        dxf = torch.zeros(shape + (cin,), dtype=torch.float32, device="cuda")
        assert lib.mhd3d_conv3d(cout, cin, _p(dy), _p(wt), None, _p(x), 0, None, _p(dxf), nx, ny, nz, _p(err),
                                C.c_void_p(s)) == 0
        torch.cuda.synchronize()
        ref = conv3d_dx(_np(dy), _np(w), cin) * (_np(x) > 0)
        assert np.abs(_np(dxf) - ref).max() <= FWD_TOL * np.abs(ref).max()
    # weight gradient
    dw = torch.zeros((cout, 27 * cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    assert lib.mhd3d_conv3d_wgrad(cin, cout, _p(x), _p(dy), _p(dw), _p(db), nx, ny, nz, C.c_void_p(s)) == 0
    torch.cuda.synchronize()
    rdw, rdb = conv3d_dw(_np(x), _np(dy))
    assert np.abs(_np(dw) - rdw).max() <= DW_TOL * np.abs(rdw).max()
    assert np.abs(_np(db) - rdb).max() <= DW_TOL * np.abs(rdb).max()
