"""The C-ABI libraries load and export every function include/*.h declares.

No compute is called here: on a machine without a GPU, creating a handle
must fail loudly with MHD3D_ERR_NO_DEVICE rather than fall back to the CPU.
"""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:int|double|void|const\s+char\s*\*)\s*\**\s*(mhd3d_\w+)\s*\(", re.M)


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(DECL.findall(src)))


def test_gpu_library_exports_header(mhd3d):
    lib = mhd3d.gpu_lib()
    names = _declared("mhd3d.h")
    assert "mhd3d_step" in names and "mhd3d_create" in names
    for n in names:
        assert hasattr(lib, n), n
    assert lib.mhd3d_version().startswith(b"mhd3d-b200")


def test_host_library_exports_header(mhd3d):
    lib = mhd3d.host_lib()
    for n in _declared("mhd3d_host.h"):
        assert hasattr(lib, n), n


def test_no_cpu_fallback_without_gpu(mhd3d):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = mhd3d.make_setup(mhd3d.convection_config(16, 12, 12))
    with pytest.raises(mhd3d.Mhd3dError) as e:
        mhd3d.GpuSim(s)
    assert e.value.code == 5      # MHD3D_ERR_NO_DEVICE


def test_bad_arguments_rejected_before_device_use(mhd3d):
    lib = mhd3d.gpu_lib()
    assert lib.mhd3d_step(None, 1, None, None, None, None, None) == 1
    assert lib.mhd3d_upload(None, *([None] * 8)) == 1
    assert lib.mhd3d_destroy(None) == 0
    assert lib.mhd3d_closure_set_bias(None, None) == 1
    # closure convolutions: empty extents, a channel pair that is not built, missing outputs
    buf = C.create_string_buffer(64)
    p = C.cast(buf, C.c_void_p)
    err = C.cast(buf, C.POINTER(C.c_int32))
    for nx, ny, nz in ((0, 4, 4), (96, 0, 4), (200, 4, -1)):
        assert lib.mhd3d_conv3d(16, 32, p, p, None, None, 0, p, None, nx, ny, nz, err, None) == 1
        assert lib.mhd3d_conv3d_wgrad(16, 32, p, p, C.cast(buf, C.POINTER(C.c_float)), None, nx, ny, nz, None) == 1
    assert lib.mhd3d_conv3d(16, 16, p, p, None, None, 0, p, None, 96, 4, 4, err, None) == 1
    assert lib.mhd3d_conv3d(16, 32, p, p, None, None, 0, None, None, 96, 4, 4, err, None) == 1
