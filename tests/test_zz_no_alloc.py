"""The allocation-free CFL entry point against the handle-based one.

mhd3d_cfl_noalloc is for hosts that cannot call cudaMalloc (static device
arrays, a framework allocator that owns the device heap, a device-memory
cap): they pass their own device arrays and output buffer, and the
reduction's scratch is a fixed __device__ array inside the library.  Its
results must equal mhd3d_cfl's in the reference-rounding mode, bit for bit,
on two calls in a row (the second call reuses the scratch the first left).
This file is collected last; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    flat = np.asfortranarray(a).ravel(order="F")
    return torch.from_numpy(flat.copy()).to("cuda")


def _call(mhd3d, torch, params, state, grid, out):
    lib = mhd3d.gpu_lib()
    dev = {f: (_dev(state[f], torch) if state.get(f) is not None else None) for f in mhd3d.FIELDS}
    met = {n: _dev(grid[n], torch) for n in ("ddx", "ddy", "ddz", "rkapa")}
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.mhd3d_cfl_noalloc(C.byref(params), *[ptr(dev[f]) for f in mhd3d.FIELDS],
                               ptr(met["ddx"]), ptr(met["ddy"]), ptr(met["ddz"]), ptr(met["rkapa"]),
                               ptr(out), C.c_void_p(stream))
    torch.cuda.synchronize()
    return st


def test_noalloc_cfl_matches_handle_twice(mhd3d):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    setup = mhd3d.make_setup(mhd3d.convection_config(40, 24, 20, ra=1e6, ta=1e6))
    sim = mhd3d.GpuSim(setup, mode=mhd3d.MODE_EXACT)
    sim.upload(setup.state)
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")

    # first call: the state as uploaded
    dt0, um0 = sim.cfl()
    assert _call(mhd3d, torch, setup.params, setup.state, setup.grid, out) == 0
    got = out.cpu().numpy()
    assert got[0] == dt0 and got[1] == um0 and got[2] == 0.0

    # second call, right after: a different state (3 steps later)
    sim.step(3)
    dt1, um1 = sim.cfl()
    state1 = sim.download()
    assert (dt1, um1) != (dt0, um0)
    out.fill_(-1.0)
    assert _call(mhd3d, torch, setup.params, state1, setup.grid, out) == 0
    got = out.cpu().numpy()
    assert got[0] == dt1 and got[1] == um1 and got[2] == 0.0
    sim.close()


def test_noalloc_cfl_hydro_and_nonfinite_flag(mhd3d):
    """The lmag=0 form (B pointers NULL) equals mhd3d_cfl bit for bit, and a
    NaN in one interior cell raises the non-finite flag."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    cfg = mhd3d.convection_config(36, 20, 16, ra=1e6, ta=1e6)
    cfg.lmag = 0
    setup = mhd3d.make_setup(cfg)
    assert setup.params.lmag == 0 and setup.state["bx"] is None
    sim = mhd3d.GpuSim(setup, mode=mhd3d.MODE_EXACT)
    sim.upload(setup.state)
    sim.step(2)
    dt, um = sim.cfl()
    state = sim.download()
    sim.close()
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(-1.0)
        assert _call(mhd3d, torch, setup.params, state, setup.grid, out) == 0
        got = out.cpu().numpy()
        assert got[0] == dt and got[1] == um and got[2] == 0.0
    bad = {f: (None if v is None else v.copy(order="F")) for f, v in state.items()}
    bad["tt"][7, 5, 9] = np.nan
    out.fill_(-1.0)
    assert _call(mhd3d, torch, setup.params, bad, setup.grid, out) == 0
    assert out.cpu().numpy()[2] == 1.0
    # and the next call on a finite state clears it again
    out.fill_(-1.0)
    assert _call(mhd3d, torch, setup.params, state, setup.grid, out) == 0
    got = out.cpu().numpy()
    assert got[0] == dt and got[1] == um and got[2] == 0.0


def test_noalloc_rejects_more_planes_than_its_scratch(mhd3d):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    lib = mhd3d.gpu_lib()
    setup = mhd3d.make_setup(mhd3d.convection_config(16, 12, 12))
    p = mhd3d.Params.from_buffer_copy(setup.params)
    p.npz = 4097
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    ptr = C.c_void_p(dummy.data_ptr())
    assert lib.mhd3d_cfl_noalloc(C.byref(p), *([ptr] * 12), ptr, None) == 1
