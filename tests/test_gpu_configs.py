"""The benchmark's named cases at their own sizes (CPU-checkable ones).

c1: 64x64x48 rotating MHD (Ra=1e5, Ta=1e4, Pr=1, Pm=4, contrast 10,
beta=1e4, stretch 1.5), 500 RK3 steps: the reference-rounding GPU path equals
the oracle bit for bit over the whole run; the FMA path's drift is bounded.
c2: 256x256x128 (Ra=Ta=1e6): the FP32 form's per-field error against the
FP64 oracle after 10 steps.
"""
import numpy as np
import pytest

from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu


def _c1(mhd3d):
    return mhd3d.make_setup(mhd3d.convection_config(64, 64, 48, ra=1e5, ta=1e4, pr=1.0, pm=4.0, contrast=10.0,
                                                    m=1.0, beta=1e4, stretch=1.5, ampt=2e-4, seed=1))


def test_c1_500_steps_exact_and_fast(mhd3d, oracle):
    _gpu_or_skip(mhd3d)
    setup = _c1(mhd3d)
    o = oracle.Oracle(setup.params, setup.grid, setup.state)
    ro = o.step(500)
    assert ro["status"] == 0 and ro["nit"] == 500
    ref = o.get_state()
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_EXACT)
    g.upload(setup.state)
    rg = g.step(500)
    for k in ("dt", "umach", "timc", "timt", "nit"):
        assert rg[k] == ro[k], k
    got = g.download()
    for f in mhd3d.FIELDS:
        assert np.array_equal(got[f], ref[f]), f
    g.close()
    # FMA path after 500 steps: the drift of a stable (pre-onset) run stays at rounding level
    h = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FAST)
    h.upload(setup.state)
    h.step(500)
    got = h.download()
    for f in mhd3d.FIELDS:
        a, b = got[f][1:-1, 1:-1, 1:-1], ref[f][1:-1, 1:-1, 1:-1]
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= 1e-9, (f, err)
    h.close()


def test_c2_fp32_error_per_field_after_10_steps(mhd3d, oracle):
    _gpu_or_skip(mhd3d)
    setup = mhd3d.make_setup(mhd3d.convection_config(256, 256, 128, ra=1e6, ta=1e6, pr=1.0, pm=4.0, contrast=10.0,
                                                     m=1.0, beta=1e4, stretch=1.5, ampt=2e-4, seed=1))
    o = oracle.Oracle(setup.params, setup.grid, setup.state)
    o.step(10)
    ref = o.get_state()
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    g.upload(setup.state)
    g.step(10)
    got = g.download()
    errs = {}
    for f in mhd3d.FIELDS:
        a, b = got[f][1:-1, 1:-1, 1:-1], ref[f][1:-1, 1:-1, 1:-1]
        errs[f] = float(np.abs(a - b).max() / np.abs(b).max())
    print("c2 FP32 vs FP64 oracle after 10 steps, max|d|/max|field|:", errs)
    for f, e in errs.items():
        assert e <= 5e-6, (f, e)
    g.close()
