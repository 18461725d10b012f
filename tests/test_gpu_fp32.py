"""The FP32 form (MHD3D_MODE_FP32) against the FP64 oracle, through the C-ABI.

The FP32 form holds the state as FP32 perturbations from FP64 background
profiles (the horizontal means of TT, RO, BX, BY, BZ at upload) and computes
in FP32; metrics and the CFL reduction stay FP64.  Its error is stated per
field in two norms, both max-norms over the interior:

  rel_full = max|fp32 - oracle| / max|oracle|
  rel_pert = max|fp32 - oracle| / max|oracle - horizontal mean of oracle|

The tolerances below are the stated error bounds of the FP32 form (the
measured values are a factor of a few to ten below them).
"""
import numpy as np
import pytest

from test_gpu_parity import CASES, _cfg, _fields, _gpu_or_skip, _random_state

pytestmark = pytest.mark.gpu

# Stated error bounds of the FP32 form (measured on B200 over the cases of
# test_gpu_parity: round trip <= 6e-8; right-hand sides 1e-7..2e-6, except the
# 140-plane stretched case where the FP32 second z-differences of smooth
# fields lose eps32 * N**2 and the viscous terms reach 2.5e-4; after 10 steps
# <= 1.3e-6 of max|field| and <= 1.8e-6 of the perturbation scale; DT equal,
# UMACH <= 2e-8).
RT_PERT = 1e-7        # upload/download round trip, relative to the perturbation scale
RHS_REL = 5e-4        # right-hand sides on a random state, relative to max|F|
STEP_FULL = 5e-6      # after 10 steps, relative to max|field|
STEP_PERT = 2e-5      # after 10 steps, relative to the perturbation scale
CFL_REL = 1e-6        # DT and UMACH


def _pert_scale(a):
    inner = a[1:-1, 1:-1, 1:-1]
    mean = inner.mean(axis=(0, 1), keepdims=True)
    return max(np.abs(inner - mean).max(), 1e-300)


def _errs(got, ref):
    a, b = got[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1]
    d = np.abs(a - b).max()
    return d / max(np.abs(b).max(), 1e-300), d / _pert_scale(ref)


@pytest.fixture(scope="module", params=list(CASES))
def case(request, mhd3d):
    _gpu_or_skip(mhd3d)
    kw = dict(CASES[request.param])
    cfg = _cfg(mhd3d, kw.pop("nx"), kw.pop("ny"), kw.pop("nz"), **kw)
    return mhd3d.make_setup(cfg)


def test_fp32_roundtrip(case, mhd3d):
    st = _random_state(mhd3d, case, amp=0.01)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FP32)
    g.upload(st)
    back = g.download()
    for f in _fields(case.params):
        ref = st[f]
        # halos come back as the periodic copies of the interior (as uploaded)
        d = np.abs(back[f] - ref).max()
        assert d <= RT_PERT * _pert_scale(ref) + 1e-300, (f, d, _pert_scale(ref))
    g.close()


def test_fp32_fluxes_random_state(case, mhd3d, oracle):
    st = _random_state(mhd3d, case)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FP32)
    g.upload(st)
    o = oracle.Oracle(case.params, case.grid, st)
    fg, fo = g.fluxes(), o.fluxes()
    names = ("fu", "fv", "fw", "fr", "ft", "ww1", "ww2", "ww3")[: 8 if case.params.lmag else 5]
    for f in names:
        if f in ("fu", "fv", "fw", "ft", "ww3"):
            sl = (slice(1, -1), slice(1, -1), slice(2, -2))
        else:
            sl = (slice(1, -1), slice(1, -1), slice(1, -1))
        scale = np.abs(fo[f][sl]).max()
        assert scale > 0, f
        err = np.abs(fg[f][sl] - fo[f][sl]).max() / scale
        assert err <= RHS_REL, (f, err)
    g.close()


def test_fp32_cfl(case, mhd3d, oracle):
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FP32)
    g.upload(case.state)
    o = oracle.Oracle(case.params, case.grid, case.state)
    st, dt, um = o.cfl()
    assert st == 0
    gdt, gum = g.cfl()
    assert abs(gdt - dt) <= CFL_REL * dt, (gdt, dt)
    assert abs(gum - um) <= CFL_REL * max(um, 1e-300) + 1e-12, (gum, um)
    g.close()


def test_fp32_steps_error_per_field(case, mhd3d, oracle):
    st = _random_state(mhd3d, case, amp=0.01)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FP32)
    g.upload(st)
    o = oracle.Oracle(case.params, case.grid, st)
    rg, ro = g.step(10), o.step(10)
    assert rg["nit"] == ro["nit"]
    assert abs(rg["dt"] - ro["dt"]) <= 1e-5 * ro["dt"], (rg["dt"], ro["dt"])
    got, ref = g.download(), o.get_state()
    for f in _fields(case.params):
        full, pert = _errs(got[f], ref[f])
        assert full <= STEP_FULL and pert <= STEP_PERT, (f, full, pert)
    g.close()


def test_fp32_bcon_not_available(case, mhd3d):
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FP32)
    g.upload(case.state)
    assert mhd3d.gpu_lib().mhd3d_bcon(g.h) == 1
    g.close()
