"""Device horizontal-mean profiles (mhd3d_profiles) against the CPU oracle,
and the long-run profile error of the FP32 form against the FP64 path.

The oracle's profiles equal the reference's HORIZONTAL_MEAN bit for bit
(tests/test_oracle_golden.py).  The device sums a plane in a different (but
fixed) order, so the FP64 modes agree with the oracle to the rounding of a
sum of NPX*NPY terms; the FP32 form to its storage precision.
"""
import numpy as np
import pytest

from test_gpu_parity import CASES, _cfg, _gpu_or_skip, _random_state

pytestmark = pytest.mark.gpu

PROF_FP64 = 1e-12     # device sum order vs the sequential oracle, relative to max|row|
                      # (measured <= 2.1e-13, on the convective flux, a cancelling sum)
PROF_FAST10 = 1e-11   # FMA mode after 10 steps
PROF_FP32 = 1e-6      # FP32 form on the same state
# long run: 256x256x128, Ra=Ta=1e6, FP32 form against the FP64 FMA path over 2000 steps,
# max over 8 samples of max|dP|/max|P| per profile.  Measured on B200: rho 1.0e-11,
# T 3.9e-12, KE 1.7e-7, enthalpy 2.2e-12, convective flux 3.0e-7, radiative flux 2.5e-10,
# magnetic energy 3.4e-9; the stated bounds are 10x those.
LONG_STEPS, LONG_EVERY = 2000, 250
LONG_TOL = {"rho": 1e-10, "t": 4e-11, "ke": 2e-6, "enth": 2e-11, "fconv": 3e-6, "frad": 3e-9, "me": 4e-8}


def _rel(a, b):
    return np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)


@pytest.fixture(scope="module", params=list(CASES))
def case(request, mhd3d):
    _gpu_or_skip(mhd3d)
    kw = dict(CASES[request.param])
    cfg = _cfg(mhd3d, kw.pop("nx"), kw.pop("ny"), kw.pop("nz"), **kw)
    return mhd3d.make_setup(cfg)


def _rows(mhd3d, p):
    return [i for i, n in enumerate(mhd3d.PROFILES) if p.lmag or n != "me"]


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_profiles_fp64(case, mhd3d, oracle, mode):
    st = _random_state(mhd3d, case, amp=0.05)
    g = mhd3d.GpuSim(case, mode=getattr(mhd3d, "MODE_" + mode.upper()))
    g.upload(st)
    o = oracle.Oracle(case.params, case.grid, st)
    r = _rel(g.profiles(), o.profiles())
    for i in _rows(mhd3d, case.params):
        assert r[i] <= PROF_FP64, (mhd3d.PROFILES[i], r[i])
    g.step(10)
    o.step(10)
    r = _rel(g.profiles(), o.profiles())
    tol = PROF_FP64 if mode == "exact" else PROF_FAST10
    for i in _rows(mhd3d, case.params):
        assert r[i] <= tol, (mhd3d.PROFILES[i], r[i])
    g.close()


def test_profiles_fp32(case, mhd3d, oracle):
    st = _random_state(mhd3d, case, amp=0.05)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FP32)
    g.upload(st)
    o = oracle.Oracle(case.params, case.grid, st)
    r = _rel(g.profiles(), o.profiles())
    for i in _rows(mhd3d, case.params):
        assert r[i] <= PROF_FP32, (mhd3d.PROFILES[i], r[i])
    g.close()


def test_long_run_profiles_fp32_vs_fp64(mhd3d):
    _gpu_or_skip(mhd3d)
    cfg = mhd3d.convection_config(256, 256, 128, ra=1e6, ta=1e6, pr=1.0, pm=4.0, contrast=10.0, m=1.0,
                                  beta=1e4, stretch=1.5, ampt=2e-4, seed=1)
    setup = mhd3d.make_setup(cfg)
    sims = {m: mhd3d.GpuSim(setup, mode=m) for m in (mhd3d.MODE_FAST, mhd3d.MODE_FP32)}
    for s in sims.values():
        s.upload(setup.state)
    worst = {n: 0.0 for n in mhd3d.PROFILES}
    for _ in range(LONG_STEPS // LONG_EVERY):
        for s in sims.values():
            s.step(LONG_EVERY)
        r = _rel(sims[mhd3d.MODE_FP32].profiles(), sims[mhd3d.MODE_FAST].profiles())
        for i, n in enumerate(mhd3d.PROFILES):
            worst[n] = max(worst[n], float(r[i]))
    print("long-run FP32 vs FP64 profile error:", worst)
    for n, tol in LONG_TOL.items():
        assert worst[n] <= tol, (n, worst[n])
    for s in sims.values():
        s.close()
