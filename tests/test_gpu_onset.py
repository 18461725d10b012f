"""Parity through convective onset, the first plume burst and the end of the run.

The other long comparisons start from +-1e-4 noise and stop while the layer
is still laminar.  These start from +-2.5e-2 temperature noise (AMPT=5e-2)
at the closure case's physics (Ra=Ta=1e6, contrast 10, tanh stretch 1.5)
and at the large case's (Ra=Ta=1e7, contrast 30, stretch 2) on reduced
grids, so that convection sets in within a few thousand steps, and run until
STEP's own checks end the run:

- 32x32x24, both physics: the first plume burst drains the density of a
  top-wall cell (to ~7e-6 of its start at the closure physics), W2 and W3
  (both proportional to RO, 3dmhdsub.f:838-851) collapse, DT halves every
  few hundred steps and the driver's DT<1e-8 check (3dmhd.f:924) stops the
  run: status MHD3D_ERR_DT_SMALL at NIT 5409 and 4389.
- 64x64x48, closure physics: the burst drives the Mach number past 0.9 and
  the centred scheme goes unstable: after step 10895 every value is still
  finite, but the temperature is negative in 4 cells and the density in 1,
  so the CFL limits of STEP (square roots of the fast-mode speed, 3dmhdsub.f
  :749-857) are not finite, and step 10896 runs with DT=NaN.

The oracle (bit-equal to the reference's own STEP, translated) does the same
in every case, so these ends are the reference scheme's behaviour on these
grids, not the GPU path's.  The reference-rounding GPU path must equal the
oracle bit for bit at every checkpoint up to and including the stop (fields,
DT, UMACH, TIMT, NIT, status).  For a non-finite state the library stops one
step earlier than the oracle: it ends the run when the CFL reduction of the
state after step N meets a non-finite value and does not run step N+1 with a
non-finite DT; the oracle runs that step (all NaN) and then reports.  The
test checks that the state after step N is the same on both sides, that the
oracle's CFL of it is not finite, and the oracle's status one step later.

The FMA path and the FP32 form are checked on the horizontal-mean profiles
(HORIZONTAL_MEAN, 3dmhdsub.f:3143-3223) of KE, enthalpy and convective flux
at every checkpoint, relative L2 against the oracle's.  Measured on B200:
FMA <= 1.2e-13 on every profile; FP32 KE <= 1.4e-5, enthalpy <= 1e-7,
convective flux <= 1.4e-5 (the largest just before the DT collapse).  The FMA
path stops at the oracle's step with its status; the FP32 form ends the same
way within 10 % of the oracle's step count.
"""
import numpy as np
import pytest

from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu

AMPT = 5e-2
CLOSURE_PHYSICS = dict(ra=1e6, ta=1e6, contrast=10.0, stretch=1.5)
LARGE_PHYSICS = dict(ra=1e7, ta=1e7, contrast=30.0, stretch=2.0)
# name: (grid, physics, checkpoint interval, expected end: status, NIT on the GPU)
CASES = {
    "closure_32x32x24": ((32, 32, 24), CLOSURE_PHYSICS, 250, (4, 5409)),
    "large_32x32x24": ((32, 32, 24), LARGE_PHYSICS, 250, (4, 4389)),
    "closure_64x64x48": ((64, 64, 48), CLOSURE_PHYSICS, 500, (3, 10895)),
}
# relative L2 of the KE, enthalpy and convective-flux profiles against the oracle
FAST_PROF_TOL = 1e-12
FP32_PROF_TOL = {"ke": 5e-5, "enth": 1e-6, "fconv": 5e-5}
ROWS = {"ke": 2, "enth": 3, "fconv": 4}    # MHD3D_PROF_KE, _ENTH, _FCONV


def _rel_l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max(float((b ** 2).sum()), 1e-300)))


def _same_state(mhd3d, a, b):
    return all(np.array_equal(a[f], b[f], equal_nan=True) for f in mhd3d.FIELDS)


@pytest.mark.parametrize("name", list(CASES))
def test_onset_to_end_of_run(mhd3d, oracle, name):
    _gpu_or_skip(mhd3d)
    (nx, ny, nz), phys, chunk, (end_status, end_nit) = CASES[name]
    setup = mhd3d.make_setup(mhd3d.convection_config(nx, ny, nz, ampt=AMPT, **phys))
    orc = oracle.Oracle(setup.params, setup.grid, setup.state)
    sims = {m: mhd3d.GpuSim(setup, mode=getattr(mhd3d, "MODE_" + m.upper())) for m in ("exact", "fast", "fp32")}
    for g in sims.values():
        g.upload(setup.state)
    n = 0
    umach_max = 0.0
    ke_first = None
    fp32_worst = {k: 0.0 for k in ROWS}
    fast_worst = 0.0
    ended = {}
    while "exact" not in ended:
        assert n < 2 * end_nit, "the run did not end where the oracle's does"
        rg = sims["exact"].step(chunk, check=False)
        steps = rg["nit"] - n
        ro = orc.step(steps)
        if rg["status"] == 3:
            # the GPU stopped at the CFL of a non-finite state: the oracle,
            # after the same steps, holds the same state and stops one step later
            assert ro["status"] == 0 and ro["nit"] == rg["nit"]
            assert _same_state(mhd3d, sims["exact"].download(), orc.get_state())
            assert orc.cfl()[0] == 3    # its CFL limits are not finite
            ro1 = orc.step(1)
            assert ro1["status"] == 3 and ro1["nit"] == rg["nit"] + 1 and not np.isfinite(ro1["dt"])
        else:
            for k in ("status", "nit", "dt", "umach", "timc", "timt"):
                assert rg[k] == ro[k], (name, n, k, rg[k], ro[k])
            assert _same_state(mhd3d, sims["exact"].download(), orc.get_state()), (name, rg["nit"])
        n = rg["nit"]
        if rg["status"]:
            ended["exact"] = (rg["status"], rg["nit"])
            break
        umach_max = max(umach_max, ro["umach"])
        prof_o = orc.profiles()
        if ke_first is None:
            ke_first = float(prof_o[ROWS["ke"]].mean())
        # the FMA path and the FP32 form at the same step
        for m in ("fast", "fp32"):
            if m in ended:
                continue
            r = sims[m].step(chunk, check=False)
            if r["status"] or r["nit"] != n:
                ended[m] = (r["status"], r["nit"])
                continue
            prof = sims[m].profiles()
            for key, row in ROWS.items():
                e = _rel_l2(prof[row], prof_o[row])
                if m == "fast":
                    fast_worst = max(fast_worst, e)
                else:
                    fp32_worst[key] = max(fp32_worst[key], e)
    print(name, "end", ended, "max Mach", umach_max, "fast worst", fast_worst, "fp32 worst", fp32_worst)
    assert ended["exact"] == (end_status, end_nit)
    # the run went through onset: the Mach number grew past 0.15 and the mean KE tenfold
    assert umach_max > 0.15
    ke_peak = float(orc.profiles()[ROWS["ke"]].mean()) if end_status == 4 else None
    if ke_peak is not None:
        assert ke_peak > 10 * ke_first
    assert fast_worst <= FAST_PROF_TOL, fast_worst
    for key, tol in FP32_PROF_TOL.items():
        assert fp32_worst[key] <= tol, (key, fp32_worst[key])
    # the FMA path ends where the oracle's does
    while "fast" not in ended:
        r = sims["fast"].step(chunk, check=False)
        if r["status"] or r["nit"] > 1.2 * end_nit:
            ended["fast"] = (r["status"], r["nit"])
    assert ended["fast"][0] == end_status and abs(ended["fast"][1] - end_nit) <= 1, ended["fast"]
    # the FP32 form: a non-finite end within 10 % of the oracle's step; a DT
    # collapse the same way, DT below 1e-7 at the oracle's last step (the
    # FP32 perturbation of the drained wall density bottoms out near the
    # FP32 resolution of its background, so its own DT<1e-8 stop comes later
    # or not at all)
    g32 = sims["fp32"]
    if "fp32" in ended:
        s32, nit32, dt32 = ended["fp32"] + (None,)
    else:
        r = g32.step(0, check=False)
        nit32 = r["nit"]
        s32, dt32 = 0, None
        while s32 == 0 and nit32 < end_nit:
            r = g32.step(min(chunk, end_nit - nit32), check=False)
            s32, nit32, dt32 = r["status"], r["nit"], r["dt"]
    if end_status == 3:
        while s32 == 0 and nit32 < 1.1 * end_nit:
            r = g32.step(chunk, check=False)
            s32, nit32 = r["status"], r["nit"]
        assert s32 == 3 and abs(nit32 - end_nit) <= 0.1 * end_nit, (s32, nit32)
    else:
        assert s32 == 4 or (dt32 is not None and dt32 < 1e-7), (s32, nit32, dt32)
    for g in sims.values():
        g.close()
