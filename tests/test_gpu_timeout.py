"""The bounded device-side wait: its expiry path, exercised without a fault.

Every wait of the FP64 stage kernels on their shared-memory ring is bounded;
on expiry the CTA waits (again bounded) for the copies it has in flight,
records MHD3D_ERR_TIMEOUT and returns.  mhd3d_set_wait_limit lowers the
limit of each CTA's first wait to 0 polls, so that wait gives up at once
while every copy is valid and lands: the step must report the timeout and
complete no step, and after the normal limit is restored a re-uploaded state
must step exactly as the oracle does (the reference's only run-time check is
DT<1e-8, 3dmhd.f:924; this status is the library's own).
"""
import numpy as np
import pytest

from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu

MHD3D_ERR_TIMEOUT = 6


@pytest.mark.parametrize("mode", ["EXACT", "FAST"])
def test_first_ring_wait_expiry_reports_timeout(mhd3d, oracle, mode):
    _gpu_or_skip(mhd3d)
    setup = mhd3d.make_setup(mhd3d.convection_config(40, 24, 36, ra=1e6, ta=1e6))
    o = oracle.Oracle(setup.params, setup.grid, setup.state)
    ro = o.step(3)
    ref = o.get_state()
    g = mhd3d.GpuSim(setup, mode=getattr(mhd3d, "MODE_" + mode))
    g.upload(setup.state)
    g.set_wait_limit(0)
    r = g.step(2, check=False)
    assert r["status"] == MHD3D_ERR_TIMEOUT and r["nit"] == 0, r
    # the stop holds: a further call does not step
    r = g.step(1, check=False)
    assert r["status"] == MHD3D_ERR_TIMEOUT and r["nit"] == 0, r
    # normal limit, state uploaded again: the run equals the oracle's
    g.set_wait_limit(1 << 22)
    g.upload(setup.state)
    rg = g.step(3)
    got = g.download()
    g.close()
    assert rg["nit"] == ro["nit"] == 3
    for f in mhd3d.FIELDS:
        a, b = got[f], ref[f]
        if mode == "EXACT":
            assert np.array_equal(a, b), f
        else:
            i = (slice(1, -1),) * 3
            err = np.abs(a[i] - b[i]).max() / np.abs(b[i]).max()
            assert err <= 1e-11, (f, err)
    if mode == "EXACT":
        assert rg["dt"] == ro["dt"] and rg["umach"] == ro["umach"]


def test_wait_limit_arguments(mhd3d):
    _gpu_or_skip(mhd3d)
    setup = mhd3d.make_setup(mhd3d.convection_config(16, 12, 12))
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_FP32)
    with pytest.raises(mhd3d.Mhd3dError):
        g.set_wait_limit(0)          # the FP64 stage kernels only
    g.close()
    g = mhd3d.GpuSim(setup, mode=mhd3d.MODE_EXACT)
    with pytest.raises(mhd3d.Mhd3dError):
        g.set_wait_limit(-1)
    g.close()
