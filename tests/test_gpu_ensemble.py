"""The batched FP32 ensemble (mhd3d_ensemble_*) against single-grid FP32 runs.

An ensemble runs every member's stages in one persistent launch per stage
and a step as a CUDA graph; the arithmetic per cell is the same as the
single-grid FP32 kernel's, so each member must match the same grid stepped
alone bit for bit, whatever the z-chunk length the autotuner picks.
"""
import numpy as np
import pytest

from test_gpu_parity import _gpu_or_skip

pytestmark = pytest.mark.gpu

SPECS = [  # uneven grids, partial tiles, members of very different work
    (64, 64, 48, 1e5, 1e4, 1),
    (40, 20, 18, 1e6, 1e5, 2),
    (96, 64, 32, 1e4, 1e3, 3),
    (33, 17, 12, 1e5, 1e6, 4),
]


def _setups(mhd3d):
    out = []
    for nx, ny, nz, ra, ta, seed in SPECS:
        cfg = mhd3d.convection_config(nx, ny, nz, ra=ra, ta=ta, ampt=1e-3, seed=seed)
        out.append(mhd3d.make_setup(cfg))
    return out


def _singles(mhd3d, setups, nsteps):
    res = []
    for su in setups:
        g = mhd3d.GpuSim(su, mode=mhd3d.MODE_FP32)
        g.upload(su.state)
        r = g.step(nsteps)
        res.append((r, g.download()))
        g.close()
    return res


def _check(mhd3d, ens, singles):
    for m, (r, st) in zip(ens.members, singles):
        got = m.download()
        for f in mhd3d.FIELDS[: 8 if m.params.lmag else 5]:
            assert np.array_equal(got[f], st[f]), f


def test_ensemble_matches_single_runs(mhd3d):
    _gpu_or_skip(mhd3d)
    setups = _setups(mhd3d)
    ens = mhd3d.Ensemble(setups)
    for m, su in zip(ens.members, setups):
        m.upload(su.state)
    r = ens.step(7)
    assert r["first_status"] == 0
    singles = _singles(mhd3d, setups, 7)
    for i, (rs, _) in enumerate(singles):
        assert r["nit"][i] == rs["nit"] == 7
        assert r["dt"][i] == rs["dt"]
    _check(mhd3d, ens, singles)
    # profiles of a member through its handle
    p = ens.members[0].profiles()
    assert np.isfinite(p).all() and p.shape == (len(mhd3d.PROFILES), setups[0].params.npz)
    ens.close()


def test_ensemble_tune_leaves_state(mhd3d):
    _gpu_or_skip(mhd3d)
    setups = _setups(mhd3d)
    ens = mhd3d.Ensemble(setups)
    for m, su in zip(ens.members, setups):
        m.upload(su.state)
    ens.step(2)
    t = ens.tune(steps=2)
    # the search: tile rows 2, 4, 8 (32 columns) x z chunk x CTAs per SM
    assert t["zlen"] in (4, 6, 8, 12, 16, 24, 32, 48, 64)
    allowed = {2: (4, 6, 8), 4: (2, 3, 4), 8: (1, 2)}
    assert t["tile"][0] == 32 and t["ctas_per_sm"] in allowed[t["tile"][1]], t
    assert t["ms_per_step"] > 0 and ens.tile() == t["tile"]
    r = ens.step(3)
    assert list(r["nit"]) == [5] * len(setups)
    _check(mhd3d, ens, _singles(mhd3d, setups, 5))
    ens.close()


@pytest.mark.parametrize("rows", [2, 8])
def test_ensemble_tile_shapes_give_the_same_bits(mhd3d, rows):
    """The 32x2 and 32x8 tile instances against single-grid runs (32x4)."""
    _gpu_or_skip(mhd3d)
    setups = _setups(mhd3d)
    ens = mhd3d.Ensemble(setups)
    ens.set_tile(rows)
    assert ens.tile() == [32, rows]
    for m, su in zip(ens.members, setups):
        m.upload(su.state)
    r = ens.step(5)
    assert list(r["nit"]) == [5] * len(setups)
    _check(mhd3d, ens, _singles(mhd3d, setups, 5))
    with pytest.raises(mhd3d.Mhd3dError):
        ens.set_tile(3)
    ens.close()


def test_ensemble_member_stop_is_isolated(mhd3d):
    _gpu_or_skip(mhd3d)
    setups = _setups(mhd3d)
    setups[1].params.dtmin = 1.0      # this member's DT check trips after its first step
    ens = mhd3d.Ensemble(setups)
    for m, su in zip(ens.members, setups):
        m.upload(su.state)
    r = ens.step(4)
    assert r["status"][1] == 4 and r["nit"][1] == 1        # MHD3D_ERR_DT_SMALL
    for i in (0, 2, 3):
        assert r["status"][i] == 0 and r["nit"][i] == 4
    setups[1].params.dtmin = 1e-8
    _check(mhd3d, ens, [s if i != 1 else (None, ens.members[1].download()) for i, s in
                        enumerate(_singles(mhd3d, setups, 4))])
    ens.close()
