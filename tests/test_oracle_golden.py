"""The CPU oracle against golden fixtures written by the reference's own step.

tests/golden/*.npz come from the reference's STEP/FLUXES/BCON/COMMUNICATE
source, translated mechanically and run with its MPI decomposition
(tests/golden/make_golden.py).  The oracle must reproduce them bit for bit.
"""
import glob
import os

import numpy as np
import pytest

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _load(path, mhd3d):
    z = np.load(path)
    p = mhd3d.Params.from_buffer_copy(z["params"].tobytes())
    grid = {k[5:]: z[k] for k in z.files if k.startswith("grid_")}
    nf = 8 if p.lmag else 5
    fields = mhd3d.FIELDS[:nf]
    st_in = {f: np.asfortranarray(z["in_" + f]) for f in fields}
    for f in mhd3d.FIELDS[nf:]:
        st_in[f] = None
    return z, p, grid, st_in, fields


def test_fixtures_present():
    assert len(GOLDEN) >= 5


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_oracle_matches_reference_steps(path, mhd3d, oracle):
    z, p, grid, st_in, fields = _load(path, mhd3d)
    nsteps = int(z["meta"][0])
    o = oracle.Oracle(p, grid, st_in)
    r = o.step(nsteps)
    dt, timc, timt, umach, nit = z["scalars"]
    assert (r["dt"], r["timc"], r["timt"], r["umach"], r["nit"]) == (dt, timc, timt, umach, int(nit))
    got = o.get_state()
    for f in fields:
        assert np.array_equal(got[f], z["out_" + f]), f


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_oracle_matches_reference_fluxes(path, mhd3d, oracle):
    z, p, grid, st_in, fields = _load(path, mhd3d)
    o = oracle.Oracle(p, grid, st_in)
    fl = o.fluxes()
    sl = (slice(1, -1),) * 3
    for f in mhd3d.FLUXES[: len(fields)]:
        assert np.array_equal(fl[f][sl], z["flux_" + f][sl]), f


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(g)[:-4] for g in GOLDEN])
def test_oracle_matches_reference_profiles(path, mhd3d, oracle):
    z, p, grid, st_in, fields = _load(path, mhd3d)
    o = oracle.Oracle(p, grid, st_in)
    assert np.array_equal(o.profiles(), z["profiles"])
