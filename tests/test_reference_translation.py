"""The oracle against the translated reference run live (when it is built).

oracle/_ref/ref3dmhd is built from the reference checkout by
oracle/make_ref.py; without it these tests skip (the golden fixtures still
pin the oracle).
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.reference_available():
        pytest.skip("translated reference not built (python oracle/make_ref.py)")
    return oracle


def _setup(mhd3d, nx, ny, nz, **kw):
    c = mhd3d.convection_config(nx, ny, nz, ra=kw.pop("ra", 1e5), ta=kw.pop("ta", 1e4))
    for k, v in kw.items():
        setattr(c, k, v)
    return mhd3d.make_setup(c)


@pytest.mark.parametrize("npey,npez", [(1, 2), (2, 2), (3, 2), (1, 4)])
def test_decompositions_agree_with_oracle(mhd3d, ref, npey, npez):
    s = _setup(mhd3d, 18, 12, 16)
    o = ref.Oracle(s.params, s.grid, s.state)
    ro = o.step(4)
    rr = ref.run_reference(s.params, s.grid, s.state, 4, npey=npey, npez=npez)
    assert ro["dt"] == rr["dt"] and ro["umach"] == rr["umach"] and ro["timt"] == rr["timt"]
    got = o.get_state()
    for f in mhd3d.FIELDS:
        assert np.array_equal(got[f], rr[f]), f


def test_npez1_hydro_agrees(mhd3d, ref):
    """With one z rank the reference skips only MHD one-sided stencils; hydro is unaffected."""
    s = _setup(mhd3d, 12, 10, 12, lmag=0)
    o = ref.Oracle(s.params, s.grid, s.state)
    o.step(3)
    rr = ref.run_reference(s.params, s.grid, s.state, 3, npey=1, npez=1)
    got = o.get_state()
    for f in mhd3d.FIELDS[:5]:
        assert np.array_equal(got[f], rr[f]), f


def test_npez1_mhd_differs_only_near_the_bottom(mhd3d, ref):
    """NPEZ=1 takes the ELSE IF at 3dmhdsub.f:1120-1126/1391-1392/1511-1513 and skips
    the bottom-wall one-sided stencils; the library follows NPEZ>=2, so the two
    differ first on the bottom wall plane."""
    s = _setup(mhd3d, 12, 10, 12)
    o = ref.Oracle(s.params, s.grid, s.state)
    o.step(1)
    rr = ref.run_reference(s.params, s.grid, s.state, 1, npey=1, npez=1)
    got = o.get_state()
    d = np.zeros(got["bx"].shape[2], dtype=bool)
    for f in mhd3d.FIELDS:
        d |= (got[f] != rr[f]).any(axis=(0, 1))
    ks = np.nonzero(d)[0]
    assert len(ks) > 0 and ks.min() >= s.shape[2] - 4


def test_longer_run_rot_mhd(mhd3d, ref):
    s = _setup(mhd3d, 20, 16, 24, ra=1e6, ta=1e6)
    o = ref.Oracle(s.params, s.grid, s.state)
    o.step(25)
    rr = ref.run_reference(s.params, s.grid, s.state, 25, npey=2, npez=3)
    got = o.get_state()
    for f in mhd3d.FIELDS:
        assert np.array_equal(got[f], rr[f]), f
