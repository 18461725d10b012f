"""Analytic known-answer tests of the CPU oracle (second-order operators)."""
import numpy as np


def _uniform_setup(mhd3d, nx, ny, nz, m=1.0, **kw):
    c = mhd3d.convection_config(nx, ny, nz, ampt=0.0, m=m)
    c.ngrid = mhd3d.GRID_UNIFORM
    for k, v in kw.items():
        setattr(c, k, v)
    return mhd3d.make_setup(c)


def test_uniform_state_is_stationary(mhd3d, oracle):
    """No gravity, uniform rho, T, B, zero velocity: every RHS is 0 and steps keep the state."""
    s = _uniform_setup(mhd3d, 12, 10, 12, izcon=0)
    s.params.grav = 0.0
    s.params.tb = 1.0
    st = s.copy_state()
    for f in st:
        if st[f] is not None:
            st[f][...] = 0.0
    st["ro"][...] = 1.0
    st["tt"][...] = 1.0
    st["by"][...] = 0.75      # dyadic values: the one-sided wall stencils cancel exactly
    st["bx"][...] = -0.25
    o = oracle.Oracle(s.params, s.grid, st)
    fl = o.fluxes()
    for f, v in fl.items():
        assert np.all(v[1:-1, 1:-1, 1:-1] == 0.0), f
    o.step(3)
    got = o.get_state()
    for f in ("ru", "rv", "rw", "tt", "ro", "bx", "by", "bz"):
        assert np.array_equal(got[f][1:-1, 1:-1, 1:-1], st[f][1:-1, 1:-1, 1:-1]), f


def test_hydrostatic_residual_is_second_order(mhd3d, oracle):
    """Polytrope at rest: FW = g rho - dP/dz vanishes to O(dz^2) on a uniform grid.

    m = 1.5 makes P = T^2.5 non-polynomial (for m = 1, P = T^2 and the
    centred difference is exact)."""
    res = []
    for nz in (24, 48, 96):
        s = _uniform_setup(mhd3d, 8, 8, nz, m=1.5, lmag=0, lrot=0)
        o = oracle.Oracle(s.params, s.grid, s.state)
        fw = o.fluxes()["fw"][4, 4, 2:-2]
        scale = s.params.grav * s.state["ro"][4, 4, 2:-2]
        res.append(np.abs(fw / scale).max())
    assert res[0] / res[1] > 3.5 and res[1] / res[2] > 3.7   # -> 4 as dz -> 0


def test_conduction_operator_exact_discrete_symbol(mhd3d, oracle):
    """T = T0 + e sin(2 pi x / L) at rest, no gravity: FT is the discrete second derivative times OCV/(REPR rho)."""
    s = _uniform_setup(mhd3d, 32, 8, 8, lmag=0, lrot=0)
    p = s.params
    p.grav = 0.0
    st = s.copy_state()
    nx = p.npx
    x = np.arange(nx + 2) - 1            # halo at -1 and nx wrap periodically
    L = nx                               # the domain is periodic over NPX cells
    eps = 1e-3
    for f in ("ru", "rv", "rw"):
        st[f][...] = 0.0
    st["ro"][...] = 2.0
    st["tt"][...] = 1.0 + eps * np.sin(2 * np.pi * x / L)[:, None, None]
    o = oracle.Oracle(p, s.grid, st)
    ft = o.fluxes()["ft"][1:-1, 4, 4]
    h = 1.0 / (nx - 1)                   # code-grid spacing, x physical = s * XMAX
    dx = s.grid["dxxdx"][1]              # ds/dx
    k = 2 * np.pi / L
    sym = (2 * np.cos(k) - 2) / h**2 * dx * dx
    want = p.ocv / p.repr / 2.0 * eps * np.sin(2 * np.pi * np.arange(nx) / L) * sym
    assert np.allclose(ft, want, rtol=1e-9, atol=1e-14)


def test_oracle_periodic_shift_equivariance(mhd3d, oracle):
    s = mhd3d.make_setup(mhd3d.convection_config(16, 12, 10))
    sh = {}
    for f, v in s.state.items():
        a = np.zeros_like(v)
        a[1:-1, 1:-1, :] = np.roll(np.roll(v[1:-1, 1:-1, :], 5, axis=0), -3, axis=1)
        sh[f] = mhd3d.wrap_periodic(a)
    o1 = oracle.Oracle(s.params, s.grid, s.state)
    o1.step(2)
    o2 = oracle.Oracle(s.params, s.grid, sh)
    o2.step(2)
    a, b = o1.get_state(), o2.get_state()
    for f in mhd3d.FIELDS:
        want = np.roll(np.roll(a[f][1:-1, 1:-1, :], 5, axis=0), -3, axis=1)
        assert np.array_equal(b[f][1:-1, 1:-1, :], want), f
