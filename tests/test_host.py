"""Host set-up mirror: literal rounding, RAN2, grid maps, static state."""
import ctypes as C

import numpy as np


def f32(x):
    return float(np.float32(x))


def test_params_hold_float_rounded_literals(mhd3d):
    s = mhd3d.make_setup(mhd3d.convection_config(64, 64, 48))
    p = s.params
    assert p.c13 == f32(np.float32(1) / np.float32(3))
    assert p.c43 == 4.0 * p.c13 and p.c23 == 2.0 * p.c13
    assert p.gam1 == float(np.float32(8) / np.float32(15))
    assert p.gam2 == float(np.float32(5) / np.float32(12))
    assert p.gam3 == 0.75
    assert p.zeta1 == float(np.float32(-17) / np.float32(60))
    assert p.zeta2 == float(np.float32(-5) / np.float32(12))
    assert p.sf == f32(0.4) and p.gamma == float(np.float32(5) / np.float32(3))
    assert p.hx == 31.5 and p.h2x == 63.0 * 63.0
    assert p.dtmin == f32(1e-8)
    assert p.cv == 1.0 / (p.gamma - 1.0) and p.ocv == 1.0 / p.cv


def _ran2_reference(idum, n):
    """Numerical-Recipes RAN2 (M=714025, IA=1366, IC=150889) restated independently."""
    M, IA, IC = 714025, 1366, 150889
    rm = float(np.float32(1.0) / np.float32(714025.0))
    ir = [0] * 97
    idum = (IC - idum) % M
    for j in range(97):
        idum = (IA * idum + IC) % M
        ir[j] = idum
    idum = (IA * idum + IC) % M
    iy = idum
    out = []
    for _ in range(n):
        j = 1 + (97 * iy) // M
        iy = ir[j - 1]
        out.append(iy * rm)
        idum = (IA * idum + IC) % M
        ir[j - 1] = idum
    return out


def test_ran2_sequence(mhd3d):
    lib = mhd3d.host_lib()
    idum, iy, ir = C.c_int32(-62659), C.c_int32(0), (C.c_int32 * 97)()
    got = [lib.mhd3d_host_ran2(C.byref(idum), C.byref(iy), ir) for _ in range(500)]
    assert got == _ran2_reference(-62659, 500)
    assert all(0.0 <= v < 1.0 for v in got)


def test_uniform_and_tanh_grid(mhd3d):
    cfg = mhd3d.convection_config(32, 24, 40, stretch=1.5)
    s = mhd3d.make_setup(cfg)
    g = s.grid
    assert np.all(g["dxxdx"][1:-1] == 1.0 / 4.0) and np.all(g["d2xxdx2"][1:-1] == 0.0)
    z = g["zee"][1:-1]
    assert z[0] == 0.0 and z[-1] == 1.0 and np.all(np.diff(z) > 0)
    dz = np.diff(z)
    assert dz[0] < dz[-1]                       # clustered at the top
    # metric = ds/dz, checked against centred differences of z(s)
    ds = 1.0 / 39
    dzds = (z[2:] - z[:-2]) / (2 * ds)
    assert np.allclose(g["dzzdz"][2:-2], 1.0 / dzds, rtol=2e-3)
    d2 = (z[2:] - 2 * z[1:-1] + z[:-2]) / ds**2
    want = -d2 * g["dzzdz"][2:-2] ** 3
    assert np.allclose(g["d2zzdz2"][2:-2], want, rtol=5e-3, atol=1e-3 * np.abs(want).max())


def test_static_polytrope_and_layer(mhd3d):
    cfg = mhd3d.convection_config(16, 12, 20, ampt=0.0)
    s = mhd3d.make_setup(cfg)
    p, st, z = s.params, s.state, s.grid["zee"]
    t = 1.0 + cfg.theta * z[1:-1]
    assert np.allclose(st["tt"][5, 5, 1:-1], t, rtol=1e-13)
    assert st["tt"][5, 5, 0] == 1.0 and st["tt"][5, 5, -1] == p.tb == 1.0 + cfg.theta
    by = st["by"][5, 5, 1:-1]
    assert np.all(by == 1.0)                    # TUBE model 4 with RMAX >> ZMAX
    rho_poly = t ** (cfg.grav / cfg.theta) / t
    assert np.allclose(st["ro"][5, 5, 1:-1], (rho_poly * t - by**2 * p.obeta / 2) / t, rtol=1e-12)
    assert np.all(st["ru"] == 0) and np.all(st["bz"] == 0)
    # periodic halos as COMMUNICATE leaves them
    assert np.array_equal(st["tt"][0], st["tt"][-2]) and np.array_equal(st["tt"][:, -1], st["tt"][:, 1])


def test_perturbation_amplitude(mhd3d):
    cfg = mhd3d.convection_config(16, 12, 20, ampt=2e-4)
    base = mhd3d.make_setup(mhd3d.convection_config(16, 12, 20, ampt=0.0)).state["tt"]
    tt = mhd3d.make_setup(cfg).state["tt"]
    rel = tt[1:-1, 1:-1, 1:-1] / base[1:-1, 1:-1, 1:-1] - 1.0
    assert np.abs(rel).max() <= 1e-4 + 1e-12 and np.abs(rel).max() > 9e-5


def test_dimensionless_mapping(mhd3d):
    cfg = mhd3d.convection_config(16, 16, 16, ra=1e5, ta=1e4, pm=4.0)
    # 178.2 assumes gamma = 5/3 exactly; the host uses the REAL(4) 5.00E00/3.00E00
    assert abs(cfg.re - np.sqrt(1e5 / 178.2)) < 1e-6 * cfg.re
    assert abs(cfg.theta - 9.0) < 1e-12 and abs(cfg.grav - 18.0) < 1e-12
    rho_mid = 5.5
    assert abs(cfg.ry - cfg.re * rho_mid / 100.0) < 1e-12 * cfg.ry
    assert abs(cfg.rm - 4.0 * cfg.re * rho_mid) < 1e-12 * cfg.rm


def test_field_array_keeps_index_order(mhd3d):
    """A C-ordered field is copied to Fortran order, never read transposed."""
    import numpy as np
    a = np.arange(4 * 3 * 2, dtype=np.float32).reshape(4, 3, 2)   # C order
    f = mhd3d.field_array(a, (4, 3, 2))
    assert f.flags.f_contiguous and f.dtype == np.float64
    assert np.array_equal(f, a)
    g = np.asfortranarray(a, dtype=np.float64)
    assert mhd3d.field_array(g, (4, 3, 2)) is g or np.shares_memory(mhd3d.field_array(g, (4, 3, 2)), g)
    assert mhd3d.field_array(None, (4, 3, 2)) is None
    import pytest
    with pytest.raises(ValueError):
        mhd3d.field_array(a, (2, 3, 4))
