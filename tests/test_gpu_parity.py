"""GPU parity: the CUDA path through the C-ABI against the CPU oracle.

Reference-rounding mode (MHD3D_MODE_EXACT) must be identical to the oracle
cell by cell (+0 == -0), including DT, UMACH, TIMC, TIMT and NIT; the FMA
mode must stay within 1e-11 of it, normwise per field
(max|gpu - oracle| / max|oracle|), after 10 steps.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-11


def _gpu_or_skip(mhd3d):
    import ctypes
    try:
        n = ctypes.c_int()
        cudart = ctypes.CDLL("libcudart.so")
        cudart.cudaGetDeviceCount(ctypes.byref(n))
        if n.value == 0:
            pytest.fail("no CUDA device on a GPU test run")
    except OSError:
        pass
    return mhd3d.gpu_lib()


def _cfg(mhd3d, nx, ny, nz, **kw):
    lmag = kw.pop("lmag", 1)
    lrot = kw.pop("lrot", 1)
    c = mhd3d.convection_config(nx, ny, nz, ra=kw.pop("ra", 1e5), ta=kw.pop("ta", 1e4))
    c.lmag, c.lrot = lmag, lrot
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _fields(p):
    return ("ru", "rv", "rw", "tt", "ro", "bx", "by", "bz")[: 8 if p.lmag else 5]


def _eq(a, b):
    return np.array_equal(a, b)


def _host_mem_gb():
    """Memory this process may still use: MemAvailable, bounded by a cgroup limit."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) / 1e6
    except OSError:
        pass
    for path in ("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory/memory.limit_in_bytes"):
        try:
            with open(path) as f:
                v = f.read().strip()
            if v != "max":
                lim = int(v) / 1e9
                avail = lim if avail is None else min(avail, lim)
        except (OSError, ValueError):
            pass
    return avail if avail is not None else 0.0


def _random_state(mhd3d, setup, seed=7, amp=0.05):
    """Smooth random velocity and field perturbations; walls and ghost planes left live."""
    rng = np.random.default_rng(seed)
    st = setup.copy_state()
    nx, ny, nz = setup.shape
    x = np.arange(nx)[:, None, None] / (nx - 2)
    y = np.arange(ny)[None, :, None] / (ny - 2)
    z = np.arange(nz)[None, None, :] / (nz - 1)
    def smooth():
        a, b, c, ph = rng.uniform(-1, 1, 4)
        return amp * (np.sin(2 * np.pi * (x + ph)) * np.cos(2 * np.pi * y + a) * np.cos(np.pi * z * (1 + b)) + 0.3 * c)
    ro = st["ro"]
    st["ru"] = np.asfortranarray(ro * smooth())
    st["rv"] = np.asfortranarray(ro * smooth())
    st["rw"] = np.asfortranarray(ro * smooth())
    st["tt"] = np.asfortranarray(st["tt"] * (1 + 0.1 * smooth()))
    if setup.params.lmag:
        st["bx"] = np.asfortranarray(st["bx"] + smooth())
        st["by"] = np.asfortranarray(st["by"] + smooth())
        st["bz"] = np.asfortranarray(st["bz"] + smooth())
    for v in st.values():
        if v is not None:
            mhd3d.wrap_periodic(v)
    return st


CASES = {
    "rot_mhd_16x12x12": dict(nx=16, ny=12, nz=12),
    "rot_mhd_40x20x18_partial_tiles": dict(nx=40, ny=20, nz=18),
    "rot_hydro_33x17x9": dict(nx=33, ny=17, nz=9, lmag=0),
    "mhd_norot_izc0_itc1": dict(nx=24, ny=16, nz=8, lrot=0, izcon=0, itcon=1),
    "plume_itc0": dict(nx=20, ny=12, nz=10, tp=0.8, hh=0.5, xp=2.0, yp=2.0),
    "itc4_half_cooler": dict(nx=20, ny=12, nz=10, itcon=4, tp=0.05),
    "z_chunks_36x10x140": dict(nx=36, ny=10, nz=140, lrot=0),
}


@pytest.fixture(scope="module", params=list(CASES))
def case(request, mhd3d):
    _gpu_or_skip(mhd3d)
    kw = dict(CASES[request.param])
    cfg = _cfg(mhd3d, kw.pop("nx"), kw.pop("ny"), kw.pop("nz"), **kw)
    return mhd3d.make_setup(cfg)


def test_roundtrip_exact(case, mhd3d, oracle):
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_EXACT)
    g.upload(case.state)
    back = g.download()
    o = oracle.Oracle(case.params, case.grid, case.state)
    ref = o.get_state()
    for f in _fields(case.params):
        assert _eq(back[f], ref[f]), f


def test_cfl_exact(case, mhd3d, oracle):
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_EXACT)
    g.upload(case.state)
    o = oracle.Oracle(case.params, case.grid, case.state)
    st, dt, um = o.cfl()
    assert st == 0
    assert g.cfl() == (dt, um)


def test_steps_exact(case, mhd3d, oracle):
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_EXACT)
    g.upload(case.state)
    o = oracle.Oracle(case.params, case.grid, case.state)
    for n in (1, 9):
        rg, ro = g.step(n), o.step(n)
        for k in ("dt", "umach", "timc", "timt", "nit"):
            assert rg[k] == ro[k], (n, k, rg[k], ro[k])
        got, ref = g.download(), o.get_state()
        for f in _fields(case.params):
            assert _eq(got[f], ref[f]), (n, f, np.abs(got[f] - ref[f]).max())


def test_steps_fast_within_tolerance(case, mhd3d, oracle):
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_FAST)
    g.upload(case.state)
    o = oracle.Oracle(case.params, case.grid, case.state)
    g.step(10)
    o.step(10)
    got, ref = g.download(), o.get_state()
    for f in _fields(case.params):
        a, b = got[f][1:-1, 1:-1, 1:-1], ref[f][1:-1, 1:-1, 1:-1]
        err = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
        assert err <= FAST_TOL, (f, err)


def test_fluxes_random_state_exact(case, mhd3d, oracle):
    st = _random_state(mhd3d, case)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_EXACT)
    g.upload(st)
    o = oracle.Oracle(case.params, case.grid, st)
    fg, fo = g.fluxes(), o.fluxes()
    names = ("fu", "fv", "fw", "fr", "ft", "ww1", "ww2", "ww3")[: 8 if case.params.lmag else 5]
    for f in names:
        if f in ("fu", "fv", "fw", "ft", "ww3"):
            sl = (slice(1, -1), slice(1, -1), slice(2, -2))   # wall values BCON discards are not reported
        else:
            sl = (slice(1, -1), slice(1, -1), slice(1, -1))
        assert np.abs(fo[f][sl]).max() > 0, f
        assert _eq(fg[f][sl], fo[f][sl]), (f, np.abs(fg[f][sl] - fo[f][sl]).max())


def test_random_state_steps_exact(case, mhd3d, oracle):
    st = _random_state(mhd3d, case, amp=0.01)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_EXACT)
    g.upload(st)
    o = oracle.Oracle(case.params, case.grid, st)
    rg, ro = g.step(3), o.step(3)
    assert rg["dt"] == ro["dt"] and rg["umach"] == ro["umach"]
    got, ref = g.download(), o.get_state()
    for f in _fields(case.params):
        assert _eq(got[f], ref[f]), f


def test_bcon_exact(case, mhd3d, oracle):
    st = _random_state(mhd3d, case)
    g = mhd3d.GpuSim(case, mode=mhd3d.MODE_EXACT)
    g.upload(st)
    g.bcon()
    o = oracle.Oracle(case.params, case.grid, st)
    o.bcon()
    got, ref = g.download(), o.get_state()
    for f in _fields(case.params):
        assert _eq(got[f][1:-1, 1:-1, 1:-1], ref[f][1:-1, 1:-1, 1:-1]), f


def test_async_equals_sync(mhd3d):
    _gpu_or_skip(mhd3d)
    s = mhd3d.make_setup(_cfg(mhd3d, 24, 16, 12))
    a = mhd3d.GpuSim(s, mode=mhd3d.MODE_EXACT)
    b = mhd3d.GpuSim(s, mode=mhd3d.MODE_EXACT)
    a.upload(s.state)
    b.upload(s.state)
    ra = a.step(5)
    b.step_async(2)
    b.step_async(3)
    rb = b.sync()
    assert ra == rb
    da, db = a.download(), b.download()
    for f in mhd3d.FIELDS:
        assert _eq(da[f], db[f])


def test_dt_small_stops_after_the_step(mhd3d, oracle):
    _gpu_or_skip(mhd3d)
    s = mhd3d.make_setup(_cfg(mhd3d, 16, 12, 12))
    s.params.dtmin = 1.0   # every DT is below it: the driver's emergency stop after step 1
    g = mhd3d.GpuSim(s, mode=mhd3d.MODE_EXACT)
    g.upload(s.state)
    r = g.step(5, check=False)
    assert r["status"] == 4 and r["nit"] == 1
    o = oracle.Oracle(s.params, s.grid, s.state)
    ro = o.step(5)
    assert ro["status"] == 4 and ro["nit"] == 1
    got, ref = g.download(), o.get_state()
    for f in mhd3d.FIELDS:
        assert _eq(got[f], ref[f])


def test_nonfinite_state_reports_status(mhd3d):
    _gpu_or_skip(mhd3d)
    s = mhd3d.make_setup(_cfg(mhd3d, 16, 12, 12))
    st = s.copy_state()
    st["ro"][5, 5, 5] = np.nan
    g = mhd3d.GpuSim(s, mode=mhd3d.MODE_EXACT)
    g.upload(st)
    r = g.step(3, check=False)
    assert r["status"] == 3 and r["nit"] == 0


def test_invalid_configurations_rejected(mhd3d):
    _gpu_or_skip(mhd3d)
    s = mhd3d.make_setup(_cfg(mhd3d, 16, 12, 12))
    for field, val in (("npz", 3), ("itcon", 2), ("izcon", 5), ("mode", 9)):
        p = mhd3d.Params.from_buffer_copy(s.params)
        setattr(p, field, val)
        bad = mhd3d.Setup(s.config, p, s.grid, s.state)
        with pytest.raises(mhd3d.Mhd3dError) as e:
            mhd3d.GpuSim(bad)
        assert e.value.code == 1


def test_full_size_one_step_exact(mhd3d, oracle):
    """The benchmark's 512x512x256 workload: one step identical to the oracle."""
    _gpu_or_skip(mhd3d)
    if _host_mem_gb() < 48:
        pytest.skip(f"needs ~40 GB of host memory for the CPU oracle, {_host_mem_gb():.0f} GB available")
    cfg = mhd3d.convection_config(512, 512, 256, ra=1e6, ta=1e6)
    s = mhd3d.make_setup(cfg)
    g = mhd3d.GpuSim(s, mode=mhd3d.MODE_EXACT)
    g.upload(s.state)
    rg = g.step(1)
    got = g.download()
    g.close()
    o = oracle.Oracle(s.params, s.grid, s.state)
    ro = o.step(1)
    assert rg["dt"] == ro["dt"] and rg["umach"] == ro["umach"]
    ref = o.get_state()
    o.close()
    for f in mhd3d.FIELDS:
        assert _eq(got[f], ref[f]), f


def test_full_size_periodic_shift_equivariance(mhd3d):
    """Uniform x,y metrics: rolling the state in x and y commutes with the step, bit for bit."""
    _gpu_or_skip(mhd3d)
    cfg = mhd3d.convection_config(512, 512, 256, ra=1e6, ta=1e6)
    s = mhd3d.make_setup(cfg)
    sh = {}
    for f, v in s.state.items():
        w = np.roll(np.roll(v[1:-1, 1:-1, :], 37, axis=0), -101, axis=1)
        a = np.zeros_like(v)
        a[1:-1, 1:-1, :] = w
        sh[f] = mhd3d.wrap_periodic(a)
    g = mhd3d.GpuSim(s, mode=mhd3d.MODE_FAST)
    g.upload(s.state)
    g.step(2)
    base = g.download()
    g.upload(sh)
    g.step(2)
    moved = g.download()
    g.close()
    for f in mhd3d.FIELDS:
        want = np.roll(np.roll(base[f][1:-1, 1:-1, :], 37, axis=0), -101, axis=1)
        assert _eq(moved[f][1:-1, 1:-1, :], want), f
