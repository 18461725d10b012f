"""Python binding of the 3dmhd B200 time-step library (ctypes over the C-ABI).

This is the host-side mirror a Python caller uses in place of the Fortran
driver: it builds the run set-up with libmhd3d_host.so (the driver's
initialisation, 3dmhd.f:105-496) and drives the GPU path through
libmhd3d_gpu.so (include/mhd3d.h), the drop-in for CALL STEP
(3dmhd.f:912 -> 3dmhdsub.f:687).

Arrays are numpy arrays in Fortran order with shape (NX, NY, NZ) =
(NPX+2, NPY+2, NPZ+2), exactly the reference's COMMON/BIG arrays for one
domain.  There is no CPU fallback: without the CUDA library or a GPU the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

FIELDS = ("ru", "rv", "rw", "tt", "ro", "bx", "by", "bz")
FLUXES = ("fu", "fv", "fw", "fr", "ft", "ww1", "ww2", "ww3")
# rows of mhd3d_profiles (MHD3D_PROF_*)
PROFILES = ("rho", "t", "ke", "enth", "fconv", "frad", "me")

MODE_EXACT = 0
MODE_FAST = 1
MODE_FP32 = 2

GRID_UNIFORM, GRID_ARCTAN, GRID_DIP, GRID_TANH_Z = 0, 1, 2, 3

STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "non-finite value",
          4: "DT below DTMIN", 5: "no CUDA device", 6: "device wait timed out", 7: "out of device memory"}


class Mhd3dError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: status {code} ({STATUS.get(code, '?')})")
        self.code = code


class Params(C.Structure):
    """mirror of struct mhd3d_params (include/mhd3d.h)"""
    _fields_ = [(n, C.c_int32) for n in ("npx", "npy", "npz", "lmag", "lrot", "izcon", "itcon", "ibcon",
                                          "mode", "reserved0")] + \
               [(n, C.c_double) for n in ("c13", "c23", "c43", "hx", "h2x", "hy", "h2y", "hz", "h2z",
                                           "gam1", "gam2", "gam3", "zeta1", "zeta2",
                                           "cv", "ocv", "ore", "re", "repr", "theta", "grav", "gamma", "sf",
                                           "omx", "omz", "orm", "rm", "obeta",
                                           "tb", "tp", "tc", "xp", "yp", "hh", "timi", "timc", "dtmin")]


class RunConfig(C.Structure):
    """mirror of struct mhd3d_run_config (include/mhd3d_host.h)"""
    _fields_ = [(n, C.c_int32) for n in ("npx", "npy", "npz", "lmag", "lrot", "izcon", "itcon", "ibcon",
                                          "ngrid", "ntube", "seed", "mode")] + \
               [(n, C.c_double) for n in ("xmax", "ymax", "zmax", "zstretch",
                                           "xx1", "xx2", "yy1", "yy2", "zz1", "zz2",
                                           "xa", "xb", "xc", "xd", "ya", "yb", "yc", "yd", "za", "zb", "zc", "zd",
                                           "re", "pr", "theta", "grav", "ry", "ang", "rm", "beta",
                                           "pzp", "sigma", "polys", "tp", "tc", "xp", "yp", "hh",
                                           "ampt", "ampb", "bfh", "bzp", "zcent", "rmax", "cmt", "atube",
                                           "gamma", "sff", "timi")]


_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="F_CONTIGUOUS")
_libs: dict[str, C.CDLL] = {}


def _load(name: str) -> C.CDLL:
    if name not in _libs:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise OSError(f"{path} is not built (run: make -C {HERE})")
        _libs[name] = C.CDLL(path)
    return _libs[name]


def host_lib() -> C.CDLL:
    lib = _load("libmhd3d_host.so")
    lib.mhd3d_host_params.argtypes = [C.POINTER(RunConfig), C.POINTER(Params)]
    lib.mhd3d_host_grid.argtypes = [C.POINTER(RunConfig)] + [C.c_void_p] * 14
    lib.mhd3d_host_static.argtypes = [C.POINTER(RunConfig), C.c_void_p] + [C.c_void_p] * 8
    lib.mhd3d_host_convection_config.argtypes = [C.POINTER(RunConfig), C.c_int32, C.c_int32, C.c_int32,
                                                 C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                                 C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32]
    lib.mhd3d_host_default_config.argtypes = [C.POINTER(RunConfig), C.c_int32, C.c_int32, C.c_int32]
    lib.mhd3d_host_ran2.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.mhd3d_host_ran2.restype = C.c_double
    vp = C.c_void_p
    lib.mhd3d_host_par1.argtypes = [C.POINTER(RunConfig), vp, C.c_int32, C.c_int32, C.c_int32, C.c_double,
                                    C.c_double, C.c_double, vp]
    lib.mhd3d_host_write_dump.argtypes = [C.c_char_p, C.c_int32, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32] + \
        [vp] * 8 + [C.c_double] * 4
    lib.mhd3d_host_read_dump.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                         C.c_int32, C.c_int32, vp] + [vp] * 8
    return lib


def gpu_lib() -> C.CDLL:
    lib = _load("libmhd3d_gpu.so")
    vp = C.c_void_p
    lib.mhd3d_create.argtypes = [C.POINTER(Params)] + [vp] * 14 + [C.POINTER(vp)]
    lib.mhd3d_destroy.argtypes = [vp]
    lib.mhd3d_upload.argtypes = [vp] + [vp] * 8
    lib.mhd3d_download.argtypes = [vp] + [vp] * 8
    lib.mhd3d_step.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    lib.mhd3d_fluxes.argtypes = [vp] + [vp] * 8
    lib.mhd3d_cfl.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.mhd3d_bcon.argtypes = [vp]
    lib.mhd3d_profiles.argtypes = [vp, vp]
    lib.mhd3d_ensemble_create.argtypes = [C.c_int32, C.POINTER(Params), C.POINTER(vp), C.POINTER(vp)]
    lib.mhd3d_ensemble_destroy.argtypes = [vp]
    lib.mhd3d_ensemble_member.argtypes = [vp, C.c_int32, C.POINTER(vp)]
    lib.mhd3d_ensemble_step.argtypes = [vp, C.c_int32]
    lib.mhd3d_ensemble_sync.argtypes = [vp, vp, vp, vp, vp]
    lib.mhd3d_ensemble_set_stream.argtypes = [vp, vp]
    i32 = C.c_int32
    lib.mhd3d_conv3d.argtypes = [i32, i32, vp, vp, vp, vp, i32, vp, vp, i32, i32, i32, vp, vp]
    lib.mhd3d_conv3d_wtranspose.argtypes = [i32, i32, vp, vp, vp]
    lib.mhd3d_conv3d_wgrad.argtypes = [i32, i32, vp, vp, vp, vp, i32, i32, i32, vp]
    lib.mhd3d_closure_set.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_float]
    lib.mhd3d_closure_status.argtypes = [vp, vp, vp, vp]
    lib.mhd3d_closure_set_bias.argtypes = [vp, vp]
    lib.mhd3d_coarsen.argtypes = [vp, i32, vp, vp, vp]
    lib.mhd3d_closure_features.argtypes = [vp, vp, vp, vp, vp]
    lib.mhd3d_closure_loss.argtypes = [vp, vp, C.c_int64, vp, vp, vp]
    lib.mhd3d_adam.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, i32, vp, vp]
    lib.mhd3d_closure_tendency.argtypes = [vp, vp, vp, vp, vp, C.c_float, vp]
    lib.mhd3d_closure_tendency_loss.argtypes = [vp, vp, vp, C.c_int64, vp, vp, vp]
    lib.mhd3d_closure_tendency_adjoint.argtypes = [vp, vp, vp, vp, vp]
    lib.mhd3d_ensemble_tune.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_double)]
    lib.mhd3d_ensemble_tile.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.mhd3d_ensemble_set_tile.argtypes = [vp, C.c_int32]
    lib.mhd3d_version.restype = C.c_char_p
    lib.mhd3d_set_stream.argtypes = [vp, vp]
    lib.mhd3d_step_async.argtypes = [vp, C.c_int32]
    lib.mhd3d_sync.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    lib.mhd3d_profile.argtypes = [vp, C.c_int32]
    lib.mhd3d_set_wait_limit.argtypes = [vp, C.c_int64]
    lib.mhd3d_profile_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    lib.mhd3d_cfl_noalloc.argtypes = [C.POINTER(Params)] + [vp] * 13 + [vp]
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def field_array(a, shape):
    """A field as the C-ABI reads it: float64, Fortran order, shape (NX,NY,NZ).
    Arrays in another memory order are copied (index order is kept), so a
    C-ordered array is never read transposed."""
    if a is None:
        return None
    a = np.asarray(a)
    if a.shape != tuple(shape):
        raise ValueError(f"field shape {a.shape} != {tuple(shape)}")
    return np.asfortranarray(a, dtype=np.float64)


GRID_NAMES = ("exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy",
              "zee", "dzzdz", "d2zzdz2", "ddz", "rkapa", "dkapa")


@dataclass
class Setup:
    """Everything the driver holds before its first CALL STEP."""
    config: RunConfig
    params: Params
    grid: dict
    state: dict

    @property
    def shape(self):
        p = self.params
        return (p.npx + 2, p.npy + 2, p.npz + 2)

    def grid_args(self):
        return [_ptr(self.grid[n]) for n in GRID_NAMES]

    def copy_state(self) -> dict:
        return {k: (None if v is None else v.copy(order="F")) for k, v in self.state.items()}


def default_config(npx: int, npy: int, npz: int) -> RunConfig:
    c = RunConfig()
    host_lib().mhd3d_host_default_config(C.byref(c), npx, npy, npz)
    return c


def convection_config(npx: int, npy: int, npz: int, ra: float = 1e5, ta: float = 1e4, pr: float = 1.0,
                      pm: float = 4.0, contrast: float = 10.0, m: float = 1.0, beta: float = 1e4,
                      stretch: float = 1.5, ampt: float = 2e-4, seed: int = 62659) -> RunConfig:
    """Rotating MHD polytrope from dimensionless numbers (mid-depth convention)."""
    c = RunConfig()
    host_lib().mhd3d_host_convection_config(C.byref(c), npx, npy, npz, ra, ta, pr, pm, contrast, m, beta,
                                            stretch, ampt, seed)
    return c


def make_setup(cfg: RunConfig) -> Setup:
    lib = host_lib()
    p = Params()
    st = lib.mhd3d_host_params(C.byref(cfg), C.byref(p))
    if st:
        raise Mhd3dError(st, "mhd3d_host_params")
    nx, ny, nz = cfg.npx + 2, cfg.npy + 2, cfg.npz + 2
    lens = (nx,) * 4 + (ny,) * 4 + (nz,) * 6
    grid = {n: np.zeros(L) for n, L in zip(GRID_NAMES, lens)}
    st = lib.mhd3d_host_grid(C.byref(cfg), *[_ptr(grid[n]) for n in GRID_NAMES])
    if st:
        raise Mhd3dError(st, "mhd3d_host_grid")
    shape = (nx, ny, nz)
    state = {f: np.zeros(shape, order="F") for f in FIELDS[:5]}
    for f in FIELDS[5:]:
        state[f] = np.zeros(shape, order="F") if cfg.lmag else None
    st = lib.mhd3d_host_static(C.byref(cfg), _ptr(grid["zee"]), *[_ptr(state[f]) for f in FIELDS])
    if st:
        raise Mhd3dError(st, "mhd3d_host_static")
    return Setup(cfg, p, grid, state)


def wrap_periodic(a: np.ndarray) -> np.ndarray:
    """COMM_MPI's periodic copies (y then x) on a Fortran (NX,NY,NZ) array, in place."""
    a[:, 0, :] = a[:, -2, :]
    a[:, -1, :] = a[:, 1, :]
    a[0, :, :] = a[-2, :, :]
    a[-1, :, :] = a[1, :, :]
    return a


class GpuSim:
    """A handle of the GPU time-step library (one per simulation)."""

    def __init__(self, setup: Setup, mode: int | None = None, _handle: C.c_void_p | None = None):
        self.lib = gpu_lib()
        self.setup = setup
        p = Params.from_buffer_copy(setup.params)
        if mode is not None:
            p.mode = mode
        self.params = p
        self.owned = _handle is None
        if _handle is not None:   # a member of an Ensemble, owned by it
            self.h = _handle
            return
        self.h = C.c_void_p()
        st = self.lib.mhd3d_create(C.byref(p), *setup.grid_args(), C.byref(self.h))
        if st:
            raise Mhd3dError(st, "mhd3d_create")

    def close(self):
        if self.h and self.owned:
            self.lib.mhd3d_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, state: dict):
        arrs = [field_array(state.get(f), self.setup.shape) for f in FIELDS]
        st = self.lib.mhd3d_upload(self.h, *[_ptr(a) for a in arrs])
        if st:
            raise Mhd3dError(st, "mhd3d_upload")

    def download(self) -> dict:
        shape = self.setup.shape
        lmag = self.params.lmag
        out = {f: np.zeros(shape, order="F") for f in FIELDS[:5]}
        for f in FIELDS[5:]:
            out[f] = np.zeros(shape, order="F") if lmag else None
        st = self.lib.mhd3d_download(self.h, *[_ptr(out[f]) for f in FIELDS])
        if st:
            raise Mhd3dError(st, "mhd3d_download")
        return out

    def step(self, n: int = 1, check: bool = True) -> dict:
        dt, timc, timt, umach = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        nit = C.c_int32()
        st = self.lib.mhd3d_step(self.h, n, C.byref(dt), C.byref(timc), C.byref(timt), C.byref(umach),
                                 C.byref(nit))
        if st and check:
            raise Mhd3dError(st, "mhd3d_step")
        return {"status": st, "dt": dt.value, "timc": timc.value, "timt": timt.value,
                "umach": umach.value, "nit": nit.value}

    def set_stream(self, stream_handle: int | None):
        st = self.lib.mhd3d_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None)
        if st:
            raise Mhd3dError(st, "mhd3d_set_stream")

    def step_async(self, n: int = 1):
        st = self.lib.mhd3d_step_async(self.h, n)
        if st:
            raise Mhd3dError(st, "mhd3d_step_async")

    def sync(self, check: bool = True) -> dict:
        dt, timc, timt, umach = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        nit = C.c_int32()
        st = self.lib.mhd3d_sync(self.h, C.byref(dt), C.byref(timc), C.byref(timt), C.byref(umach), C.byref(nit))
        if st and check:
            raise Mhd3dError(st, "mhd3d_sync")
        return {"status": st, "dt": dt.value, "timc": timc.value, "timt": timt.value,
                "umach": umach.value, "nit": nit.value}

    def set_wait_limit(self, polls: int):
        """Poll limit of the FP64 stage kernels' first ring wait (test use)."""
        st = self.lib.mhd3d_set_wait_limit(self.h, polls)
        if st:
            raise Mhd3dError(st, "mhd3d_set_wait_limit")

    def profile(self, enable: bool = True):
        st = self.lib.mhd3d_profile(self.h, 1 if enable else 0)
        if st:
            raise Mhd3dError(st, "mhd3d_profile")

    def profile_read(self):
        ms = (C.c_double * 3)()
        n = (C.c_int32 * 3)()
        st = self.lib.mhd3d_profile_read(self.h, ms, n)
        if st:
            raise Mhd3dError(st, "mhd3d_profile_read")
        return list(ms), list(n)

    def fluxes(self) -> dict:
        shape = self.setup.shape
        out = {f: np.zeros(shape, order="F") for f in FLUXES}
        st = self.lib.mhd3d_fluxes(self.h, *[_ptr(out[f]) for f in FLUXES])
        if st:
            raise Mhd3dError(st, "mhd3d_fluxes")
        return out

    def profiles(self) -> np.ndarray:
        """Horizontal-mean profiles (rows PROFILES) over the interior planes K=2..NZ-1."""
        out = np.zeros((len(PROFILES), self.params.npz))
        st = self.lib.mhd3d_profiles(self.h, out.ctypes.data_as(C.c_void_p))
        if st:
            raise Mhd3dError(st, "mhd3d_profiles")
        return out

    def closure_set_bias(self, bias):
        """Per-plane bias tendency of the closure, [7, NPZ] float32 (RU, RV,
        RW, TT, BX, BY, BZ; host or device array): added to an attached
        network's tendencies, or applied alone on every step when no network
        is attached; None removes it."""
        if bias is None:
            st = self.lib.mhd3d_closure_set_bias(self.h, None)
        else:
            n = 7 * self.params.npz
            if hasattr(bias, "data_ptr"):
                bias = bias.float().contiguous()
                if bias.numel() != n:
                    raise ValueError(f"closure bias has {bias.numel()} values, expected {n}")
                ptr = bias.data_ptr()
            else:
                bias = np.ascontiguousarray(bias, dtype=np.float32)
                if bias.size != n:
                    raise ValueError(f"closure bias has {bias.size} values, expected {n}")
                ptr = bias.ctypes.data
            st = self.lib.mhd3d_closure_set_bias(self.h, C.c_void_p(ptr))
        if st:
            raise Mhd3dError(st, "mhd3d_closure_set_bias")

    def closure_status(self) -> dict:
        t, e, r = C.c_int32(), C.c_int32(), C.c_int32()
        st = self.lib.mhd3d_closure_status(self.h, C.byref(t), C.byref(e), C.byref(r))
        if st:
            raise Mhd3dError(st, "mhd3d_closure_status")
        return {"trips": t.value, "evals": e.value, "err": r.value}

    def cfl(self):
        dt, um = C.c_double(), C.c_double()
        st = self.lib.mhd3d_cfl(self.h, C.byref(dt), C.byref(um))
        if st:
            raise Mhd3dError(st, "mhd3d_cfl")
        return dt.value, um.value

    def bcon(self):
        st = self.lib.mhd3d_bcon(self.h)
        if st:
            raise Mhd3dError(st, "mhd3d_bcon")


class Ensemble:
    """A batched ensemble of FP32 grids (mhd3d_ensemble_*): one persistent
    launch per RK3 stage for all members, one CUDA graph per step."""

    def __init__(self, setups: list):
        self.lib = gpu_lib()
        n = len(setups)
        self.setups = setups
        ps = (Params * n)()
        for i, su in enumerate(setups):
            ps[i] = Params.from_buffer_copy(su.params)
            ps[i].mode = MODE_FP32
        grids = (C.c_void_p * (14 * n))()
        for i, su in enumerate(setups):
            for j, a in enumerate(su.grid_args()):
                grids[14 * i + j] = a.value if isinstance(a, C.c_void_p) else a
        self.h = C.c_void_p()
        st = self.lib.mhd3d_ensemble_create(n, ps, grids, C.byref(self.h))
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_create")
        self.members = []
        for i, su in enumerate(setups):
            mh = C.c_void_p()
            st = self.lib.mhd3d_ensemble_member(self.h, i, C.byref(mh))
            if st:
                raise Mhd3dError(st, "mhd3d_ensemble_member")
            self.members.append(GpuSim(su, mode=MODE_FP32, _handle=mh))

    def close(self):
        if self.h:
            for m in self.members:
                m.h = C.c_void_p()
            self.lib.mhd3d_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step_async(self, n: int = 1):
        st = self.lib.mhd3d_ensemble_step(self.h, n)
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_step")

    def sync(self) -> dict:
        n = len(self.members)
        dt, timt = np.zeros(n), np.zeros(n)
        nit, status = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        st = self.lib.mhd3d_ensemble_sync(self.h, dt.ctypes.data_as(C.c_void_p), timt.ctypes.data_as(C.c_void_p),
                                          nit.ctypes.data_as(C.c_void_p), status.ctypes.data_as(C.c_void_p))
        if st == 2:
            raise Mhd3dError(st, "mhd3d_ensemble_sync")
        return {"status": status, "dt": dt, "timt": timt, "nit": nit, "first_status": st}

    def step(self, n: int = 1) -> dict:
        self.step_async(n)
        return self.sync()

    def set_stream(self, stream_handle: int | None):
        st = self.lib.mhd3d_ensemble_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None)
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_set_stream")

    def tune(self, steps: int = 3) -> dict:
        z, c, ms = C.c_int32(), C.c_int32(), C.c_double()
        st = self.lib.mhd3d_ensemble_tune(self.h, steps, C.byref(z), C.byref(c), C.byref(ms))
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_tune")
        tx, ty = C.c_int32(), C.c_int32()
        st = self.lib.mhd3d_ensemble_tile(self.h, C.byref(tx), C.byref(ty))
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_tile")
        return {"zlen": z.value, "ctas_per_sm": c.value, "ms_per_step": ms.value, "tile": [tx.value, ty.value]}

    def set_tile(self, rows: int):
        st = self.lib.mhd3d_ensemble_set_tile(self.h, rows)
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_set_tile")

    def tile(self) -> list:
        tx, ty = C.c_int32(), C.c_int32()
        st = self.lib.mhd3d_ensemble_tile(self.h, C.byref(tx), C.byref(ty))
        if st:
            raise Mhd3dError(st, "mhd3d_ensemble_tile")
        return [tx.value, ty.value]


def par1_record(cfg: RunConfig, ncase=1, ncasep=1, ntotal=1000, nstep0=100, nstart=0, npe=1, npey=1, nit=0,
                dt=0.0, par64=0.0, par65=0.0) -> np.ndarray:
    """The reference's 96-value PAR1 dump record (mhd3d_host_par1)."""
    out = np.zeros(96)
    ip = np.array([ncase, ncasep, ntotal, nstep0, nstart], dtype=np.int32)
    host_lib().mhd3d_host_par1(C.byref(cfg), ip.ctypes.data_as(C.c_void_p), npe, npey, nit, dt, par64, par65,
                               out.ctypes.data_as(C.c_void_p))
    return out


def write_dump(fout: str, ndump: int, par1: np.ndarray, cfg: RunConfig, state: dict, timt: float, timc: float,
               umach: float, dt: float):
    """Dump ndump of a single-domain state in the reference's .dat0/.par/.lis layout."""
    st = host_lib().mhd3d_host_write_dump(fout.encode(), ndump, np.ascontiguousarray(par1).ctypes.data_as(C.c_void_p),
                                          cfg.npx, cfg.npy, cfg.npz, cfg.lmag,
                                          *[_ptr(None if state.get(f) is None else np.asfortranarray(state[f]))
                                            for f in FIELDS], timt, timc, umach, dt)
    if st:
        raise Mhd3dError(st, "mhd3d_host_write_dump")


def read_dump(finp: str, nstart: int, npey: int, npez: int, cfg: RunConfig):
    """Restart state from dump nstart (1-based) of a run with npey x npez ranks."""
    shape = (cfg.npx + 2, cfg.npy + 2, cfg.npz + 2)
    out = {f: np.zeros(shape, order="F") for f in FIELDS[:5]}
    for f in FIELDS[5:]:
        out[f] = np.zeros(shape, order="F") if cfg.lmag else None
    par1 = np.zeros(96)
    st = host_lib().mhd3d_host_read_dump(finp.encode(), nstart, npey, npez, cfg.lmag, cfg.npx, cfg.npy, cfg.npz,
                                         par1.ctypes.data_as(C.c_void_p), *[_ptr(out[f]) for f in FIELDS])
    if st:
        raise Mhd3dError(st, "mhd3d_host_read_dump")
    return out, par1
