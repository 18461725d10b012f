"""Python access to the CPU checkers (test infrastructure only).

- Oracle: the C restatement in oracle/liboracle3dmhd.so.
- run_reference: the translated reference build oracle/_ref/ref3dmhd
  (oracle/make_ref.py), run with the reference's own MPI decomposition.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EXE = os.path.join(HERE, "_ref", "ref3dmhd")

FIELDS = ("ru", "rv", "rw", "tt", "ro", "bx", "by", "bz")
NPROF = 7   # MHD3D_NPROF rows: rho, T, KE, enthalpy, convective flux, radiative flux, magnetic energy
FLUXES = ("fu", "fv", "fw", "fr", "ft", "ww1", "ww2", "ww3")
GRID_NAMES = ("exx", "dxxdx", "d2xxdx2", "ddx", "wyy", "dyydy", "d2yydy2", "ddy",
              "zee", "dzzdz", "d2zzdz2", "ddz", "rkapa", "dkapa")

_lib = None


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def oracle_lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle3dmhd.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.oracle_create.restype = vp
        lib.oracle_create.argtypes = [vp] + [vp] * 14
        lib.oracle_destroy.argtypes = [vp]
        lib.oracle_set_state.argtypes = [vp] + [vp] * 8
        lib.oracle_get_state.argtypes = [vp] + [vp] * 8
        lib.oracle_step.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.oracle_fluxes.argtypes = [vp] + [vp] * 8
        lib.oracle_cfl.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.oracle_bcon.argtypes = [vp]
        lib.oracle_profiles.argtypes = [vp, vp]
        lib.oracle_set_threads.argtypes = [C.c_int]
        lib.oracle_get_threads.restype = C.c_int
        _lib = lib
    return _lib


class Oracle:
    """CPU restatement of STEP/FLUXES/BCON/COMMUNICATE for one domain."""

    def __init__(self, params, grid: dict, state: dict | None = None):
        self.lib = oracle_lib()
        self.params = params
        self.shape = (params.npx + 2, params.npy + 2, params.npz + 2)
        self._grid = {k: np.ascontiguousarray(v) for k, v in grid.items()}
        self.h = self.lib.oracle_create(C.byref(params), *[_ptr(self._grid[n]) for n in GRID_NAMES])
        if state is not None:
            self.set_state(state)

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, state: dict):
        arrs = [None if state.get(f) is None else np.asfortranarray(state[f]) for f in FIELDS]
        self.lib.oracle_set_state(self.h, *[_ptr(a) for a in arrs])

    def get_state(self) -> dict:
        out = {f: np.zeros(self.shape, order="F") for f in FIELDS[:5]}
        for f in FIELDS[5:]:
            out[f] = np.zeros(self.shape, order="F") if self.params.lmag else None
        self.lib.oracle_get_state(self.h, *[_ptr(out[f]) for f in FIELDS])
        return out

    def step(self, n: int = 1) -> dict:
        dt, timc, timt, um = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        nit = C.c_int()
        st = self.lib.oracle_step(self.h, n, C.byref(dt), C.byref(timc), C.byref(timt), C.byref(um), C.byref(nit))
        return {"status": st, "dt": dt.value, "timc": timc.value, "timt": timt.value, "umach": um.value,
                "nit": nit.value}

    def fluxes(self) -> dict:
        out = {f: np.zeros(self.shape, order="F") for f in FLUXES}
        self.lib.oracle_fluxes(self.h, *[_ptr(out[f]) for f in FLUXES])
        return out

    def cfl(self):
        dt, um = C.c_double(), C.c_double()
        st = self.lib.oracle_cfl(self.h, C.byref(dt), C.byref(um))
        return st, dt.value, um.value

    def bcon(self):
        self.lib.oracle_bcon(self.h)

    def profiles(self) -> np.ndarray:
        """Horizontal-mean profiles, rows MHD3D_PROF_* x interior planes."""
        out = np.zeros((NPROF, self.params.npz))
        self.lib.oracle_profiles(self.h, _ptr(out))
        return out


def set_threads(n: int):
    oracle_lib().oracle_set_threads(n)


def reference_available() -> bool:
    return os.path.exists(REF_EXE)


def run_reference(params, grid: dict, state: dict, nsteps: int, npey: int = 1, npez: int = 2,
                  mode: int = 0, exe: str = REF_EXE, timeout: float = 3600.0, warmup: int = 0) -> dict:
    """Run the translated reference on the given global state.

    mode 0: nsteps x STEP, returns the fields and DT/TIMC/TIMT/UMACH/NIT.
    mode 1: one FLUXES, returns the right-hand sides.
    mode 2: the MHD3D_PROF_* profiles averaged by the reference's
            HORIZONTAL_MEAN, returned as {"profiles": (NPROF, NPZ) array}.
    warmup steps run before the timed ones ("seconds" covers the nsteps only).
    """
    nfld = 8 if params.lmag else 5
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(b"R3DI")
            f.write(struct.pack("<6i", 2, npey, npez, nsteps, mode, warmup))
            f.write(bytes(params))
            for n in GRID_NAMES:
                f.write(np.ascontiguousarray(grid[n], dtype=np.float64).tobytes())
            for fld in FIELDS[:nfld]:
                f.write(np.asfortranarray(state[fld], dtype=np.float64).tobytes(order="F"))
        r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-2000:]}")
        data = open(fout, "rb").read()
    if mode == 2:
        assert data[:4] == b"R3DP"
        return {"profiles": np.frombuffer(data, dtype=np.float64, count=NPROF * params.npz, offset=4)
                .reshape(NPROF, params.npz).copy()}
    assert data[:4] == b"R3DO"
    st, nit = struct.unpack_from("<2i", data, 4)
    dt, timc, timt, umach, nitd, secs = struct.unpack_from("<6d", data, 12)
    off = 12 + 48
    shape = (params.npx + 2, params.npy + 2, params.npz + 2)
    n = shape[0] * shape[1] * shape[2]
    names = FIELDS if mode == 0 else FLUXES
    out = {}
    for a in range(nfld):
        out[names[a]] = np.frombuffer(data, dtype=np.float64, count=n, offset=off + 8 * n * a).reshape(shape, order="F").copy()
    out.update({"dt": dt, "timc": timc, "timt": timt, "umach": umach, "nit": int(nitd), "seconds": secs})
    return out
