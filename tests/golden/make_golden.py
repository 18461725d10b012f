"""Generate the golden fixtures of the time step from the reference's own code.

The reference has no tests or golden data.  These fixtures come from its
STEP/FLUXES/BCON/COMMUNICATE/HORIZONTAL_MEAN source, translated mechanically
to C and run with its own MPI decomposition (oracle/make_ref.py builds oracle/_ref/ref3dmhd
from the reference checkout).  Each fixture holds the inputs (COMMON scalars,
metric arrays, the state in Fortran layout) and the reference's outputs, so
tests can pin the CPU oracle without the reference checkout.

    python tests/golden/make_golden.py        # needs oracle/_ref/ref3dmhd
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rast-3dmhd_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import mhd3d  # noqa: E402
import oracle_py  # noqa: E402


def random_state(setup, seed, amp):
    """Smooth random momentum/temperature/field perturbations with live walls and ghost planes."""
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
        for f in ("bx", "by", "bz"):
            st[f] = np.asfortranarray(st[f] + smooth())
    for v in st.values():
        if v is not None:
            mhd3d.wrap_periodic(v)
    return st


def cases():
    out = []
    c = mhd3d.convection_config(12, 10, 10)
    out.append(("rot_mhd_12x10x10", c, None, 3, 1, 2))
    c = mhd3d.convection_config(12, 8, 12)
    c.lmag = 0
    out.append(("rot_hydro_12x8x12", c, None, 3, 2, 2))
    c = mhd3d.convection_config(12, 8, 12)
    c.tp, c.hh, c.itcon, c.tc, c.xp, c.yp = 0.8, 0.5, 1, 0.01, 2.0, 2.0
    out.append(("plume_itc1_tc_12x8x12", c, None, 2, 2, 2))
    c = mhd3d.convection_config(12, 8, 8)
    c.itcon, c.tp, c.lrot, c.izcon = 4, 0.05, 0, 0
    out.append(("itc4_izc0_norot_12x8x8", c, None, 2, 1, 2))
    c = mhd3d.convection_config(12, 10, 10)
    out.append(("random_mhd_12x10x10", c, (11, 0.01), 2, 1, 2))
    return out


def main():
    if not oracle_py.reference_available():
        raise SystemExit("build the translated reference first: python oracle/make_ref.py")
    for name, cfg, rnd, nsteps, npey, npez in cases():
        setup = mhd3d.make_setup(cfg)
        state = setup.state if rnd is None else random_state(setup, *rnd)
        p = setup.params
        res = oracle_py.run_reference(p, setup.grid, state, nsteps, npey=npey, npez=npez)
        flux = oracle_py.run_reference(p, setup.grid, state, 0, npey=npey, npez=npez, mode=1)
        nf = 8 if p.lmag else 5
        arrs = {"params": np.frombuffer(bytes(p), dtype=np.uint8),
                "meta": np.array([nsteps, npey, npez], dtype=np.int64),
                "scalars": np.array([res["dt"], res["timc"], res["timt"], res["umach"], res["nit"]])}
        for g in oracle_py.GRID_NAMES:
            arrs["grid_" + g] = setup.grid[g]
        for f in oracle_py.FIELDS[:nf]:
            arrs["in_" + f] = state[f]
            arrs["out_" + f] = res[f]
        for f in oracle_py.FLUXES[:nf]:
            arrs["flux_" + f] = flux[f]
        # horizontal-mean profiles by the reference's HORIZONTAL_MEAN (one y rank:
        # with more, the reference's own sum over y ranks rounds differently)
        arrs["profiles"] = oracle_py.run_reference(p, setup.grid, state, 0, npey=1, npez=npez, mode=2)["profiles"]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **arrs)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
