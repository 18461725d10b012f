"""Dump/restart files in the reference driver's layout (3dmhd.f:284-363,
505-524, 912-1009): .dat0.NNNN direct-access records of each rank's
interior, .par PAR1 records, .lis 80-character log records."""
import os

import numpy as np


def _state(mhd3d, cfg, seed=3):
    setup = mhd3d.make_setup(cfg)
    rng = np.random.default_rng(seed)
    st = setup.copy_state()
    for f in mhd3d.FIELDS[: 8 if cfg.lmag else 5]:
        st[f] = np.asfortranarray(st[f] + 0.01 * rng.standard_normal(st[f].shape))
        mhd3d.wrap_periodic(st[f])
    return setup, st


def test_write_layout_and_roundtrip(mhd3d, tmp_path):
    cfg = mhd3d.convection_config(12, 10, 8)
    setup, st = _state(mhd3d, cfg)
    base = str(tmp_path / "run1")
    for nd in range(2):
        par1 = mhd3d.par1_record(cfg, nstep0=100, nit=100 * (nd + 1), dt=1e-3, par64=0.0, par65=0.1 * (nd + 1))
        mhd3d.write_dump(base, nd, par1, cfg, st, timt=0.1 * (nd + 1), timc=0.1 * (nd + 1), umach=0.05, dt=1e-3)
    recl = 8 * 12 * 10 * 8
    assert os.path.getsize(base + ".dat0.0000") == 2 * 8 * recl
    assert os.path.getsize(base + ".par") == 2 * 96 * 8
    # record 8*1+5 (second dump, RO) at offset 12*recl, Fortran order of the interior
    raw = np.fromfile(base + ".dat0.0000", dtype=np.float64)
    ro = raw[12 * (recl // 8): 13 * (recl // 8)].reshape((12, 10, 8), order="F")
    assert np.array_equal(ro, st["ro"][1:-1, 1:-1, 1:-1])
    par = np.fromfile(base + ".par", dtype=np.float64).reshape(2, 96)
    assert par[1, 14] == 200.0 and par[1, 10] == 12 and par[1, 20] == 1 and par[1, 62] == 1e-3
    back, p1 = mhd3d.read_dump(base, 2, 1, 1, cfg)
    assert p1[63] + p1[64] == 0.2   # TIMI = PAR1(64) + PAR1(65) (3dmhd.f:329)
    for f in mhd3d.FIELDS:
        assert np.array_equal(back[f][1:-1, 1:-1, 1:-1], st[f][1:-1, 1:-1, 1:-1]), f
        assert np.array_equal(back[f][0, 1:-1, 1:-1], st[f][-2, 1:-1, 1:-1])   # periodic halo


def test_lis_records(mhd3d, tmp_path):
    cfg = mhd3d.convection_config(8, 8, 6)
    setup, st = _state(mhd3d, cfg)
    base = str(tmp_path / "run2")
    par1 = mhd3d.par1_record(cfg, nstep0=50, nit=100, dt=1.2345e-3)
    mhd3d.write_dump(base, 1, par1, cfg, st, timt=12.5, timc=2.25e-2, umach=0.3, dt=1.2345e-3)
    data = open(base + ".lis", "rb").read()
    irec = 59 + 7 * 100 // 50
    assert len(data) == 80 * irec
    recs = [data[80 * i: 80 * (i + 1)].decode() for i in range(irec)]
    assert all(len(r) == 80 and r.endswith("\n") for r in recs)
    assert recs[irec - 6].rstrip() == "     Iteration     100 completed"
    assert recs[irec - 4].rstrip() == "     Total simulation time:   1.2500D+01"
    assert recs[irec - 3].rstrip() == "     Present simulation time: 2.2500D-02"
    assert recs[irec - 1].rstrip() == "     Present time step:       1.2345D-03"


def test_read_multirank_dump(mhd3d, tmp_path):
    """A dump set written by NPEY x NPEZ = 2 x 3 ranks (each rank's file holds its slab)."""
    cfg = mhd3d.convection_config(8, 12, 12)
    setup, st = _state(mhd3d, cfg)
    npey, npez = 2, 3
    ny1, nz1 = 12 // npey, 12 // npez
    base = str(tmp_path / "mpi")
    par1 = mhd3d.par1_record(cfg, npe=npey * npez, npey=npey, nit=7, dt=1e-3, par64=0.5, par65=0.25)
    par1.astype(np.float64).tofile(base + ".par")
    for r in range(npey * npez):
        my, mz = r % npey, r // npey
        recs = []
        for f in mhd3d.FIELDS:
            sl = st[f][1:-1, 1 + my * ny1: 1 + (my + 1) * ny1, 1 + mz * nz1: 1 + (mz + 1) * nz1]
            recs.append(np.asfortranarray(sl).ravel(order="F"))
        np.concatenate(recs).tofile(base + ".dat0.%04d" % r)
    back, p1 = mhd3d.read_dump(base, 1, npey, npez, cfg)
    assert p1[63] + p1[64] == 0.75
    for f in mhd3d.FIELDS:
        assert np.array_equal(back[f][1:-1, 1:-1, 1:-1], st[f][1:-1, 1:-1, 1:-1]), f


def test_read_rejects_size_mismatch(mhd3d, tmp_path):
    cfg = mhd3d.convection_config(8, 8, 6)
    setup, st = _state(mhd3d, cfg)
    base = str(tmp_path / "run3")
    mhd3d.write_dump(base, 0, mhd3d.par1_record(cfg), cfg, st, 0.0, 0.0, 0.0, 0.0)
    other = mhd3d.convection_config(8, 8, 8)
    try:
        mhd3d.read_dump(base, 1, 1, 1, other)
    except mhd3d.Mhd3dError as e:
        assert e.code == 1
    else:
        raise AssertionError("size mismatch not rejected")
