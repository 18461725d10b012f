"""bench.py's multi-rank timing on CPU: world_size 2 over gloo.  Every rank
reports the slowest rank's time and the whole-job rate counts all ranks."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
    q.put((rank, ms, bench.aggregate_rate(1000, 4, ms, world)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]
    # 2 ranks x 1000 cells x 4 steps in 15 ms
    assert out[0][2] == pytest.approx(2 * 1000 * 4 / 0.015 / 1e6)


def test_single_rank_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5


def test_reference_decomposition():
    """The emulated MPI layout of the CPU reference: NPEY*NPEZ ranks, a power
    of two within the cores, NPEZ dividing NPZ with at least 4 planes each."""
    sys.path.insert(0, ROOT)
    import bench
    for cores, npy, npz in ((16, 512, 32), (8, 512, 32), (12, 64, 48), (1, 64, 48), (64, 512, 32)):
        npey, npez = bench.decomposition(cores, npy, npz)
        p = npey * npez
        assert p <= cores and p & (p - 1) == 0
        assert npz % npez == 0 and npz // npez >= 4
        assert npy % npey == 0


def test_named_cases_match_their_configs():
    sys.path.insert(0, ROOT)
    import bench
    assert [bench.CASES["c1"][k] for k in ("npx", "npy", "npz", "ra", "ta")] == [64, 64, 48, 1e5, 1e4]
    assert [bench.CASES["c2"][k] for k in ("npx", "npy", "npz", "ra", "ta")] == [256, 256, 128, 1e6, 1e6]
    c5, c5d = bench.CASES["c5"], bench.CASES["c5fp64"]
    assert (c5["npx"], c5["npy"], c5["npz"], c5["mode"]) == (1024, 1024, 512, "fp32")
    assert (c5d["npx"], c5d["npy"], c5d["npz"], c5d["mode"]) == (768, 768, 384, "fast")
    for c in (c5, c5d):
        assert (c["ra"], c["ta"], c["contrast"], c["stretch"]) == (1e7, 1e7, 30.0, 2.0)
