"""The multi-GPU path has no exchange step: two gloo ranks on the CPU check
the host-side pieces bench.py uses for N > 1 - every rank draws distinct
inputs (replicas), bricks are partitioned by byte size and their results
gathered on the host (partition), the job's step time is the maximum over
ranks, and the whole-job throughput counts all ranks' bytes over it."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from cudacompress_b200 import replicas  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        wl = dict(n=16, modes=8, kmax=4, seeds=(5, 6))
        vols = bench.make_fields(wl, rank)
        # this rank's "device-timed" step times: rank 1 is slower in the first, rank 0 in the second
        mine = [10.0 + 5.0 * rank, 20.0 - 5.0 * rank]
        got = replicas.max_over_ranks(mine, dist, "cpu")
        gbs = replicas.job_gbs(world, 1 << 20, got[0])
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(got + [gbs], np.float64))
        np.save(os.path.join(out_dir, f"vol{rank}.npy"), vols[0])
        # partition of a brick set; each rank "codes" its bricks (a stand-in
        # result: the brick's byte size + 1), then the host-side gather
        sizes = [int(s) for s in np.random.default_rng(3).integers(1, 1000, 37)]
        mine_idx = replicas.partition_by_bytes(sizes, world)[rank]
        got_all = replicas.gather_on_host({i: sizes[i] + 1 for i in mine_idx}, dist)
        np.save(os.path.join(out_dir, f"gather{rank}.npy"), np.array([got_all[i] for i in range(len(sizes))]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas(tmp_path):
    world = 2
    mp.spawn(rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True)
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    assert np.array_equal(r0, r1)                           # every rank sees the same job numbers
    assert list(r0[:2]) == [15.0, 20.0]                      # element-wise max over ranks
    assert r0[2] == pytest.approx(2 * (1 << 20) / 15e-3 / 1e9)
    v0, v1 = np.load(tmp_path / "vol0.npy"), np.load(tmp_path / "vol1.npy")
    assert v0.shape == v1.shape and not np.array_equal(v0, v1)   # distinct inputs per rank
    sizes = [int(s) for s in np.random.default_rng(3).integers(1, 1000, 37)]
    for r in range(world):   # every rank holds every brick's result after the gather
        assert list(np.load(tmp_path / f"gather{r}.npy")) == [s + 1 for s in sizes]


def test_partition_by_bytes():
    rng = np.random.default_rng(11)
    for world in (1, 2, 3, 8):
        sizes = [int(s) for s in rng.integers(1, 10 ** 6, 500)]
        parts = replicas.partition_by_bytes(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))                 # each brick exactly once
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)           # balanced to within one brick
    assert replicas.partition_by_bytes([5, 5, 5], 4) == [[0], [1], [2], []]


def test_single_process_identity():
    assert replicas.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert replicas.rank_seeds((7, 8), 0) == (7, 8)
    assert replicas.rank_seeds((7, 8), 3) == (307, 308)
    with pytest.raises(ValueError):
        replicas.job_gbs(1, 100, 0.0)
