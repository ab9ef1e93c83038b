"""The multi-GPU path's host logic with two gloo ranks on the CPU: slice sharding covers the
problem exactly once, the shards' results (computed here by the CPU oracle) assemble into the
unsharded result, and the max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest

from ttm_b200.replicas import shard_slices


def test_shard_slices_partition():
    for outer in (1, 2, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            got = [shard_slices(outer, r, world) for r in range(world)]
            assert got[0][0] == 0 and got[-1][1] == outer
            assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
            sizes = [e - b for b, e in got]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_slices(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import sys
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path.insert(0, root)
        from oracle import Oracle, dense_strides
        from ttm_b200.replicas import max_over_ranks, shard_slices
        # A (8, 6, 10) first-order, q = 2: slices k over mode 3 (outer = 10)
        na, pia, q, m = [8, 6, 10], [1, 2, 3], 2, 5
        rng = np.random.default_rng(0)            # same data on every rank
        a = rng.standard_normal(int(np.prod(na)))
        b = rng.standard_normal(m * na[q - 1])
        inner, nq, outer = 8, 6, 10
        k0, k1 = shard_slices(outer, rank, world)
        sub_na = [8, 6, k1 - k0]
        sub_nc = [8, m, k1 - k0]
        sa = a[k0 * inner * nq:k1 * inner * nq].copy()
        sc = np.zeros(int(np.prod(sub_nc)))
        Oracle().ttm(q, sa, sub_na, dense_strides(sub_na, pia), pia, b, [m, nq], [1, 2], sc, sub_nc,
                     dense_strides(sub_nc, pia))
        np.save(os.path.join(outdir, f"c{rank}.npy"), sc)
        t = max_over_ranks(1.0 + rank)
        assert t == float(world), t
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    from oracle import Oracle, dense_strides
    na, pia, q, m = [8, 6, 10], [1, 2, 3], 2, 5
    rng = np.random.default_rng(0)
    a = rng.standard_normal(int(np.prod(na)))
    b = rng.standard_normal(m * 6)
    full = np.zeros(8 * m * 10)
    Oracle().ttm(q, a, na, dense_strides(na, pia), pia, b, [m, 6], [1, 2], full, [8, m, 10],
                 dense_strides([8, m, 10], pia))
    got = np.concatenate([np.load(tmp_path / f"c{r}.npy") for r in range(world)])
    assert np.array_equal(got, full)
