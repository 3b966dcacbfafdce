"""Multi-rank sharding of a work list, on the CPU with gloo ranks (world sizes 2 and 3):
partition coverage and balance, halo exchange of remote neighbour records, and
a sharded solve (shard.sharded_problem per rank, the oracle as the per-rank
compute) equal to the global one; records pack and unpack losslessly; a work
list with two items for one subgrid is refused."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from octotiger_b200 import amr, shard


def _small_amr():
    return amr.polytrope_batch(radius=0.05, max_level=5, seed=91)


def test_partition_covers_and_balances():
    b = _small_amr()
    w = shard.item_weights(b.items)
    for world in (2, 3, 8):
        parts = shard.partition(b.items, b.levels, b.positions, world, w)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(b.items)))
        loads = np.array([w[p].sum() for p in parts])
        assert loads.max() <= loads.mean() * 1.35 + w.max()


def test_morton_order_is_local():
    # consecutive items in a part are spatially close: parts of a uniform level are compact boxes
    from octotiger_b200 import synthetic as syn
    b = syn.uniform_level(2)
    parts = shard.partition(b.items, b.levels, b.positions, 8)
    for p in parts:
        pos = b.positions[b.items["subgrid"][p]]
        assert (pos.max(0) - pos.min(0) <= 1).all()   # each of 8 parts is one 2x2x2 octant


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_path):
    import datetime

    import torch.distributed as dist

    from oracle.pyoracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = _small_amr()
        # the function bench.py --sharded runs per rank (there with NCCL and a CUDA device)
        local = shard.sharded_problem(b, rank, world, dist)
        # every record the rank reads equals the global one
        for li, g in enumerate(local.global_ids):
            assert np.array_equal(local.pool.M[li], b.pool.M[g])
            assert np.array_equal(local.pool.mon[li], b.pool.mon[g])
            assert local.pool.is_leaf[li] == b.pool.is_leaf[g]
        L, Lc = Oracle().batch(0.5, local.pool, local.items, rho=True, nthreads=2)
        out = {int(local.global_ids[s]): (L[s], Lc[s]) for s in local.items["subgrid"]}
        np.save(f"{result_path}.{rank}.npy", np.array([out], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_solve_equals_global(tmp_path, world):
    """World sizes 2 and 3 (uneven parts, a rank whose neighbours live on
    both others)."""
    import torch.multiprocessing as mp

    from oracle.pyoracle import Oracle
    port = _free_port()
    res = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, port, res), nprocs=world, start_method="spawn", join=True)
    b = _small_amr()
    Lg, Lcg = Oracle().batch(0.5, b.pool, b.items, rho=True, nthreads=4)
    seen = set()
    for r in range(world):
        out = np.load(f"{res}.{r}.npy", allow_pickle=True)[0]
        for g, (L, Lc) in out.items():
            assert g not in seen
            seen.add(g)
            np.testing.assert_array_equal(L, Lg[g])
            np.testing.assert_array_equal(Lc, Lcg[g])
    assert seen == set(int(s) for s in b.items["subgrid"])


def test_records_round_trip():
    import torch
    b = _small_amr()
    idx = [0, 3, 5]
    t = shard.pack_records(b.pool.M[idx], b.pool.com[idx], b.pool.mon[idx], b.pool.is_leaf[idx])
    assert t.shape == (3, shard.RECORD)
    M, com, mon, leaf = shard.unpack_records(t)
    assert np.array_equal(M.numpy(), b.pool.M[idx]) and np.array_equal(com.numpy(), b.pool.com[idx])
    assert np.array_equal(mon.numpy(), b.pool.mon[idx]) and np.array_equal(leaf.numpy(), b.pool.is_leaf[idx])
    # the device path packs torch tensors the same way
    tt = shard.pack_records(*(torch.from_numpy(getattr(b.pool, k)[idx]) for k in ("M", "com", "mon", "is_leaf")))
    assert torch.equal(tt, t)


def test_partition_refuses_split_subgrid():
    b = _small_amr()
    items = np.concatenate([b.items, b.items[:1]])
    with pytest.raises(ValueError):
        shard.partition(items, b.levels, b.positions, 2)
