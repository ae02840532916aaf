"""Host logic of the multi-GPU paths, on CPU: two `gloo` ranks on 127.0.0.1.

One SPD system does not shard (the tile Cholesky exchanges a panel every
step), so `bench.py --gpus N` runs replicas for it.  The batched solver's one
batch of independent systems does shard: lnb_batched_partition splits it
longest-processing-time first on the estimated cost n^3/3 + 2 n^2 nrhs, every
rank computing the same split; the bench times a multi-rank run as the
maximum over ranks and all-gathers per-rank summaries.  These tests run that
code with world size 2 and check the split against a direct restatement.
"""
import datetime
import os
import socket

import numpy as np
import pytest

import linompss_b200 as lnb


def _cost(ns, rs):
    ns = np.asarray(ns, dtype=np.float64)
    return ns ** 3 / 3.0 + 2.0 * ns ** 2 * np.asarray(rs, dtype=np.float64)


def _lpt_reference(ns, rs, parts):
    """the split restated: decreasing cost (equal costs by index), least-loaded part first"""
    c = _cost(ns, rs)
    order = sorted(range(len(c)), key=lambda i: (-c[i], i))
    load = np.zeros(parts)
    owner = np.empty(len(c), dtype=np.int32)
    for i in order:
        p = int(np.argmin(load))          # first minimum: lowest part on ties
        owner[i] = p
        load[p] += c[i]
    return owner, load


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_batched_partition_matches_lpt(parts):
    rng = np.random.default_rng(parts)
    ns = rng.integers(16, 513, 3000)
    rs = rng.integers(1, 9, 3000)
    owner, load = lnb.batched_partition(ns, rs, parts)
    ref_owner, ref_load = _lpt_reference(ns, rs, parts)
    np.testing.assert_array_equal(owner, ref_owner)
    np.testing.assert_allclose(load, ref_load, rtol=1e-12)
    c = _cost(ns, rs)
    assert np.isclose(load.sum(), c.sum())
    # LPT bound: no part exceeds the mean by more than the largest single system
    assert load.max() <= c.sum() / parts + c.max() + 1e-6
    o2, _ = lnb.batched_partition(ns, rs, parts)
    np.testing.assert_array_equal(owner, o2)


def test_batched_partition_edge_cases():
    owner, load = lnb.batched_partition(np.array([512, 16]), np.array([8, 1]), 4)
    assert list(owner) == [0, 1] and load[2] == 0 and load[3] == 0
    owner, load = lnb.batched_partition(np.array([], dtype=np.int32), np.array([], dtype=np.int32), 2)
    assert owner.size == 0 and np.all(load == 0)
    with pytest.raises(lnb.LinompssError):
        lnb.batched_partition(np.array([64]), np.array([1]), 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, count):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ns, rs = bench.batch_shape(count, 4321)
        mine, load = bench.shard_batch(ns, rs, world, rank)
        my_cost = float(_cost(ns[mine], rs[mine]).sum())
        slowest = bench.allmax(world, my_cost)
        summary = bench.allgather_vec(world, [float(len(mine)), my_cost])
        everyone = [None] * world
        dist.all_gather_object(everyone, mine.tolist())
        bench.barrier(world)
        if rank == 0:
            np.savez(os.path.join(out_dir, "ranks.npz"), slowest=slowest, summary=summary, load=load,
                     idx=np.array(sorted(i for part in everyone for i in part)),
                     n0=len(everyone[0]), n1=len(everyone[1]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_one_batch(tmp_path):
    import torch.multiprocessing as mp
    count = 10000
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path), count), nprocs=2, join=True)
    r = np.load(os.path.join(tmp_path, "ranks.npz"))
    # every system on exactly one rank
    np.testing.assert_array_equal(r["idx"], np.arange(count))
    assert int(r["n0"]) + int(r["n1"]) == count
    # the gathered per-rank costs are the partition's loads, the max-over-ranks their maximum
    np.testing.assert_allclose(r["summary"][:, 1], r["load"], rtol=1e-12)
    assert np.isclose(float(r["slowest"]), r["load"].max())
    assert r["summary"][:, 0].sum() == count
    # a balanced split: the two ranks' estimated work within 1 % of each other
    assert r["load"].max() / r["load"].mean() < 1.01
