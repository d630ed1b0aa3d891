"""Multi-GPU batched builds: every rank takes a bin-packed share of the
collection and the ranks reduce only their timings.  Checked on CPU with
gloo ranks (world size 2)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sufkit_b200 import shard, synth


def test_assign_covers_disjoint_and_balanced():
    rng = np.random.default_rng(3)
    for ranks in (1, 2, 3, 4, 8):
        sizes = [int(x) for x in rng.integers(1, 1_000_000, size=257)]
        shares = shard.assign(sizes, ranks)
        assert len(shares) == ranks
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in s) for s in shares]
        # LPT: the heaviest share exceeds the mean by at most one item.
        assert max(loads) <= sum(sizes) / ranks + max(sizes)
        assert all(s == sorted(s) for s in shares)


def test_assign_small_cases():
    assert shard.assign([], 3) == [[], [], []]
    assert shard.assign([5], 2) == [[0], []]
    assert shard.assign([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]
    assert shard.assign([9, 1, 1, 1, 1, 1, 1, 1, 1, 1], 2) == [[0], list(range(1, 10))]
    with pytest.raises(ValueError):
        shard.assign([1], 0)


def test_reductions_without_group():
    assert shard.max_over_ranks(2.5) == 2.5
    assert shard.sum_over_ranks(7) == 7.0


def test_uneven_reference_is_independent_of_the_rest():
    sizes = synth.uneven_sizes(6, scale=0.001)
    assert sizes == synth.uneven_sizes(6, scale=0.001)
    assert all(s >= 500 for s in sizes)
    a = synth.uneven_reference(4, sizes[4]).logical_text()
    b = synth.uneven_reference(4, sizes[4]).logical_text()
    c = synth.uneven_reference(5, sizes[4]).logical_text()
    assert a.size == b.size and (a == b).all()
    assert a.size != c.size or not (a == c).all()
    contigs = synth.uneven_reference(4, sizes[4]).contigs
    assert sum(x.size for x in contigs) == sizes[4]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_collection_shares_make_up_the_collection():
    world, count, scale = 3, 7, 0.001
    seen = {}
    for rank in range(world):
        idx, texts = shard.collection_share(count, world, rank, scale)
        for i, t in zip(idx, texts):
            assert i not in seen
            seen[i] = t
    assert sorted(seen) == list(range(count))
    sizes = synth.uneven_sizes(count, scale)
    for i, t in seen.items():
        one = synth.uneven_reference(i, sizes[i]).logical_text()
        assert one.size == t.size and (one == t).all()


def _rank_main(rank, world, port, sizes, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        share = shard.assign(sizes, world)[rank]
        # Each rank's "time" is its share's size: the reduction must give
        # the heaviest share on every rank.
        load = float(sum(sizes[i] for i in share))
        out[rank] = (share, load, shard.max_over_ranks(load, dist),
                     shard.sum_over_ranks(load, dist))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    sizes = [s + 1 for s in synth.uneven_sizes(17, scale=0.01)]
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), sizes, out),
                           nprocs=world, join=True, start_method="spawn")
        got = dict(out)
    shares = [got[r][0] for r in range(world)]
    assert sorted(i for s in shares for i in s) == list(range(len(sizes)))
    loads = [got[r][1] for r in range(world)]
    assert got[0][2] == got[1][2] == max(loads)
    assert got[0][3] == got[1][3] == sum(sizes)
    assert shares == shard.assign(sizes, world)
