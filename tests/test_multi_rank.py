"""The multi-GPU path's host side, on CPU.

The database is split into length-balanced shards of whole profiles; each
rank searches its shard with E-values for the whole database, the ranks
exchange their hit lists (an all-gather over a gloo process group here,
NCCL on GPUs) and merge them by log E-value. The merged list must equal one
search of the whole database: the same hits, in the same order, with the
same E-values and alignments. The searches use the oracle so that no GPU is
needed.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from conftest import GOLDEN


def _inputs():
    from cother_b200 import synth
    q = synth.make_profiles([40], 901, True)
    lens = synth.lognormal_lengths(14, 70, 30, 160, seed=902)
    db = synth.make_profiles(lens, 903, False)
    synth.plant_homologs(q, db, 3 / 14, seed=904)
    return q, db


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as O
    from cother_b200.sharding import Hit, gather_hits, merge_hit_lists, shard_ranges
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            init_method=f"tcp://127.0.0.1:{port}", timeout=timedelta(seconds=60))
    try:
        ss = np.load(os.path.join(GOLDEN, "ssss.npy"))
        q, db = _inputs()
        first, count = shard_ranges(db.lens, world)[rank]
        hits = []
        if count:
            found = O.search(q, db.subset(first, count), ss, db.npositions, db.nprofiles,
                             first_profile=first)
            hits = [Hit(profile=p, log_evalue=e, record=np.zeros(18, np.float32), alignment=a)
                    for p, e, a in found]
        merged = merge_hit_lists(gather_hits(hits))
        out.put((rank, [(h.profile, h.log_evalue, h.alignment) for h in merged]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_search_merges_to_whole_database(world, ss_table, oracle_lib):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = dict(out.get(timeout=180) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    q, db = _inputs()
    expected = oracle_lib.search(q, db, ss_table, db.npositions, db.nprofiles)
    assert len(expected) >= 2
    for r in range(world):
        assert got[r] == expected


def test_shard_ranges_balance_and_cover():
    from cother_b200.sharding import shard_ranges
    rng = np.random.default_rng(3)
    lens = rng.integers(30, 1500, 5000)
    for n in (1, 2, 3, 8):
        parts = shard_ranges(lens, n)
        assert parts[0][0] == 0 and sum(c for _, c in parts) == len(lens)
        assert all(parts[k][0] + parts[k][1] == parts[k + 1][0] for k in range(n - 1))
        sizes = [int(lens[f:f + c].sum()) for f, c in parts]
        assert max(sizes) - min(sizes) <= 2 * lens.max()
    few = shard_ranges([5, 7], 4)        # fewer profiles than shards
    assert sum(c for _, c in few) == 2 and all(c >= 0 for _, c in few)


def test_merge_is_stable_by_log_evalue():
    from cother_b200.sharding import Hit, merge_hit_lists
    def h(p, e):
        return Hit(profile=p, log_evalue=e, record=np.zeros(18, np.float32))
    parts = [[h(0, -5.0), h(1, -1.0), h(2, 2.0)], [h(10, -5.0), h(11, 0.5)], [], [h(20, -9.0)]]
    merged = [x.profile for x in merge_hit_lists(parts)]
    assert merged == [20, 0, 10, 1, 11, 2]
