"""Database sharding across GPUs and the merge of their hit lists.

The search path shards by database profile: every profile is scored,
aligned and given its E-value independently of the others, and the E-values
use the size of the whole database (set on every shard with
``BatchProcessing.set_db_details``), so one query's results on the shards
are exactly the whole database's results, split. The only exchange is the
merge of the per-shard hit lists, which the reference does on the host when
it joins the parts of one query's results (``AlnWriter::MergeResults``,
src/libmycu/cualn/AlnWriter.cpp:211-256): a stable merge by log E-value, the
parts taken in order, each part already sorted by its finalizer
(src/libmycu/cupro/CuBatchProcessingFinalizer.cpp:283-292).

Shards are contiguous runs of whole profiles with about the same number of
positions (the work of the score matrix and the DPs grows with positions).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def shard_ranges(lens, nshards: int):
    """Split profiles 0..P-1 into `nshards` contiguous runs with about
    equal total length. Returns [(first, count), ...]; runs may be empty
    when there are fewer profiles than shards."""
    lens = np.asarray(lens, dtype=np.int64)
    P = len(lens)
    if nshards < 1:
        raise ValueError("nshards must be >= 1")
    cum = np.concatenate([[0], np.cumsum(lens)])
    total = int(cum[-1])
    cuts = [0]
    for k in range(1, nshards):
        target = total * k / nshards
        j = int(np.searchsorted(cum, target, side="left"))
        j = min(max(j, cuts[-1]), P)
        cuts.append(j)
    cuts.append(P)
    return [(cuts[k], cuts[k + 1] - cuts[k]) for k in range(nshards)]


@dataclass
class Hit:
    """One reported hit: the profile's index in the whole database, its
    record (CBP_REC_FLOATS floats) and its alignment rows."""
    profile: int
    log_evalue: float
    record: np.ndarray
    alignment: tuple = field(default_factory=tuple)


def local_hits(bp, first_profile: int, query_len: int):
    """The reported hits of a shard's last search (BatchProcessing `bp`),
    in its finalizer's order, with profile indices of the whole database."""
    import cother_b200 as cb
    recs = bp.hit_records()
    order = bp.hit_list()
    alns = bp.alignments(query_len)
    tab = cb.records_table(recs)
    out = []
    for i in order:
        out.append(Hit(profile=int(tab["org_pro_no"][i]) + first_profile,
                       log_evalue=float(recs[i, 8]), record=recs[i].copy(),
                       alignment=alns[i]))
    return out


def merge_hit_lists(parts):
    """Stable merge of per-shard hit lists (each sorted by log E-value),
    shards in order: equal log E-values keep the shard order, then the
    order within the shard. The merge runs in the library's C++
    (cbp_merge_hit_lists, the writer's join of a query's parts)."""
    from .report import merge_hit_lists as merge_keys
    keys = [np.array([h.log_evalue for h in part], np.float32) for part in parts]
    return [parts[k][i] for k, i in merge_keys(keys)]


def gather_hits(hits, group=None):
    """All ranks' hit lists, in rank order, on every rank (one all-gather of
    small host objects over the process group)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, hits, group=group)
    return parts
