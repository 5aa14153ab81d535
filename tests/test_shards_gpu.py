"""Sharded search on the GPU: the CUDA path run on three database shards
(E-values for the whole database), with the hit lists merged by E-value,
gives exactly the search of the whole database, which in turn equals the
oracle's. The shards run one after another on one GPU; across GPUs each
shard is one rank (bench.py --gpus N), the merge the same."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs():
    from cother_b200 import synth
    q = synth.make_profiles([90], 911, True)
    lens = synth.lognormal_lengths(40, 120, 30, 400, seed=912)
    db = synth.make_profiles(lens, 913, False)
    synth.plant_homologs(q, db, 6 / 40, seed=914)
    return q, db


def _search(ss, q, db, db_len, n_seqs, first):
    import cother_b200 as cb
    from cother_b200.sharding import local_hits
    with cb.BatchProcessing(ss) as bp:
        bp.set_db_details(db_len, n_seqs)
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        return local_hits(bp, first, q.npositions)


def test_shards_merge_to_whole_database(ss_table, oracle_lib):
    from cother_b200.sharding import merge_hit_lists, shard_ranges
    q, db = _inputs()
    N, P = db.npositions, db.nprofiles
    whole = _search(ss_table, q, db, N, P, 0)
    parts = [_search(ss_table, q, db.subset(f, c), N, P, f) for f, c in shard_ranges(db.lens, 3)]
    merged = merge_hit_lists(parts)
    key = lambda hits: [(h.profile, h.log_evalue, h.alignment) for h in hits]
    assert len(whole) >= 3
    assert key(merged) == key(whole)
    for a, b in zip(merged, whole):
        assert np.array_equal(a.record[[0, 3, 8, 16, 17]], b.record[[0, 3, 8, 16, 17]])
    expected = oracle_lib.search(q, db, ss_table, N, P)
    assert [(p, e, a) for p, e, a in expected] == [(h.profile, h.log_evalue, h.alignment) for h in whole]
