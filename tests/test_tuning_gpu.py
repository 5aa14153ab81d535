"""The kernel tuner: every candidate variant (score-kernel rows per block,
column-ordering window, phase-1 DP warps per block) gives bit-identical
score matrices, phase-1 results and hit records, and the tuner's choice is
one of them with a positive sample time for each candidate."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = [(16, 1024, 2), (8, 1024, 2), (32, 1024, 2), (16, 256, 2), (16, 4096, 2), (16, 1024, 1),
            (32, 32, 1)]


def _run(q, db, ss, variant=None, autotune=1):
    import cother_b200 as cb
    o = cb.Options.defaults()
    o.autotune = autotune
    o.all_codes = 1     # compare the whole backtrack matrix
    with cb.BatchProcessing(ss, o) as bp:
        if variant is not None:
            bp.set_kernels(q.npositions, *variant)
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        sc, ms, _ = bp.read_score_matrix(q.npositions, db.npositions)
        bt = bp.read_btck(q.npositions, db.npositions)
        assert bp.graph_launches() >= 1   # the plain form runs phase 1 as a CUDA graph
        bp.process_score_matrix(q)        # a second query updates the same graph
        assert bp.graph_launches() >= 2
        return sc, ms, bt, bp.hit_records(), bp.alignment_rows(), bp.tuning(q.npositions)


def test_variants_are_bit_identical(ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=31, ndb=60, homologs=0.1)
    ref = _run(q, db, ss_table, autotune=0)
    assert ref[5]["score_rows"] == 16 and ref[5]["order_window"] == 1024 and ref[5]["dp_warps"] == 2
    for v in VARIANTS:
        got = _run(q, db, ss_table, variant=v)
        assert got[5]["score_rows"] == v[0] and got[5]["order_window"] == v[1] and got[5]["dp_warps"] == v[2]
        for a, b in zip(ref[:5], got[:5]):
            assert np.array_equal(a, b), v


def test_tuner_choice(ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=32, ndb=40)
    ref = _run(q, db, ss_table, autotune=0)
    got = _run(q, db, ss_table, autotune=1)
    t = got[5]
    assert (t["score_rows"], t["order_window"]) in {(r, w) for r, w, _ in VARIANTS[:5]}
    assert t["dp_warps"] in (1, 2)
    assert all(x > 0 for x in t["score_candidates_ms"]) and all(x > 0 for x in t["dp_candidates_ms"])
    for a, b in zip(ref[:5], got[:5]):
        assert np.array_equal(a, b)
