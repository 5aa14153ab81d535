"""Statistics and E-values on the GPU vs the CPU oracle: the histogram,
lambda, H, K, estimated gapped parameters and E-values of every passed
pair are bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["lambda_est", "K_est", "log_evalue", "log_evalue_pair", "min", "max", "expected",
          "entropy", "lambda", "K"]


def _run(q, db, ss, thld, ssemodel=2, db_len=None, nseqs=None):
    import cother_b200 as cb
    o = cb.Options.defaults()
    o.ssemodel = ssemodel
    bp = cb.BatchProcessing(ss, o)
    bp.set_score_threshold(thld)
    if db_len:
        bp.set_db_details(db_len, nseqs)
        bp.set_query_len(q.npositions)
    bp.transfer_cpm_data(db)
    bp.process_score_matrix(q)
    return bp


def _check_records(bp, oracle_lib, q, db, ssemodel, expect_min=1):
    import cother_b200 as cb
    # the records as the statistics stage leaves them (one slab here)
    recs = cb.records_table(bp.read_statistics())
    n = len(recs["score"])
    assert n >= expect_min
    sc, _, first = bp.read_score_matrix(q.npositions, db.npositions)
    assert first == 0
    sspace, _ = bp.search_space()
    rec1, plist = bp.read_phase1()
    assert np.array_equal(recs["org_pro_no"], plist.astype(np.uint32))
    lens = db.lens[plist]
    assert np.array_equal(recs["pro_new_dst"], (np.cumsum(lens) - lens).astype(np.uint32))
    nlam = 0
    for k in range(n):
        p = int(recs["org_pro_no"][k])
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        r, _ = oracle_lib.pair_statistics(sc[:, s0:s0 + Ld], q.aa, db.aa[s0:s0 + Ld],
                                          recs["score"][k], recs["psts"][k], q.npositions, Ld,
                                          q.eno[0], db.eno[p], sspace, ssemodel=ssemodel)
        got = np.array([recs[f][k] for f in FIELDS], np.float32)
        assert np.array_equal(got, r.astype(np.float32)), (p, got, r)
        nlam += recs["lambda"][k] > 0
    return n, nlam


def test_stats_homologs_ss18(oracle_lib, ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=5, ndb=48, homologs=0.25)
    thld, _ = oracle_lib.score_threshold(q.npositions, 180 * 1000)
    bp = _run(q, db, ss_table, thld, db_len=180000, nseqs=1000)
    ss, dl = bp.search_space()
    assert (ss, dl) == oracle_lib.length_adjustment(q.npositions, 180000, 1000)
    _check_records(bp, oracle_lib, q, db, 2, expect_min=8)
    bp.close()


@pytest.mark.parametrize("ssemodel", [0, 1, 2])
def test_stats_random_pairs_all_models(oracle_lib, ss_table, ssemodel):
    """A threshold below every score passes random pairs too: their expected
    score is negative, so lambda, H and K are all estimated."""
    from cother_b200 import synth
    q = synth.make_profiles([90], 71, True)
    db = synth.make_profiles([30, 64, 128, 250, 45, 90, 300, 12], 72, False)
    bp = _run(q, db, ss_table, -1.0, ssemodel=ssemodel)
    n, nlam = _check_records(bp, oracle_lib, q, db, ssemodel, expect_min=db.nprofiles)
    assert nlam >= 4
    bp.close()


def test_stats_x_masking(oracle_lib, ss_table):
    """Positions whose residue is X do not enter the score histogram."""
    from cother_b200 import synth
    q = synth.make_profiles([60], 81, True)
    db = synth.make_profiles([70, 40], 82, False)
    q.aa[5:15] = ord("X")
    db.aa[20:30] = ord("X")
    bp = _run(q, db, ss_table, -1.0)
    _check_records(bp, oracle_lib, q, db, 2, expect_min=2)
    bp.close()
