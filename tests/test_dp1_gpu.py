"""Phase-1 DP and finalization on the GPU vs the CPU oracle (bit-identical
backtrack codes, scores with correlation bonus, coordinates, pass list)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _search(q, db, ss, thld, max_slab=0, all_codes=1):
    import cother_b200 as cb
    o = cb.Options.defaults()
    o.all_codes = all_codes
    bp = cb.BatchProcessing(ss, o)
    if max_slab:
        bp.set_max_slab_positions(max_slab)
    bp.set_score_threshold(thld)
    bp.transfer_cpm_data(db)
    bp.process_score_matrix(q)
    return bp


def _compare(bp, oracle_lib, q, db, thld, p0=0, all_codes=True, mixed=True):
    sc, ms, first = bp.read_score_matrix(q.npositions, db.npositions)
    assert first == p0
    rec, plist = bp.read_phase1()
    nprof = len(rec["score"])
    col0 = int(db.starts[p0])
    btck = bp.read_btck(q.npositions, sc.shape[1])
    orec, obt = oracle_lib.dp1(q, db, sc, col0, p0, nprof, thld)
    if all_codes:
        assert np.array_equal(btck, obt)
    else:
        # codes only for the finalization's candidates: DP maximum > threshold
        cand = orec["maxsc"] > np.float32(thld)
        if mixed:
            assert cand.any() and not cand.all()
        for k in np.nonzero(cand)[0]:
            c0 = int(db.starts[p0 + k]) - col0
            L = int(db.lens[p0 + k])
            assert np.array_equal(btck[:, c0:c0 + L], obt[:, c0:c0 + L]), k
    assert np.array_equal(rec["passed"], orec["passed"])
    assert np.array_equal(rec["score"], orec["score"])
    m = orec["passed"] == 1
    assert np.array_equal(rec["psts"][m], orec["psts"][m])
    assert np.array_equal(rec["beg"][m], orec["beg"][m].astype(np.uint32))
    assert np.array_equal(rec["end"][m], orec["end"][m].astype(np.uint32))
    assert np.array_equal(plist, np.nonzero(orec["passed"])[0])
    return rec, plist


def test_dp1_workload_with_homologs(oracle_lib, ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=5, ndb=48, homologs=0.25)
    thld, _ = oracle_lib.score_threshold(q.npositions, 180 * 1000)
    bp = _search(q, db, ss_table, thld)
    rec, plist = _compare(bp, oracle_lib, q, db, thld)
    assert len(plist) >= 8
    bp.close()


def test_dp1_codes_for_candidates_only(oracle_lib, ss_table):
    """The default: a sweep without codes finds each profile's maximum and
    only the profiles above the threshold sweep again with codes; records,
    pass list and the candidates' codes equal the oracle's."""
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=5, ndb=48, homologs=0.25)
    thld, _ = oracle_lib.score_threshold(q.npositions, 180 * 1000)
    bp = _search(q, db, ss_table, thld, all_codes=0)
    rec, plist = _compare(bp, oracle_lib, q, db, thld, all_codes=False)
    assert len(plist) >= 8
    bp.close()
    bp = _search(q, db, ss_table, thld, max_slab=2000, all_codes=0)
    lens, p0, acc = db.lens, 0, 0
    for p, L in enumerate(lens):
        if acc + L > 2000:
            p0, acc = p, 0
        acc += int(L)
    _compare(bp, oracle_lib, q, db, thld, p0=p0, all_codes=False, mixed=False)
    bp.close()


def test_dp1_low_threshold_many_pass(oracle_lib, ss_table):
    """Every profile passes: exercises the backtrace and bonus on random
    (non-homologous) alignments, including corner-triangle cells."""
    from cother_b200 import synth
    q = synth.make_profiles([75], 61, True)
    db = synth.make_profiles([3, 40, 130, 75, 1, 33, 64, 200], 62, False)
    bp = _search(q, db, ss_table, -1.0)
    rec, plist = _compare(bp, oracle_lib, q, db, -1.0)
    assert len(plist) == db.nprofiles
    bp.close()


def test_dp1_multislab_last_slab(oracle_lib, ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=9, ndb=30, homologs=0.3)
    thld = 1.5
    lens = db.lens
    bp = _search(q, db, ss_table, thld, max_slab=600)
    # reproduce the slab planner: greedy runs of whole profiles <= 600 positions
    p0, acc, first = 0, 0, 0
    for p, L in enumerate(lens):
        if acc + L > 600:
            first, acc = p, 0
        acc += int(L)
    rec, plist = _compare(bp, oracle_lib, q, db, thld, p0=first)
    bp.close()


def test_score_threshold_matches_reference_formula(oracle_lib):
    import cother_b200 as cb
    for ql, dbl, ev in [(200, 180000, 10.0), (400, 12_000_000, 1.0), (64, 5000, 0.1), (50, 100, 0.0)]:
        assert cb.score_threshold(ql, dbl, ev) == oracle_lib.score_threshold(ql, dbl, ev)
