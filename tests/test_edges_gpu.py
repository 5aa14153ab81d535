"""Edge shapes of the search path on the GPU against the CPU oracle: queries
of one to three positions, profiles of one and two positions, a database of
one profile, and positions whose distance lists are empty or shorter than
DSTSEGM (the DDMS term is then skipped for the cell). Every stage is
compared exactly: score and modular-score cells, phase-1 records and
backtrack codes, statistics, and the MAP alignments of the pairs that pass
(a threshold low enough that pairs pass)."""
import numpy as np
import pytest

from test_dp1_gpu import _compare
from test_map_gpu import _check_map, _search

pytestmark = pytest.mark.gpu


def _check(oracle_lib, ss, q, db):
    bp = _search(q, db, ss, thld=-1.0, logethld=1e9, minpp=0.05, all_codes=1)
    try:
        sc, ms, first = bp.read_score_matrix(q.npositions, db.npositions)
        assert first == 0
        osc, oms = oracle_lib.score_matrix(q, db, ss, nthreads=4)
        assert np.array_equal(sc, osc) and np.array_equal(ms, oms)
        rec, plist = _compare(bp, oracle_lib, q, db, -1.0, all_codes=True)
        nreal = _check_map(bp, oracle_lib, q, db, minpp=0.05, logethld=1e9)
        return len(plist), nreal
    finally:
        bp.close()


@pytest.mark.parametrize("Lq", [1, 2, 3])
def test_tiny_queries_and_profiles(oracle_lib, ss_table, Lq):
    from cother_b200 import synth
    q = synth.make_profiles([Lq], 700 + Lq, True)
    db = synth.make_profiles([1, 2, 5, 40, 3], 710 + Lq, False)
    npass, _ = _check(oracle_lib, ss_table, q, db)
    assert npass >= 1


def test_single_profile_database(oracle_lib, ss_table):
    from cother_b200 import synth
    q = synth.make_profiles([70], 721, True)
    db = synth.make_profiles([90], 722, False)
    synth.plant_homologs(q, db, 1.0, seed=723)
    npass, nreal = _check(oracle_lib, ss_table, q, db)
    assert npass == 1 and nreal == 1


def test_empty_and_short_distance_lists(oracle_lib, ss_table):
    """Positions with no distances (count 0) and with fewer than DSTSEGM,
    in the query and in the database, beside full lists."""
    from cother_b200 import synth
    q = synth.make_profiles([60], 731, True)
    db = synth.make_profiles([50, 45, 64], 732, False)
    synth.plant_homologs(q, db, 0.7, seed=733)
    for ps, rows in ((q, range(0, 60, 4)), (db, range(0, db.npositions, 5))):
        for i, r in enumerate(rows):
            n = 0 if i % 2 == 0 else 1 + (i % 5)       # empty, or 1..5 (< DSTSEGM = 6)
            ps.dd[0, r] = float(n)
            ps.dd[1 + n:, r] = 0.0
    assert np.any(q.dd[0] == 0) and np.any((db.dd[0] > 0) & (db.dd[0] < 6))
    npass, _ = _check(oracle_lib, ss_table, q, db)
    assert npass >= 1
