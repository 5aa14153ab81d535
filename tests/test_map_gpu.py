"""Phase-2 MAP realignment on the GPU vs the CPU oracle: identical
alignment strings, identities, positives, gaps and coordinates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _search(q, db, ss, thld=None, logethld=None, max_slab=0, **opt):
    import cother_b200 as cb
    o = cb.Options.defaults()
    for k, v in opt.items():
        setattr(o, k, v)
    bp = cb.BatchProcessing(ss, o)
    if thld is not None:
        bp.set_score_threshold(thld)
    if logethld is not None:
        bp.set_logE_threshold(logethld)
    if max_slab:
        bp.set_max_slab_positions(max_slab)
    bp.transfer_cpm_data(db)
    bp.process_score_matrix(q)
    return bp


def _check_map(bp, oracle_lib, q, db, minpp=0.28, logethld=2.302585):
    import cother_b200 as cb
    recs = cb.records_table(bp.hit_records())
    alns = bp.alignments(q.npositions)
    sc, ms, first = bp.read_score_matrix(q.npositions, db.npositions)
    assert first == 0
    sspace, _ = bp.search_space()
    ph1, _ = bp.read_phase1()
    nrealigned = 0
    for k in range(len(recs["score"])):
        p = int(recs["org_pro_no"][k])
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        st, _ = oracle_lib.pair_statistics(sc[:, s0:s0 + Ld], q.aa, db.aa[s0:s0 + Ld],
                                           recs["score"][k], ph1["psts"][p], q.npositions, Ld, q.eno[0],
                                           db.eno[p], sspace)
        logE, epa = st[2], st[3]
        assert np.float32(logE) == recs["log_evalue"][k]
        if logethld < logE:
            assert alns[k] is None
            continue
        m = oracle_lib.map_pair(q, db, p, sc[:, s0:s0 + Ld], ms[:, s0:s0 + Ld], epa, minpp=minpp)
        if m["alnlen"] == 0:
            assert alns[k] is None
            continue
        nrealigned += 1
        assert alns[k] == tuple(m["aln"]), (p, alns[k][0][:40], m["aln"][0][:40])
        assert recs["identities"][k] == m["idts"]
        assert recs["psts"][k] == m["psts"]
        assert recs["gaps"][k] == m["gaps"]
        assert recs["beg_coords"][k] == m["beg"]
        assert recs["end_coords"][k] == m["end"]
    return nrealigned


def test_map_homologs(oracle_lib, ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=5, ndb=48, homologs=0.25)
    bp = _search(q, db, ss_table)
    n = _check_map(bp, oracle_lib, q, db)
    assert n >= 8
    bp.close()


def test_map_weak_pairs_and_minpp(oracle_lib, ss_table):
    """A permissive threshold realigns random pairs too (short, gappy MAP
    alignments, corner cells, logZ near zero); MINPP changes the DP."""
    from cother_b200 import synth
    q = synth.make_profiles([70], 91, True)
    db = synth.make_profiles([40, 90, 33, 150, 64], 92, False)
    for minpp in (0.28, 0.05):
        bp = _search(q, db, ss_table, thld=-1.0, logethld=1e9, minpp=minpp)
        _check_map(bp, oracle_lib, q, db, minpp=minpp, logethld=1e9)
        bp.close()


@pytest.mark.parametrize("Lq", [9, 32, 45, 300, 530])
def test_map_query_lengths(oracle_lib, ss_table, Lq):
    """Query lengths that give one band (one warp per pair), a last band of
    a few rows, and more bands than warps (each warp takes several bands);
    profiles from 1 to 200 positions, shorter and longer than 32 and than
    the query."""
    from cother_b200 import synth
    q = synth.make_profiles([Lq], 300 + Lq, True)
    db = synth.make_profiles([1, 7, 31, 32, 33, 64, 65, 150, 200, 96], 301 + Lq, False)
    synth.plant_homologs(q, db, 0.8, seed=302 + Lq)
    bp = _search(q, db, ss_table, thld=-1.0, logethld=1e9, minpp=0.05)
    n = _check_map(bp, oracle_lib, q, db, minpp=0.05, logethld=1e9)
    assert n >= 2
    bp.close()


def test_map_multislab_offsets(oracle_lib, ss_table):
    """Records and alignment rows of several slabs join into one result:
    phase-2 offsets continue across slabs."""
    import cother_b200 as cb
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=8, ndb=36, homologs=0.3)
    one = _search(q, db, ss_table)
    many = _search(q, db, ss_table, max_slab=900)
    r1, r2 = cb.records_table(one.hit_records()), cb.records_table(many.hit_records())
    for f in ("score", "org_pro_no", "pro_new_dst", "log_evalue", "identities", "gaps"):
        assert np.array_equal(r1[f], r2[f]), f
    assert one.alignments(q.npositions) == many.alignments(q.npositions)
    one.close()
    many.close()


def test_mapaln0_reports_phase1_alignments(oracle_lib, ss_table):
    """MAPALN=0: the pairs within the E-value threshold get their phase-1
    alignment (from the phase-1 maximum over the phase-1 backtrack codes),
    in the same rows and record fields as the MAP path."""
    import cother_b200 as cb
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=6, ndb=40, homologs=0.25)
    bp = _search(q, db, ss_table, mapaln=0)
    recs = cb.records_table(bp.hit_records())
    alns = bp.alignments(q.npositions)
    sc, _, _ = bp.read_score_matrix(q.npositions, db.npositions)
    rec1, bt1 = oracle_lib.dp1(q, db, sc, 0, 0, db.nprofiles, -1.0e30)
    n = 0
    for k in range(len(recs["score"])):
        p = int(recs["org_pro_no"][k])
        if alns[k] is None:
            continue
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        o = oracle_lib.aln_pair(q, db, p, sc[:, s0:s0 + Ld], bt1[:, s0:s0 + Ld], rec1["maxsc"][p],
                                rec1["maxr"][p], rec1["maxc"][p])
        assert alns[k] == tuple(o["aln"]), p
        assert (recs["identities"][k], recs["psts"][k], recs["gaps"][k]) == \
            (o["idts"], o["psts"], o["gaps"]), p
        assert (recs["beg_coords"][k], recs["end_coords"][k]) == (o["beg"], o["end"]), p
        n += 1
    assert n >= 8
    bp.close()
