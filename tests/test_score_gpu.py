"""Score matrix on the GPU vs the CPU oracle: bit-identical cells."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(q, db, ss_table, max_slab=0, **opt):
    import cother_b200 as cb
    o = cb.Options.defaults()
    for k, v in opt.items():
        setattr(o, k, v)
    with cb.BatchProcessing(ss_table, o) as bp:
        if o.cvswgt > 0:
            from oracle import oracle as O
            m = O.load_cvs_map()
            bp.set_cvs2s_map(m["keys"], m["scores"])
        if max_slab:
            bp.set_max_slab_positions(max_slab)
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        sc, ms, first = bp.read_score_matrix(q.npositions, db.npositions)
    return sc, ms, first


def test_score_matrix_bit_exact_small(oracle_lib, ss_table):
    from cother_b200 import synth
    q = synth.make_profiles([37], 21, True)
    db = synth.make_profiles([45, 3, 120, 64, 31], 22, False)
    sc, ms, first = _run(q, db, ss_table)
    assert first == 0
    osc, oms = oracle_lib.score_matrix(q, db, ss_table, nthreads=8)
    assert sc.shape == osc.shape
    assert np.array_equal(sc, osc), np.abs(sc - osc).max()
    assert np.array_equal(ms, oms), np.abs(ms - oms).max()


def test_score_matrix_bit_exact_workload(oracle_lib, ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=3, ndb=60)
    sc, ms, _ = _run(q, db, ss_table)
    osc, oms = oracle_lib.score_matrix(q, db, ss_table, nthreads=16)
    assert np.array_equal(sc, osc)
    assert np.array_equal(ms, oms)


def test_score_matrix_last_slab(oracle_lib, ss_table):
    """Multi-slab processing: the last slab holds the trailing profiles."""
    from cother_b200 import synth
    q = synth.make_profiles([50], 31, True)
    lens = [70, 20, 90, 33, 64, 12]
    db = synth.make_profiles(lens, 32, False)
    sc, ms, first = _run(q, db, ss_table, max_slab=100)
    # slabs of <=100 positions: [70,20] [90] [33,64] [12]
    assert first == 5
    col0 = sum(lens[:5])
    osc, oms = oracle_lib.score_matrix(q, db, ss_table, col0=col0, ncols=12)
    assert np.array_equal(sc, osc) and np.array_equal(ms, oms)


def test_score_matrix_options(oracle_lib, ss_table):
    """DDMS off, SS off, other weights, DSTSEGM below 5 and above 6 (the kernel's
    general and long-segment cases beside its default of 6) and MAPALN=0 shift."""
    from cother_b200 import synth
    q = synth.make_profiles([21], 41, True)
    db = synth.make_profiles([33, 18], 42, False)
    for opt, orc in [
        (dict(ddmswgt=0.0), dict(ddmswgt=0.0)),
        (dict(ssswgt=0.0), dict(ssswgt=0.0)),
        (dict(ssswgt=0.3, ddmswgt=0.5, dstsegm=3), dict(ssswgt=0.3, ddmswgt=0.5, dstsegm=3)),
        (dict(dstsegm=8), dict(dstsegm=8)),
        (dict(mapaln=0), dict(initshift=0.0003)),
    ]:
        sc, ms, _ = _run(q, db, ss_table, **opt)
        osc, oms = oracle_lib.score_matrix(q, db, ss_table, **orc)
        assert np.array_equal(sc, osc), opt
        assert np.array_equal(ms, oms), opt


@pytest.mark.parametrize("ssswgt", [0.12, 0.0])
def test_score_matrix_context_vectors(oracle_lib, ss_table, ssswgt):
    """The CVS term (CVSWGT 0.15, with and without SS) against the oracle:
    bit for bit except where the oracle flags the map lookup as within the
    error bound of the __logf intrinsic of a map edge; those cells differ by
    at most one map step."""
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=4, ndb=40, context_vectors=True)
    sc, ms, _ = _run(q, db, ss_table, ssswgt=ssswgt, cvswgt=0.15)
    osc, oms, amb = oracle_lib.score_matrix(q, db, ss_table, ssswgt=ssswgt, cvswgt=0.15,
                                            ambiguous=True, nthreads=16)
    amb = amb.astype(bool)
    step = float(np.max(np.abs(np.diff(oracle_lib.load_cvs_map()["scores"])))) * 0.15 + 1e-6
    assert amb.mean() < 1e-3
    assert np.array_equal(sc[~amb], osc[~amb]) and np.array_equal(ms[~amb], oms[~amb])
    assert np.all(np.abs(sc - osc)[amb] <= step) and np.all(np.abs(ms - oms)[amb] <= step)
    # the term is there: it moves the scores
    plain = oracle_lib.score_matrix(q, db, ss_table, ssswgt=ssswgt, nthreads=16)[0]
    assert np.abs(osc - plain).mean() > 1e-3


def test_context_vectors_need_map_and_fields(ss_table):
    import cother_b200 as cb
    from cother_b200 import synth
    q = synth.make_profiles([20], 51, True)
    db = synth.make_profiles([30, 40], 52, False)
    o = cb.Options.defaults()
    o.cvswgt = 0.15
    with cb.BatchProcessing(ss_table, o) as bp:
        bp.transfer_cpm_data(synth.add_context_vectors(db, 53))
        with pytest.raises(cb.CbpError, match="context-vector map"):
            bp.process_score_matrix(synth.add_context_vectors(q, 54))


def test_bad_inputs_fail_loudly(ss_table):
    import cother_b200 as cb
    from cother_b200 import synth
    q = synth.make_profiles([10], 5, True)
    with cb.BatchProcessing(ss_table) as bp:
        with pytest.raises(cb.CbpError):
            bp.process_score_matrix(q)  # no database chunk yet
        db = synth.make_profiles([12], 6, False)
        db.dd[0, 3] = 150.0  # distance count beyond 99
        with pytest.raises(cb.CbpError):
            bp.transfer_cpm_data(db)


def test_capacities_report_a_chunk_that_fits(ss_table):
    """The chunk capacities (the reference's GetCurrentMaxDbPos and the like):
    positive with a generous budget, positions = profiles x the expected
    length, phase-2 limits equal to the chunk's, zero when the working budget
    cannot hold one slab, and unchanged by the context's own resident chunk."""
    import cother_b200 as cb
    from cother_b200 import synth
    with cb.BatchProcessing(ss_table, dev_mem_bytes=1 << 30) as bp:
        c = bp.capacities(400, 250)
        assert c["max_db_pros"] > 1000 and c["max_db_pos"] == 250 * c["max_db_pros"]
        assert c["max_pass2_pos"] == c["max_db_pos"] and c["max_pass2_pros"] == c["max_db_pros"]
        assert bp.capacities(400, 500)["max_db_pros"] < c["max_db_pros"]
        bp.transfer_cpm_data(synth.make_profiles([300] * 20, 61, False))
        c2 = bp.capacities(400, 250)
        assert abs(c2["max_db_pros"] - c["max_db_pros"]) <= 0.01 * c["max_db_pros"]
    with cb.BatchProcessing(ss_table, dev_mem_bytes=1 << 16) as bp:
        assert bp.capacities(400, 250)["max_db_pos"] == 0
