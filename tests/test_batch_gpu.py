"""Several queries in one pass over the database (cbp_process_batch): each
query's results equal its results searched alone -- hit records, alignment
rows and the hit order bit for bit -- with one or several slabs, the plain
and the tensor-core forms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _workload():
    from cother_b200 import synth
    qs = [synth.make_profiles([L], 5100 + i, True) for i, L in enumerate((70, 150, 33, 96))]
    db = synth.make_profiles(synth.lognormal_lengths(60, 120, 30, 300, seed=5200), 5201, False)
    for i, q in enumerate(qs):
        synth.plant_homologs(q, db, 0.08, seed=5300 + i)
    return qs, db


def _results(bp, Lq):
    return bp.hit_records(), bp.alignment_rows(), bp.hit_list(), bp.search_space()


def _search_alone(q, db, ss, opts, max_slab):
    import cother_b200 as cb
    with cb.BatchProcessing(ss, opts) as bp:
        bp.set_db_details(db.npositions * 50, db.nprofiles * 50)
        if max_slab:
            bp.set_max_slab_positions(max_slab)
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        out = _results(bp, q.npositions)
        sc, _, _ = bp.read_score_matrix(q.npositions, db.npositions)
    return out, sc


@pytest.mark.parametrize("form,max_slab", [("plain", 0), ("plain", 5000), ("bf16", 0)])
def test_batch_equals_alone(ss_table, form, max_slab):
    import cother_b200 as cb
    qs, db = _workload()
    opts = cb.Options.defaults()
    opts.tc_form = {"plain": cb.TC_PLAIN, "bf16": cb.TC_BF16X3}[form]
    alone = [_search_alone(q, db, ss_table, opts, max_slab) for q in qs]
    with cb.BatchProcessing(ss_table, opts) as bp:
        bp.set_db_details(db.npositions * 50, db.nprofiles * 50)
        if max_slab:
            bp.set_max_slab_positions(max_slab)
        bp.transfer_cpm_data(db)
        bp.process_batch(qs)
        # the inspection calls see the last query
        sc_last, _, _ = bp.read_score_matrix(qs[-1].npositions, db.npositions)
        if not max_slab:
            assert np.array_equal(sc_last, alone[-1][1])
        nhits = 0
        for k, q in enumerate(qs):
            assert bp.select_query(k) == len(qs)
            recs, rows, order, space = _results(bp, q.npositions)
            arecs, arows, aorder, aspace = alone[k][0]
            assert space == aspace, k
            assert np.array_equal(recs.view(np.uint32), arecs.view(np.uint32)), k
            assert np.array_equal(rows, arows), k
            assert np.array_equal(order, aorder), k
            nhits += len(order)
        assert nhits >= 8
        with pytest.raises(cb.CbpError):
            bp.select_query(len(qs))
