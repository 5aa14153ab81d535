"""The on-device hit order (top-k reduction) against the finalizer's host
order: reported records (log E at most the threshold, realigned) sorted by
log E-value with equal values in record order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _host_order(recs, logethld):
    import cother_b200 as cb
    t = cb.records_table(recs)
    alnlen = t["log_evalue_pair"].view(np.int32)
    keep = [i for i in range(len(recs)) if t["log_evalue"][i] <= np.float32(logethld) and alnlen[i] >= 1]
    return sorted(keep, key=lambda i: t["log_evalue"][i])     # stable


def _search(q, db, ss, **kw):
    import cother_b200 as cb
    bp = cb.BatchProcessing(ss)
    if "thld" in kw:
        bp.set_score_threshold(kw["thld"])
    if "logethld" in kw:
        bp.set_logE_threshold(kw["logethld"])
    if kw.get("max_slab"):
        bp.set_max_slab_positions(kw["max_slab"])
    bp.transfer_cpm_data(db)
    bp.process_score_matrix(q)
    return bp


def test_hit_order_homologs(ss_table):
    from cother_b200 import synth
    q, db = synth.make_workload("q200_db1k", seed=41, ndb=300, homologs=0.1)
    bp = _search(q, db, ss_table, max_slab=20000)        # several slabs
    import cother_b200 as cb
    recs = bp.hit_records()
    order = bp.hit_list()
    thld = cb.score_threshold(q.npositions, db.npositions)[1]
    assert order.tolist() == _host_order(recs, thld)
    assert len(order) >= 20
    assert bp.hit_list(top=7).tolist() == order[:7].tolist()
    bp.close()


def test_hit_order_many_records_and_ties(ss_table):
    """More than 4,096 records (the sort crosses shared-memory blocks), and
    many equal log E-values (duplicate profiles), whose order must stay the
    record order."""
    from cother_b200 import synth
    q = synth.make_profiles([40], 4201, True)
    base = synth.make_profiles([12, 20, 33, 8, 25], 4202, False)
    db = base.select(np.tile(np.arange(base.nprofiles), 1100))   # 5,500 profiles, 1,100 copies of each
    bp = _search(q, db, ss_table, thld=-1.0, logethld=1.0e9)
    recs = bp.hit_records()
    assert len(recs) > 4096
    order = bp.hit_list()
    assert order.tolist() == _host_order(recs, 1.0e9)
    bp.close()
