"""The CUDA search path against the reference's own CUDA kernels, end to end.

Runs cother_b200 through its public interface (BatchProcessing over the C
ABI) on the inputs of tests/golden/ref_gpu_<case>.npz, which hold what the
reference's score-matrix, phase-1, statistics and MAP kernels produced for
the same query, database and options on a B200
(tests/golden/make_ref_gpu_fixtures.py). Pass criteria, per pair:

* the same pairs pass phase 1 and the same pairs are realigned;
* phase-1 scores within 1e-4 relative, log E-values within 1e-3 relative;
* the same ranking by E-value;
* identical alignment rows, identity/positive/gap counts and coordinates.

The two paths differ only in the profile-profile term's log (the
reference's __logf intrinsic, a series restatement here), a few ulps per
cell; the modular scores, which do not contain that term, are compared bit
for bit where the fixture holds them (the CVS term included).
"""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
import make_ref_gpu_fixtures as fx  # noqa: E402


@pytest.mark.parametrize("case", sorted(fx.CASES))
def test_search_matches_reference_kernels(case, ss_table):
    import cother_b200 as cb
    F = np.load(os.path.join(GOLDEN, f"ref_gpu_{case}.npz"))
    opts = json.loads(str(F["options"]))
    q, db = fx.case_inputs(opts.get("inputs", "q64"))
    assert str(F["digest"]) == fx.input_digest(q, db)
    o = cb.Options.defaults()
    o.ssswgt, o.ddmswgt, o.dstsegm = opts["ssswgt"], opts["ddmswgt"], opts["dstsegm"]
    o.minpp, o.ssemodel, o.x_uninf = opts["minpp"], opts["ssemodel"], opts["xuninf"]
    o.cvswgt = opts.get("cvswgt", 0.0)
    o.mapaln = 0 if opts.get("nomapaln", 0) else 1
    with cb.BatchProcessing(ss_table, o) as bp:
        if o.cvswgt > 0:
            m = np.load(os.path.join(GOLDEN, "cvs2s.npz"))
            bp.set_cvs2s_map(m["keys"], m["scores"])
        bp.set_db_details(db.npositions, db.nprofiles)
        bp.set_score_threshold(float(F["scorethld"]))
        bp.set_logE_threshold(float(F["logevthld"]))
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        assert bp.search_space()[0] == int(F["searchspace"])
        recs = cb.records_table(bp.hit_records())
        alns = bp.alignments(q.npositions)
        if "modscores" in F:
            # modular scores (SS, CVS and DDMS terms; the CVS term with the
            # same __logf intrinsic) bit for bit
            _, ms, _ = bp.read_score_matrix(q.npositions, db.npositions)
            assert np.array_equal(ms, F["modscores"][:, :db.npositions])

    st, fin, rows = F["stats"], F["final"], F["alns"]
    ref_org = st[:, 1].view(np.uint32).astype(np.int64)
    ours = {int(p): k for k, p in enumerate(recs["org_pro_no"])}
    assert sorted(ours) == sorted(ref_org.tolist())
    Lq = q.npositions
    nrows = 5 if opts["ssswgt"] > 0 else 3
    ref_loge, our_loge = [], []
    for k, p in enumerate(ref_org):
        j = ours[int(p)]
        assert abs(recs["score"][j] - st[k, 0]) <= 1e-4 * abs(st[k, 0]), p
        assert abs(recs["log_evalue"][j] - st[k, 8]) <= 1e-3 * abs(st[k, 8]) + 1e-6, p
        ref_loge.append(st[k, 8])
        our_loge.append(recs["log_evalue"][j])
        alnlen = int(fin[k, 9].view(np.int32))
        if alnlen == 0:
            assert alns[j] is None, p
            continue
        assert alns[j] is not None, p
        Ld = int(db.lens[p])
        end = int(fin[k, 2].view(np.uint32)) + k * Lq + Ld + Lq - 1
        ref_rows = tuple(bytes(rows[r, end - alnlen:end]).decode() for r in range(nrows))
        assert alns[j][:nrows] == ref_rows, p
        assert (recs["identities"][j], recs["gaps"][j], recs["psts"][j]) == \
            (fin[k, 16], fin[k, 17], fin[k, 3]), p
        assert (recs["beg_coords"][j], recs["end_coords"][j]) == \
            (fin[k, 4].view(np.uint32), fin[k, 5].view(np.uint32)), p
    order_ref = ref_org[np.argsort(np.asarray(ref_loge), kind="stable")]
    order_our = ref_org[np.argsort(np.asarray(our_loge), kind="stable")]
    assert np.array_equal(order_ref, order_our)
