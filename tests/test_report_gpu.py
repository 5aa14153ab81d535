"""Text output of a search run on the GPU (cbp_format_hits on the context)
equals the same formatting of the context's records and alignment rows
from host data (cbp_format_hits_host) and the oracle's restatement of the
reference's formatters, in both formats; the report parses as JSON."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_context_text_output(ss_table):
    import cother_b200 as cb
    from cother_b200 import report as rep
    from cother_b200 import synth
    from oracle import report as R
    q, db = synth.make_workload("q200_db1k", seed=15, ndb=40, homologs=0.2)
    descs = ["profile_%d synthetic \"homolog\" test/%d" % (p, p % 7) for p in range(db.nprofiles)]
    with cb.BatchProcessing(ss_table) as bp:
        bp.transfer_cpm_data(db)
        bp.process_score_matrix(q)
        recs = bp.hit_records()
        rows = bp.alignment_rows()
        sspace, delta = bp.search_space()
        logethld = cb.score_threshold(q.npositions, db.npositions)[1]
        nrep = len(bp.hit_list())
        assert nrep >= 3
        for fmt in (rep.PLAIN, rep.JSON):
            fo = rep.FormatOptions.defaults(fmt)
            got = bp.format_hits(descs, fo)
            assert len(got) == nrep
            host = rep.format_hits_host(recs, rows, db.lens, np.asarray(db.eno).reshape(-1), q.npositions,
                                        float(q.eno[0]), logethld, float(sspace), ssswgt=0.12, descs=descs,
                                        options=fo)
            assert got == host
            want = R.format_hits(recs, rows, db.lens, np.asarray(db.eno).reshape(-1), descs, q.npositions,
                                 float(q.eno[0]), logethld, float(sspace), ssswgt=0.12, fmt=fmt)
            assert got == want
            text = rep.write_report(got, q.npositions, db.npositions, db.nprofiles, logethld, float(sspace),
                                    int(delta), query_desc="synthetic query", db_names=["synthetic_db"],
                                    options=fo)
            if fmt == rep.JSON:
                doc = json.loads(text)["cother_search"]
                assert len(doc["search_hits"]) == nrep
            else:
                assert text.count("\nQuery: ") >= nrep
