"""A search whose database chunks come from a binary database file
(cbp_db_chunk -> cbp_transfer_chunk) gives the same hit records, alignments
and text output as one whose chunks are transferred from the profile set
directly, chunk by chunk."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_search_from_database_file(tmp_path, ss_table):
    import cother_b200 as cb
    from cother_b200 import database, synth
    q, db = synth.make_workload("q200_db1k", seed=23, ndb=30, homologs=0.2)
    descs = ["synthetic profile %d" % p for p in range(db.nprofiles)]
    path = str(tmp_path / "synthetic.tbin")
    database.write_database(path, db, descs)
    with database.Database(path) as dbf:
        chunks = dbf.chunks(3000)
        assert len(chunks) >= 2
        for first, count in chunks:
            sub = db.subset(first, count)
            with cb.BatchProcessing(ss_table) as a, cb.BatchProcessing(ss_table) as b:
                for bp in (a, b):
                    bp.set_db_details(db.npositions, db.nprofiles)
                a.transfer_cpm_data(sub)
                got_descs = b.transfer_db_chunk(dbf, first, count)
                assert got_descs == descs[first:first + count]
                a.process_score_matrix(q)
                b.process_score_matrix(q)
                ra, rb = a.hit_records(), b.hit_records()
                assert ra.tobytes() == rb.tobytes()
                assert np.array_equal(a.alignment_rows(), b.alignment_rows())
                assert a.format_hits(got_descs) == b.format_hits(got_descs)
