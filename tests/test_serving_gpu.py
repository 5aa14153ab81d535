"""The request loop on the GPU (the C++ server): queries of different
lengths submitted together are searched in batches (several queries in one
pass over the resident database) through concurrent slots, under a memory
budget small enough that the longer batches are cut into several slabs; each
query's hits, E-values, alignments and records equal its results searched
alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("max_batch", [1, 3])
def test_results_same_alone_and_in_the_mix(ss_table, max_batch):
    import cother_b200 as cb
    from cother_b200 import synth
    from cother_b200.serving import SearchServer, footprint, latency_summary
    from cother_b200.sharding import local_hits
    qlens = [60, 150, 90, 200, 45, 120, 75, 33]
    qs = [synth.make_profiles([L], 921 + k, True) for k, L in enumerate(qlens)]
    lens = synth.lognormal_lengths(60, 150, 30, 400, seed=930)
    db = synth.make_profiles(lens, 931, False)
    for k, q in enumerate(qs[:3]):
        synth.plant_homologs(q, db, 3 / 60, seed=940 + k)
    N, P = db.npositions, db.nprofiles

    alone = []
    for q in qs:
        with cb.BatchProcessing(ss_table) as bp:
            bp.set_db_details(N, P)
            bp.transfer_cpm_data(db)
            bp.process_score_matrix(q)
            alone.append((local_hits(bp, 0, q.npositions), bp.hit_records()))

    budget = footprint(200, N) // 2 + footprint(60, N)     # long batches need 2+ slabs
    with SearchServer(db, ss_table, slots=3, max_batch=max_batch, budget=budget, max_share=0.5) as srv:
        assert srv.budget == budget
        futs = [srv.submit(q) for q in qs]
        mixed = [f.result(timeout=300) for f in futs]
    for (hits, recs), m in zip(alone, mixed):
        key = lambda hs: [(h.profile, h.log_evalue, h.alignment) for h in hs]
        assert key(m["hits"]) == key(hits)
        assert np.array_equal(m["records"], recs)
    assert any(len(h) > 0 for h, _ in alone)
    assert any(m["slab"] < N for m in mixed)                                 # cut into slabs
    assert max(m["batch"] for m in mixed) <= max_batch
    if max_batch > 1:
        assert any(m["batch"] > 1 for m in mixed)                            # batched
    assert any(m["finish"] > n["start"] and m["start"] < n["finish"] and m["slot"] != n["slot"]
               for i, m in enumerate(mixed) for n in mixed[i + 1:])        # slots overlapped
    s = latency_summary(mixed)
    assert s["queries"] == len(qs)
