"""Parity at the shapes of the benchmark configurations.

The other GPU tests use toy shapes (at most a few dozen profiles of a few
hundred positions). These run the CUDA path at the benchmark workloads'
shapes and compare it with the CPU oracle stage by stage:

* q1500 x long profiles (the long-query stress configuration: query 1,500
  positions, DDMS window 128, profiles of 500-1,500 positions, planted
  homologs so that several ~1,500 x 1,500 pairs are realigned through many
  MAP bands);
* q400 x the full 50,000-profile database (the batched configuration,
  12.4 M positions, one slab): the whole database is searched on the GPU
  and a sample of its profiles -- every planted homolog plus profiles drawn
  across the database -- is checked against the oracle;
* the query-length sweep 64 / 256 / 1,024 of the precision configuration
  against a sample-sized database of the same length law.

Every comparison is exact: score and modular-score cells, backtrack codes
(of the profiles the finalization backtraces), phase-1 records, statistics
records, alignment rows, counts and coordinates, and the order of the
reported hits (by log E-value, ties in database order) restricted to the
sample.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STAT_FIELDS = ["lambda_est", "K_est", "log_evalue", "log_evalue_pair", "min", "max", "expected",
               "entropy", "lambda", "K"]


def _ncpu():
    return max(1, min(os.cpu_count() or 1, 64))


def _search(q, db, ss, db_len, n_seqs):
    import cother_b200 as cb
    bp = cb.BatchProcessing(ss)
    bp.set_db_details(db_len, n_seqs)
    bp.set_query_len(q.npositions)
    bp.transfer_cpm_data(db)
    bp.process_score_matrix(q)
    return bp


def _check_sample(bp, O, q, db, ss, sample, db_len, n_seqs):
    """Compare the CUDA search (one slab holding the whole database) with
    the oracle on the profiles `sample`; returns (#passed, #realigned)."""
    import cother_b200 as cb
    Lq = q.npositions
    sample = np.sort(np.asarray(sample, np.int64))
    rec1, plist = bp.read_phase1()
    assert len(rec1["score"]) == db.nprofiles          # one slab
    starts = db.starts
    # --- score matrix and phase-1 backtrack codes of the sampled columns
    parts = [bp.read_slab_columns(Lq, int(starts[p]), int(db.lens[p])) for p in sample]
    gsc = np.concatenate([x[0] for x in parts], axis=1)
    gms = np.concatenate([x[1] for x in parts], axis=1)
    gbt = np.concatenate([x[2] for x in parts], axis=1)
    sub = db.select(sample)
    osc, oms = O.score_matrix(q, sub, ss, nthreads=_ncpu())
    bad = np.argwhere(gsc != osc)
    assert len(bad) == 0, ("scores", len(bad), bad[:5])
    assert np.array_equal(gms, oms), "modular scores"
    # --- phase 1
    thld, lthld = O.score_threshold(Lq, db_len)
    orec, obt = O.dp1(q, sub, osc, 0, 0, sub.nprofiles, thld)
    # the search writes backtrack codes for the finalization's candidates
    # only (DP maximum above the threshold): compare those profiles' codes
    cand = orec["maxsc"] > np.float32(thld)
    assert np.all(cand[orec["passed"] == 1])
    for i in np.nonzero(cand)[0]:
        s0, Ld = int(sub.starts[i]), int(sub.lens[i])
        assert np.array_equal(gbt[:, s0:s0 + Ld], obt[:, s0:s0 + Ld]), ("backtrack codes", int(sample[i]))
    assert np.array_equal(rec1["passed"][sample], orec["passed"])
    assert np.array_equal(rec1["score"][sample], orec["score"])
    m = orec["passed"] == 1
    assert np.array_equal(rec1["psts"][sample][m], orec["psts"][m])
    assert np.array_equal(rec1["beg"][sample][m], orec["beg"][m].astype(np.uint32))
    assert np.array_equal(rec1["end"][sample][m], orec["end"][m].astype(np.uint32))
    # --- statistics and E-values of the sampled passed pairs
    sspace, _ = bp.search_space()
    assert (sspace, bp.search_space()[1]) == O.length_adjustment(Lq, db_len, n_seqs)
    srecs = cb.records_table(bp.read_statistics())
    assert np.array_equal(srecs["org_pro_no"], plist.astype(np.uint32))
    where = {int(p): k for k, p in enumerate(srecs["org_pro_no"])}
    local = {int(p): i for i, p in enumerate(sample)}
    npassed = 0
    logE = {}
    for i, p in enumerate(sample):
        if not orec["passed"][i]:
            assert int(p) not in where
            continue
        npassed += 1
        k = where[int(p)]
        s0, Ld = int(sub.starts[i]), int(sub.lens[i])
        st, _ = O.pair_statistics(osc[:, s0:s0 + Ld], q.aa, sub.aa[s0:s0 + Ld], orec["score"][i],
                                  orec["psts"][i], Lq, Ld, q.eno[0], sub.eno[i], sspace)
        got = np.array([srecs[f][k] for f in STAT_FIELDS], np.float32)
        assert np.array_equal(got, st.astype(np.float32)), (int(p), got, st)
        logE[int(p)] = (float(np.float32(st[2])), st[3])
    # --- MAP realignment of the sampled pairs within the E-value threshold
    hrecs = cb.records_table(bp.hit_records())
    alns = bp.alignments(Lq)
    assert np.array_equal(hrecs["org_pro_no"], plist.astype(np.uint32))
    nreal = 0
    oracle_hits = []
    for p, (le, epa) in logE.items():
        k = where[p]
        assert hrecs["log_evalue"][k] == np.float32(le)
        if le > lthld:
            assert alns[k] is None, p
            continue
        i = local[p]
        s0, Ld = int(sub.starts[i]), int(sub.lens[i])
        mo = O.map_pair(q, sub, i, osc[:, s0:s0 + Ld], oms[:, s0:s0 + Ld], epa)
        if mo["alnlen"] == 0:
            assert alns[k] is None, p
            continue
        nreal += 1
        assert alns[k] == tuple(mo["aln"]), p
        assert (hrecs["identities"][k], hrecs["psts"][k], hrecs["gaps"][k]) == \
            (mo["idts"], mo["psts"], mo["gaps"]), p
        assert (hrecs["beg_coords"][k], hrecs["end_coords"][k]) == (mo["beg"], mo["end"]), p
        oracle_hits.append((le, p))
    # --- order of the reported hits, restricted to the sample
    order = bp.hit_list()
    gpu_order = [int(hrecs["org_pro_no"][k]) for k in order if int(hrecs["org_pro_no"][k]) in local]
    oracle_hits.sort(key=lambda h: h[0])     # stable: ties stay in database order
    assert gpu_order == [p for _, p in oracle_hits]
    return npassed, nreal


def test_q1500_long_profiles(oracle_lib, ss_table):
    """The long-query stress shape: query 1,500, window 128, ten profiles of
    500-1,500 positions, half of them planted homologs; E-values for the
    configuration's whole 20,000-profile database."""
    from cother_b200 import synth
    q = synth.make_profiles([1500], 15001, True, window=128)
    lens = synth.uniform_lengths(10, 500, 1500, seed=15002)
    db = synth.make_profiles(lens, 15003, False, window=128)
    synth.plant_homologs(q, db, 0.5, seed=15004)
    full = synth.db_lengths("q1500_db20k")
    db_len, n_seqs = int(full.sum()), len(full)
    assert np.all(q.dd[0] == 99)           # every query list is full (window 128)
    bp = _search(q, db, ss_table, db_len, n_seqs)
    npassed, nreal = _check_sample(bp, oracle_lib, q, db, ss_table, np.arange(db.nprofiles),
                                   db_len, n_seqs)
    assert nreal >= 3, (npassed, nreal)
    bp.close()


def test_q400_db50k_sampled(oracle_lib, ss_table):
    """The batched configuration at full size: query 400 against all 50,000
    profiles (12.4 M positions, one slab) on the GPU; every planted homolog
    and 300 profiles drawn across the rest of the database are checked
    against the oracle."""
    from cother_b200 import synth
    q, db = synth.make_workload("q400_db50k")
    planted = synth.planted_indices("q400_db50k")
    rest = np.setdiff1d(np.arange(db.nprofiles), planted)
    rng = np.random.default_rng(4050)
    sample = np.union1d(planted, rng.choice(rest, size=300, replace=False))
    bp = _search(q, db, ss_table, db.npositions, db.nprofiles)
    npassed, nreal = _check_sample(bp, oracle_lib, q, db, ss_table, sample, db.npositions,
                                   db.nprofiles)
    assert npassed >= 0.9 * len(planted) and nreal >= 0.9 * len(planted), (npassed, nreal)
    bp.close()


@pytest.mark.parametrize("qindex,ndb", [(0, 1500), (1, 400), (2, 100)])
def test_query_length_sweep(oracle_lib, ss_table, qindex, ndb):
    """The precision configuration's query lengths (64, 256, 1,024) against
    databases of the 50,000-profile length law sized to about 25 M cells,
    5 % planted homologs, E-values for the whole database; every profile is
    checked."""
    from cother_b200 import synth
    q, db = synth.make_workload("qsweep_db50k", ndb=ndb, qindex=qindex, homologs=0.05)
    full = synth.db_lengths("qsweep_db50k")
    db_len, n_seqs = int(full.sum()), len(full)
    bp = _search(q, db, ss_table, db_len, n_seqs)
    npassed, nreal = _check_sample(bp, oracle_lib, q, db, ss_table, np.arange(db.nprofiles),
                                   db_len, n_seqs)
    assert nreal >= 3, (npassed, nreal)
    bp.close()
