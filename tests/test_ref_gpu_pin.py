"""The oracle pinned against the reference's own CUDA kernels.

tests/golden/ref_gpu_<case>.npz hold every intermediate result of the
reference's score-matrix, phase-1 DP, statistics and MAP kernels, compiled
from their sources and run on a B200 by tests/golden/make_ref_gpu_fixtures.py
on small seeded searches. Each stage of the oracle is fed the reference's own
inputs for that stage (its score matrix, its phase-1 records, its log
E-values), so that every comparison isolates one stage:

* score matrix: modular scores (SS + DDMS) bit for bit; full scores within
  1e-6 absolute + 1e-4 relative, because the profile-profile term's log is
  the reference's __logf intrinsic there and a series restatement here;
* phase-1 DP: backtrack codes, maxima, positives and coordinates bit for bit;
* statistics: min/max exactly, lambda, K, H, E, log E and the SS18/observed
  estimates within 1e-4 relative (the reference uses __expf/__logf);
* MAP: the set of realigned pairs, alignment rows, identity/positive/gap
  counts, coordinates and alignment lengths exactly; under MAPALN=0 the same
  for the phase-1 alignments the reference reports instead.

CPU only: nothing here needs a GPU.
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
import make_ref_gpu_fixtures as fx  # noqa: E402

CASES = sorted(fx.CASES)
STAT_FIELDS = ["lambda_est", "K_est", "logE", "logEpA", "min", "max", "E", "H", "lambda", "K"]


def _load(case):
    F = np.load(os.path.join(GOLDEN, f"ref_gpu_{case}.npz"))
    opts = json.loads(str(F["options"]))
    q, db = fx.case_inputs(opts.get("inputs", "q64"))
    assert str(F["digest"]) == fx.input_digest(q, db), "regenerated inputs differ"
    if "scores" in F:
        full = F
    else:
        full = np.load(os.path.join(GOLDEN, "ref_gpu_main.npz"))
        assert json.loads(str(full["options"])).get("inputs", "q64") == opts.get("inputs", "q64")
    N = db.npositions
    return F, opts, q, db, full["scores"][:, :N], full["modscores"][:, :N]


def _org(rec):
    return rec[:, 1].view(np.uint32).astype(np.int64)


def _cvs_step(cvswgt):
    """Largest change of the weighted CVS term between neighbouring map
    entries: what a lookup moved by the reference's fast logarithm costs."""
    m = np.load(os.path.join(GOLDEN, "cvs2s.npz"))["scores"].astype(np.float64)
    return float(np.max(np.abs(np.diff(m)))) * cvswgt + 1e-6


@pytest.mark.parametrize("case", [c for c in CASES if fx.CASES[c]["full"]])
def test_score_matrix_matches_reference_kernels(case, ss_table, oracle_lib):
    """Modular scores bit for bit, full scores within the tolerance of the
    profile-profile term's log. With the CVS term, the cells whose map
    lookup lies within the error bound of the reference's __logf of a map
    edge (flagged by the oracle, about 2 in 10,000) may take the
    neighbouring entry; all others match bit for bit too."""
    F, opts, q, db, rs, rm = _load(case)
    cvswgt = opts.get("cvswgt", 0.0)
    mapaln = not opts.get("nomapaln", 0)
    out = oracle_lib.score_matrix(q, db, ss_table, ssswgt=opts["ssswgt"],
                                  ddmswgt=opts["ddmswgt"], dstsegm=opts["dstsegm"],
                                  cvswgt=cvswgt, ambiguous=cvswgt > 0, mapaln=mapaln,
                                  initshift=0.002 if mapaln else 0.0003)
    os_, om = out[0], out[1]
    amb = out[2].astype(bool) if cvswgt > 0 else np.zeros(om.shape, bool)
    assert amb.mean() < 1e-3
    assert np.array_equal(om[~amb], rm[~amb])
    assert np.all(np.abs(om[amb] - rm[amb]) <= _cvs_step(cvswgt))
    tol = 1e-6 + 1e-4 * np.abs(rs)
    assert np.all((np.abs(os_ - rs) <= tol)[~amb])
    assert np.all(np.abs(os_ - rs)[amb] <= tol[amb] + _cvs_step(cvswgt))


@pytest.mark.parametrize("case", [c for c in CASES if fx.CASES[c]["full"]])
def test_phase1_matches_reference_kernels(case, oracle_lib):
    F, opts, q, db, rs, rm = _load(case)
    N = db.npositions
    rec, bt = oracle_lib.dp1(q, db, rs, 0, 0, db.nprofiles, float(F["scorethld"]))
    assert np.array_equal(bt, F["btck"][:, :N])
    ph = F["phase1"]
    assert len(ph) == db.nprofiles == int(F["globvars"][0])
    org = _org(ph)
    assert sorted(org) == list(range(db.nprofiles))
    assert np.array_equal(ph[:, 0], rec["score"][org])
    assert np.array_equal(ph[:, 3], rec["psts"][org])
    assert np.array_equal(ph[:, 4].view(np.uint32), rec["beg"][org].astype(np.uint32))
    assert np.array_equal(ph[:, 5].view(np.uint32), rec["end"][org].astype(np.uint32))
    # phase-2 offsets: in the reference's (atomic) pass order, each passed
    # profile starts where the previous one ends in the compacted buffer
    dst = ph[:, 2].view(np.uint32).astype(np.int64)
    order = np.argsort(dst)
    ends = np.cumsum(db.lens[org[order]].astype(np.int64))
    assert np.array_equal(dst[order], np.concatenate([[0], ends[:-1]]))
    assert int(F["globvars"][1]) == int(db.lens.sum())
    assert int(F["globvars"][2]) == int(db.lens.max())


@pytest.mark.parametrize("case", CASES)
def test_statistics_match_reference_kernels(case, oracle_lib):
    F, opts, q, db, rs, rm = _load(case)
    st = F["stats"]
    Lq = q.npositions
    for k in range(len(st)):
        p = int(_org(st[k:k + 1])[0])
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        out, _ = oracle_lib.pair_statistics(
            rs[:, s0:s0 + Ld], q.aa, db.aa[s0:s0 + Ld], st[k, 0], st[k, 3], Lq, Ld, q.eno[0],
            db.eno[p], float(F["searchspace"]), ssemodel=opts["ssemodel"], xuninf=opts["xuninf"])
        ref = st[k, 6:16]
        assert out[4] == ref[4] and out[5] == ref[5], (p, "min/max")
        rel = np.abs(out - ref) / np.maximum(np.abs(ref), 1e-30)
        bad = [(n, float(a), float(b)) for n, a, b, r in zip(STAT_FIELDS, out, ref, rel) if r > 1e-4]
        assert not bad, (p, bad)


@pytest.mark.parametrize("case", CASES)
def test_map_alignments_match_reference_kernels(case, oracle_lib):
    F, opts, q, db, rs, rm = _load(case)
    st, fin, rows = F["stats"], F["final"], F["alns"]
    Lq = q.npositions
    thld = float(F["logevthld"])
    nrows = 5 if opts["ssswgt"] > 0 else 3
    nmap = 0
    if opts.get("nomapaln", 0):
        rec1, bt1 = oracle_lib.dp1(q, db, rs, 0, 0, db.nprofiles, float(F["scorethld"]))
    for k in range(len(fin)):
        p = int(_org(fin[k:k + 1])[0])
        s0, Ld = int(db.starts[p]), int(db.lens[p])
        alnlen = int(fin[k, 9].view(np.int32))
        if st[k, 8] > thld:
            assert alnlen == 0, p           # not realigned
            continue
        nmap += 1
        if opts.get("nomapaln", 0):
            # MAPALN=0: the phase-1 alignment from the phase-1 maximum
            o = oracle_lib.aln_pair(q, db, p, rs[:, s0:s0 + Ld], bt1[:, s0:s0 + Ld],
                                    rec1["maxsc"][p], rec1["maxr"][p], rec1["maxc"][p],
                                    printsss=opts["ssswgt"] > 0)
        else:
            o = oracle_lib.map_pair(q, db, p, rs[:, s0:s0 + Ld], rm[:, s0:s0 + Ld], st[k, 9],
                                    minpp=opts["minpp"],
                                    modscores=opts["ssswgt"] > 0 or opts.get("cvswgt", 0) > 0,
                                    printsss=opts["ssswgt"] > 0)
        assert alnlen == o["alnlen"], p
        end = int(fin[k, 2].view(np.uint32)) + k * Lq + Ld + Lq - 1
        for r in range(nrows):
            assert bytes(rows[r, end - alnlen:end]).decode() == o["aln"][r], (p, r)
            assert rows[r, end] == 0, (p, r)
        assert (int(fin[k, 16]), int(fin[k, 17]), int(fin[k, 3])) == \
            (o["idts"], o["gaps"], o["psts"]), p
        assert (int(fin[k, 4].view(np.uint32)), int(fin[k, 5].view(np.uint32))) == \
            (o["beg"], o["end"]), p
    assert nmap >= 2
