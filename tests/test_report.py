"""Text output of the results (plain and JSON), on the CPU.

* The oracle's restatement of the reference's description formatters equals
  the reference's own FormatDescription / FormatDescriptionJSON on the
  committed golden vectors (tests/golden/fmt_desc_ref.json).
* The library's per-hit text (cbp_format_hits_host) carries exactly those
  formatter outputs in the annotation lines and hit records.
* On the hit records and alignment rows that the reference's own kernels
  produced (tests/golden/ref_gpu_*.npz), the library's per-hit text and the
  per-query report equal the oracle's restatement byte for byte, for both
  formats and several output options.
* The merge of per-chunk hit lists is the reference writer's stable merge.
"""
import json
import os
import random
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)

from oracle import report as R  # noqa: E402


@pytest.fixture(scope="module")
def golden_desc():
    with open(os.path.join(GOLDEN, "fmt_desc_ref.json")) as f:
        return json.load(f)


def _fd(d, m, ind, w, op, lp, sep):
    out = []
    R.format_description(out, d, m, ind, w, op, lp, sep)
    return "".join(out)


def _fdj(d, m, op):
    out = []
    R.format_description_json(out, d, m, op)
    return "".join(out)


def test_oracle_description_formatters_match_reference(golden_desc):
    n = 0
    for c in golden_desc:
        d = c["desc"]
        assert _fd(d, 75, 0, 75, 0, 0, "") == c["annot_plain"]
        assert _fd(d, 1024, 13, 80, 0, 0, ">") == c["rec_plain_1024_80"]
        assert _fd(d, 60, 13, 30, 0, 0, ">") == c["rec_plain_60_30"]
        assert _fdj(d, 75, 0) == c["annot_json"]
        assert _fdj(d, 1024, 0) == c["rec_json_1024"]
        assert _fdj(d, 60, 0) == c["rec_json_60"]
        for g in c["generic"]:
            if "args" in g:
                m, ind, w, op, lp, sep = g["args"]
                assert _fd(d, m, ind, w, op, lp, sep) == g["out"], (d, g["args"])
            else:
                m, op = g["json_args"]
                assert _fdj(d, m, op) == g["out"], (d, g["json_args"])
            n += 1
    assert n == 12 * len(golden_desc)


def _one_hit_inputs():
    """A single synthetic reported hit: 9 aligned columns, one gap each side."""
    rec = np.zeros((1, 18), np.float32)
    rec[0, 0] = 31.7
    rec[0, 1] = np.uint32(0).view(np.float32)
    rec[0, 2] = np.uint32(0).view(np.float32)
    rec[0, 3] = 5
    rec[0, 4] = np.uint32((2 << 16) | 3).view(np.float32)
    rec[0, 8] = -7.25
    rec[0, 9] = np.int32(9).view(np.float32)
    rec[0, 10:16] = [-9, 7, -0.6, 0.8, 0.3, 0.05]
    rec[0, 6:8] = [0.26, 0.02]
    rec[0, 16:18] = [3, 2]
    Lq, Ld = 12, 20
    n = Ld + Lq
    rows = np.zeros((5, n), np.uint8)
    aln = ["ACD-EFGHI", "+ | + +  ", "AC-DEFGHI", "HHHE-CCCH", "HH-EECCCH"]
    beg = Ld - 1 + Lq - 9
    for s in range(5):
        rows[s, beg:beg + 9] = np.frombuffer(aln[s].encode(), np.uint8)
    return rec, rows, [Ld], [7.5]


def test_library_carries_reference_description_text(golden_desc):
    from cother_b200 import report as rep
    rec, rows, plen, peno = _one_hit_inputs()
    for c in golden_desc:
        d = c["desc"]
        for fmt in (rep.PLAIN, rep.JSON):
            for dsclen, dscwidth, key_p, key_j in ((1024, 80, "rec_plain_1024_80", "rec_json_1024"),
                                                    (60, 30, "rec_plain_60_30", "rec_json_60")):
                fo = rep.FormatOptions.defaults(fmt)
                fo.dsclen, fo.dscwidth = dsclen, dscwidth
                (ann, hit), = rep.format_hits_host(rec, rows, plen, peno, 12, 4.2, 0.0, 1e6,
                                                   descs=[d], options=fo)
                if fmt == rep.PLAIN:
                    a = c["annot_plain"]
                    assert ann == a + " " * max(0, 75 - len(a)) + ann[max(75, len(a)):]
                    assert hit.startswith(c[key_p] + "\n  Length/ENO:")
                else:
                    assert ann.startswith('    {"summary_entry": {\n      "description": "'
                                          + c["annot_json"] + '",\n')
                    assert hit.startswith('    {"hit_record": {\n      "target_description": "'
                                          + c[key_j] + '",\n')


def _descs(n, seed):
    rng = random.Random(seed)
    words = ["alpha", "beta/gamma", "delta\"q\"", "kinase", "domain", "x" * 40, "Homo sapiens",
             "\tprotein", "back\\slash", "uncharacterized", "PF00069", "1abc_A"]
    return [" ".join(rng.choice(words) for _ in range(rng.randint(0, 30))) for _ in range(n)]


CASES = ["main", "q77", "noss", "cvs", "mapaln0"]


@pytest.mark.parametrize("case", CASES)
def test_hits_and_report_match_oracle_on_reference_kernel_output(case):
    import make_ref_gpu_fixtures as fx
    from cother_b200 import report as rep
    F = np.load(os.path.join(GOLDEN, f"ref_gpu_{case}.npz"))
    opts = json.loads(str(F["options"]))
    q, db = fx.case_inputs(opts.get("inputs", "q64"))
    recs = F["final"]
    rows = F["alns"]
    plen = np.asarray(db.lens, np.int32)
    peno = np.asarray(db.eno, np.float32).reshape(-1)
    descs = _descs(db.nprofiles, 5)
    qeno = float(np.asarray(q.eno).reshape(-1)[0])
    logevthld = float(F["logevthld"])
    sspace = float(F["searchspace"])
    ssswgt = float(opts.get("ssswgt", 0.12))
    order = R.reported(recs, logevthld)
    assert len(order) > 0
    pss = np.ones(db.nprofiles, np.uint8)
    pss[::3] = 0
    for fmt in (rep.PLAIN, rep.JSON):
        for dsclen, dscwidth, alnwidth, show in ((1024, 80, 60, 1), (100, 40, 17, 0)):
            fo = rep.FormatOptions.defaults(fmt)
            fo.dsclen, fo.dscwidth, fo.alnwidth, fo.show = dsclen, dscwidth, alnwidth, show
            for prof_ss in (None, pss):
                got = rep.format_hits_host(recs, rows, plen, peno, q.npositions, qeno, logevthld, sspace,
                                           ssswgt=ssswgt, descs=descs, prof_ss=prof_ss, options=fo)
                want = R.format_hits(recs, rows, plen, peno, descs, q.npositions, qeno, logevthld, sspace,
                                     ssswgt=ssswgt, prof_ss=prof_ss, fmt=fmt, dsclen=dsclen,
                                     dscwidth=dscwidth, alnwidth=alnwidth, show=show)
                assert got == want, (case, fmt, dsclen, alnwidth)
            info = dict(query_len=q.npositions, db_size=db.npositions, db_entries=db.nprofiles,
                        log_evalue_threshold=logevthld, search_space=sspace, delta_length=17,
                        query_desc="query " + descs[0], db_names=["pdb70_synthetic", "/data/" + "d" * 120],
                        program="COTHER", version="test", references=["First reference line " * 3,
                                                                       "Second"],
                        nohits=3, noalns=2, options=fo)
            text = rep.write_report(got, **info)
            oinfo = dict(info)
            oinfo.pop("options")
            oinfo["logevthld"] = oinfo.pop("log_evalue_threshold")
            oinfo["sspace"] = oinfo.pop("search_space")
            oinfo["delta"] = oinfo.pop("delta_length")
            assert text == R.write_report(want, fmt=fmt, dsclen=dsclen, dscwidth=dscwidth, **oinfo)
            if fmt == rep.JSON and dsclen >= 512:
                # the reference ends both lists by NOHITS, so the document
                # is valid JSON when NOALNS equals NOHITS (and when DSCLEN
                # leaves room for the query section, which the reference
                # otherwise leaves open)
                info2 = dict(info, nohits=2, noalns=2)
                doc = json.loads(rep.write_report(got, **info2))["cother_search"]
                assert len(doc["search_summary"]) == min(2, len(got))
                assert len(doc["search_hits"]) == min(2, len(got))
                assert doc["search_hits"][0]["hit_record"]["alignment"]["aln_length"] > 0
            # no hits: the "not found" message
            empty = rep.write_report([], **info)
            assert empty == R.write_report([], fmt=fmt, dsclen=dsclen, dscwidth=dscwidth, **oinfo)


def test_plain_hit_layout_fields():
    from cother_b200 import report as rep
    rec, rows, plen, peno = _one_hit_inputs()
    (ann, hit), = rep.format_hits_host(rec, rows, plen, peno, 12, 4.2, 0.0, 1e6, ssswgt=0.12,
                                       descs=["d1 test"])
    lines = hit.split("\n")
    assert lines[0] == ">d1 test"
    assert lines[1] == "  Length/ENO: Query = 12/4.2, Sbjct = 20/7.5"
    assert lines[3].startswith(" Score = 31.70 (")
    assert lines[4] == " Identities = 3/9 (33%), Positives = 5/9 (55%), Gaps = 2/9 (22%)"
    # beginning coordinates (x<<16)|y = (2, 3): query from 4, subject from 3
    assert lines[6] == "struct       HHHE-CCCH"
    assert lines[7] == "Query:     4 ACD-EFGHI 11   "
    assert lines[9] == "Sbjct:     3 AC-DEFGHI 10   "
    assert ann.startswith("d1 test" + " " * 68 + "      32 ")


def test_merge_hit_lists_is_the_writers_stable_merge():
    from cother_b200 import report as rep
    rng = np.random.default_rng(3)
    for _ in range(20):
        parts = [np.sort(rng.choice([-5.0, -3.0, -1.0, 0.5, 2.0], size=rng.integers(0, 6))).astype(np.float32)
                 for _ in range(rng.integers(1, 5))]
        got = rep.merge_hit_lists(parts)
        assert got == R.merge_hit_lists(parts)
        vals = [parts[p][i] for p, i in got]
        assert vals == sorted(vals)


def test_output_filename():
    from cother_b200 import report as rep
    assert rep.output_filename("out", "/q/d1abc.tpro", 3) == "out/d1abc.tpro__3.out"
    assert rep.output_filename("out/", "/q/d1abc.pro", 0, rep.JSON) == "out/d1abc__0.json"
    assert rep.output_filename("", "query", 1) == "query__1.out"


def test_errors():
    from cother_b200 import CbpError
    from cother_b200 import report as rep
    rec, rows, plen, peno = _one_hit_inputs()
    fo = rep.FormatOptions.defaults()
    fo.format = 7
    with pytest.raises(CbpError):
        rep.format_hits_host(rec, rows, plen, peno, 12, 4.2, 0.0, 1e6, options=fo)
    bad = rec.copy()
    bad[0, 1] = np.uint32(5).view(np.float32)     # profile outside the chunk
    with pytest.raises(CbpError):
        rep.format_hits_host(bad, rows, plen, peno, 12, 4.2, 0.0, 1e6)
