"""Oracle (test infrastructure only): a plain-Python restatement of the
reference's text output of search results, the checker of the library's
formatting (cother_b200/csrc/format.cpp). Nothing in the product imports it.

Follows, line by line in effect:
  * FormatDescription / FormatDescriptionJSON  src/liblib/fmtdescription.h:35-123
  * CompressResultsPlain and its helpers      src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:35-385
  * CompressResultsJSON and its helpers       src/libmycu/cupro/CuBatchProcessingFinalizerJSON.cpp:35-380
  * GetBitScore / GetEvalue / GetPvalue        src/libmycu/cupro/CuBatchProcessingFinalizer.h:179-188
  * WriteResultsPlain and its helpers          src/libmycu/cualn/AlnWriterPlain.cpp:19-398
  * WriteResultsJSON and its helpers           src/libmycu/cualn/AlnWriterJSON.cpp:19-429
  * MergeResults                               src/libmycu/cualn/AlnWriter.cpp:216-256
Constants: OUTPUTINDENT 13, ANNOTATIONLEN 75, BUF_MAX 256, KBYTE 1024
(src/liblib/mylimits.h:41-59); szTmpBuffer 1 KiB, szWriterBuffer 4 KiB
(src/libmycu/cualn/AlnWriter.h:43-44); NL = "\\n".

FormatDescription and FormatDescriptionJSON are also pinned to the
reference's own header compiled from its source (tests/golden/fmt_desc_ref.json,
made by tests/golden/make_fmt_fixtures.py).
"""
from __future__ import annotations

import math

import numpy as np

INDENT = 13
ANNOTLEN = 75
KBYTE = 1024
TMPBUF = KBYTE
WRITERBUF = 4 * KBYTE
LN2 = np.float32(0.69314718055994530941723212146)
LOG_DP_MAX = np.float32(7.0978271289338397e+02)


def _f32bits_u(x) -> int:
    return int(np.float32(x).view(np.uint32))


def _f32bits_i(x) -> int:
    return int(np.float32(x).view(np.int32))


def format_description(out: list, desc: str, maxoutlen: int, indent: int, width: int, outpos: int,
                       linepos: int, addsep: str):
    """fmtdescription.h:35-86; appends to the list of characters `out`,
    returns (outpos, linepos)."""
    i = 0
    n = len(desc)
    while i < n and desc[i] in " \t\n\r":
        i += 1
    if addsep:
        out.append(addsep)
        outpos += 1
        linepos += 1
    while i < n and outpos < maxoutlen:
        if desc[i] in " \t":
            while i < n and desc[i] in " \t":
                i += 1
            if width < maxoutlen:
                loc = linepos + 1
                p = i
                while p < n and desc[p] not in " \t" and loc < width:
                    p += 1
                    loc += 1
                if width <= loc:
                    out.append("\n")
                    outpos += 1
                    for _ in range(indent):
                        out.append(" ")
                        outpos += 1
                    linepos = indent
                else:
                    out.append(" ")
                    outpos += 1
                    linepos += 1
            else:
                out.append(" ")
                outpos += 1
                linepos += 1
            continue
        out.append(desc[i])
        i += 1
        outpos += 1
        linepos += 1
    if maxoutlen <= outpos and 3 < maxoutlen:
        for k in range(1, 4):
            if k <= len(out):
                out[-k] = "."
    return outpos, linepos


def format_description_json(out: list, desc: str, maxoutlen: int, outpos: int) -> int:
    """fmtdescription.h:96-123."""
    i = 0
    n = len(desc)
    while i < n and desc[i] in " \t\n\r":
        i += 1
    while i < n and outpos < maxoutlen:
        if desc[i] in " \t":
            while i < n and desc[i] in " \t":
                i += 1
            out.append(" ")
            outpos += 1
            continue
        elif desc[i] in '"\\/':
            out.append("\\")
            outpos += 1
            if maxoutlen <= outpos:
                break
        out.append(desc[i])
        i += 1
        outpos += 1
    if maxoutlen <= outpos and 3 < maxoutlen:
        k = 1
        while k <= 3:
            if k <= len(out):
                out[-k] = "."
            k += 1
        while k <= outpos and k <= len(out) and out[-k] == "\\":
            out[-k] = "."
            k += 1
    return outpos


def bit_score(sspace, logeval) -> float:
    sspace = np.float32(sspace)
    if sspace <= 0:
        return 0.0
    return float((np.log(sspace) - np.float32(logeval)) / LN2)


def evalue_of(logeval) -> float:
    return 1.0e308 if LOG_DP_MAX < np.float32(logeval) else math.exp(float(logeval))


def pvalue_of(e: float) -> float:
    return e if e < 0.01 else 1.0 - math.exp(-e)


def reported(recs: np.ndarray, logevthld) -> list:
    """Finalizer order: log E <= threshold, alignment length >= 1, sorted by
    log E, ties in record order."""
    idx = [k for k in range(recs.shape[0])
           if not (np.float32(logevthld) < recs[k, 8]) and _f32bits_i(recs[k, 9]) >= 1]
    return sorted(idx, key=lambda k: float(recs[k, 8]))


def _fmt_hit_common(recs, rows, k, prof_len, query_len):
    r = recs[k]
    prof = _f32bits_u(r[1])
    plen = int(prof_len[prof])
    alnlen = _f32bits_i(r[9])
    beg = _f32bits_u(r[2]) + plen - 1 + (k + 1) * query_len - alnlen
    seg = [bytes(rows[s, beg:beg + alnlen]).decode("latin-1") for s in range(5)]
    return r, prof, plen, alnlen, seg


def _stat_pair(r, K, lmbd, na):
    kp = lp = na
    if r[12] < 0:
        if K > 0:
            kp = "%6.4f" % K
        if lmbd > 0:
            lp = "%6.4f" % lmbd
    return kp, lp


def hit_plain(recs, rows, k, prof_len, prof_eno, prof_ss, descs, query_len, query_eno, query_ss,
              ssswgt, sspace, dsclen=1024, dscwidth=80, alnwidth=60, show=1):
    """(annotation, hit record) of record k (CuBatchProcessingFinalizerPlain.cpp:93-147)."""
    r, prof, plen, alnlen, seg = _fmt_hit_common(recs, rows, k, prof_len, query_len)
    logeval = r[8]
    evalue = evalue_of(logeval)
    score = float(r[0])
    desc = descs[prof] if descs is not None else None
    # MakeAnnotationPlain (:158-181)
    a = []
    if desc is not None:
        format_description(a, desc, ANNOTLEN, 0, ANNOTLEN, 0, 0, "")
    a.extend(" " * max(0, ANNOTLEN - len(a)))
    annot = "".join(a) + " %7.0f %7.1g\n" % (score, evalue)
    o = []
    width = dscwidth if INDENT < dscwidth else 1
    if desc is not None:
        format_description(o, desc, dsclen, INDENT, width, 0, 0, ">")
    o.append("\n")
    s = "".join(o)
    # FormatScoresPlain (:193-238)
    psts, idts, gaps = int(r[3]), int(r[16]), int(r[17])
    s += "  Length/ENO: Query = %d/%.1f, Sbjct = %d/%.1f\n\n" % (query_len, query_eno, plen, prof_eno[prof])
    s += " Score = %.2f (%.1f bits),  Expect = %.2g, P-value = %.2g\n" % (
        score, bit_score(sspace, logeval), evalue, pvalue_of(evalue))
    if idts > 0:
        s += " Identities = %d/%d (%d%%)" % (idts, alnlen, idts * 100 // alnlen)
    if psts > 0:
        if idts:
            s += ","
        s += " Positives = %d/%d (%d%%)" % (psts, alnlen, psts * 100 // alnlen)
    if gaps > 0:
        if idts or psts:
            s += ","
        s += " Gaps = %d/%d (%d%%)" % (gaps, alnlen, gaps * 100 // alnlen)
    s += "\n\n"
    # FormatAlignmentPlain (:250-336)
    b = _f32bits_u(r[4])
    qrybeg = (b & 0xffff) + 1
    trgbeg = ((b >> 16) & 0xffff) + 1
    trgss = True if prof_ss is None else bool(prof_ss[prof])
    printsss = ssswgt > 0 and query_ss and trgss
    for f in range(0, alnlen, alnwidth):
        nb = min(alnwidth, alnlen - f)
        if printsss:
            s += "%-13s" % "struct" + seg[3][f:f + nb] + "\n"
        p = seg[0][f:f + nb]
        s += "Query: %5u " % qrybeg + p
        fg = p.count("-")
        qrybeg += nb - fg
        s += " %-5d\n" % (qrybeg if nb <= fg else qrybeg - 1)
        s += " " * 13 + seg[1][f:f + nb] + "\n"
        p = seg[2][f:f + nb]
        s += "Sbjct: %5u " % trgbeg + p
        fg = p.count("-")
        trgbeg += nb - fg
        s += " %-5d\n" % (trgbeg if nb <= fg else trgbeg - 1)
        if printsss:
            s += "%-13s" % "struct" + seg[4][f:f + nb] + "\n"
        s += "\n"
    # FormatFooterPlain (:342-385)
    if show:
        s += "%25s  %-6s   %-6s\n" % (" ", "K", "Lambda")
        kp, lp = _stat_pair(r, r[15], r[14], "n/a")
        s += "%-25s  %6s   %6s\n" % ("Computed  ungapped,", kp, lp)
        kp, lp = _stat_pair(r, r[7], r[6], "n/a")
        s += "%-25s  %6s   %6s\n" % ("Estimated gapped,", kp, lp)
        s += "Entropy, %6.4f; Expected, %6.4f; Min/Max, %.0f/%-.0f\n\n" % (r[13], r[12], r[10], r[11])
    s += "\n\n"
    return annot, s


def hit_json(recs, rows, k, prof_len, prof_eno, prof_ss, descs, query_len, query_eno, query_ss,
             ssswgt, sspace, dsclen=1024, **_):
    """(annotation, hit record) of record k (CuBatchProcessingFinalizerJSON.cpp:85-148)."""
    r, prof, plen, alnlen, seg = _fmt_hit_common(recs, rows, k, prof_len, query_len)
    logeval = r[8]
    evalue = evalue_of(logeval)
    score = float(r[0])
    desc = descs[prof] if descs is not None else None
    a = ['    {"summary_entry": {\n      "description": "']
    d = []
    if desc is not None:
        format_description_json(d, desc, ANNOTLEN, 0)
    annot = "".join(a) + "".join(d) + '",\n' + '      "score": %.0f,\n      "evalue": %.2g\n    }}' % (score, evalue)
    d = []
    if desc is not None:
        format_description_json(d, desc, dsclen, 0)
    s = '    {"hit_record": {\n      "target_description": "' + "".join(d) + '",\n'
    s += ('      "query_length": %d,\n      "query_eno": %.1f,\n      "target_length": %d,\n'
          '      "target_eno": %.1f,\n      "alignment": {\n') % (query_len, query_eno, plen, prof_eno[prof])
    psts, idts, gaps = int(r[3]), int(r[16]), int(r[17])
    s += ('        "score": %.2f,\n        "bit_score": %.1f,\n        "evalue": %.2g,\n'
          '        "pvalue": %.2g,\n') % (score, bit_score(sspace, logeval), evalue, pvalue_of(evalue))
    s += ('        "n_identities": %d,\n        "n_positives": %d,\n        "n_gaps": %d,\n'
          '        "aln_length": %d,\n') % (idts, psts, gaps, alnlen)
    b = _f32bits_u(r[4])
    qrybeg = (b & 0xffff) + 1
    trgbeg = ((b >> 16) & 0xffff) + 1
    ngq, ngt = seg[0].count("-"), seg[2].count("-")
    qryend, trgend = qrybeg + alnlen - ngq, trgbeg + alnlen - ngt
    trgss = True if prof_ss is None else bool(prof_ss[prof])
    pss = 1 if (query_ss and trgss) else 0
    s += ('        "query_from": %u,\n        "query_to": %u,\n        "target_from": %u,\n'
          '        "target_to": %u,\n') % (qrybeg, qryend if alnlen <= ngq else qryend - 1,
                                          trgbeg, trgend if alnlen <= ngt else trgend - 1)
    s += ('        "query_secstr_available": %d,\n        "target_secstr_available": %d,\n'
          '        "query_secstr": "') % (pss, pss)
    # SS rows that nothing filled (SSSWGT = 0) end at their first NUL
    s += (seg[3].split("\0")[0] if pss else "") + '",\n        "target_secstr": "' + \
        (seg[4].split("\0")[0] if pss else "")
    s += '",\n        "query_aln": "' + seg[0] + '",\n        "target_aln": "' + seg[2]
    s += '",\n        "middle": "' + seg[1] + '",\n'
    kp, lp = _stat_pair(r, r[15], r[14], "NA")
    s += '        "computed_K_ungapped": "%s",\n        "computed_lambda_ungapped": "%s",\n' % (kp, lp)
    kp, lp = _stat_pair(r, r[7], r[6], "NA")
    s += ('        "estimated_K_gapped": "%s",\n        "estimated_lambda_gapped": "%s",\n'
          '        "entropy": %.4f,\n        "expected_score": %.4f,\n        "min_score": %.0f,\n'
          '        "max_score": %.0f\n') % (kp, lp, r[13], r[12], r[10], r[11])
    s += "      }\n    }}"
    return annot, s


def format_hits(recs, rows, prof_len, prof_eno, descs, query_len, query_eno, logevthld, sspace,
                ssswgt=0.12, prof_ss=None, query_ss=True, fmt=0, **fo):
    fn = hit_json if fmt == 1 else hit_plain
    return [fn(recs, rows, k, prof_len, prof_eno, prof_ss, descs, query_len, query_eno, query_ss,
               ssswgt, sspace, **fo) for k in reported(recs, logevthld)]


def merge_hit_lists(logevals) -> list:
    """AlnWriter::MergeResults: std::merge of the running list with each
    part in turn (ties take the running list first)."""
    merged = []
    for p, lst in enumerate(logevals):
        add = [(p, i) for i in range(len(lst))]
        out, a, b = [], 0, 0
        while a < len(merged) and b < len(add):
            if np.float32(logevals[add[b][0]][add[b][1]]) < np.float32(logevals[merged[a][0]][merged[a][1]]):
                out.append(add[b])
                b += 1
            else:
                out.append(merged[a])
                a += 1
        out += merged[a:] + add[b:]
        merged = out
    return merged


def _eff(query_len, db_size, db_entries, delta):
    effq, effdb = query_len, db_size
    if delta < query_len:
        effq -= delta
    if db_entries * delta < db_size:
        effdb -= db_entries * delta
    return effq, effdb


def write_report(hits, query_len, db_size, db_entries, logevthld, sspace, delta, query_desc=None,
                 db_names=(), program=None, version=None, references=None, ref_lambda=1.116276,
                 ref_k=0.115812, gapped_lambda=0.561132, gapped_k=0.001488, nohits=700, noalns=700,
                 fmt=0, dsclen=1024, dscwidth=80, **_):
    """AlnWriter::WriteResultsPlain / WriteResultsJSON for one query."""
    f32 = lambda x: float(np.float32(x))  # noqa: E731
    o = []
    found = len(hits) > 0
    if fmt == 0:
        # WritePrognamePlain
        if program is not None:
            o.append(program)
        if version is not None:
            o.append(" " + version)
        if program is not None or version is not None:
            o.append("\n\n")
        size = len("".join(o))
        maxsize = WRITERBUF - size - 4
        if maxsize >= 1:
            chars = []
            outpos = linepos = 0
            for ref in (references or []):
                if not (outpos < maxsize):
                    break
                outpos, linepos = format_description(chars, ref, maxsize, 0, dscwidth, outpos, linepos, "")
                chars.append("\n")
                outpos += 1
                linepos = 0
            o.append("".join(chars) + "\n")
        # WriteQueryDescriptionPlain
        left = min(WRITERBUF - len("".join(o)), dsclen)
        if left >= 40:
            head = "\n Query (%d positions):\n" % query_len
            o.append(head)
            ms = left - len(head)
            if ms >= 1 and query_desc is not None:
                chars = []
                format_description(chars, query_desc, ms, 0, dscwidth, 0, 0, "")
                o.append("".join(chars))
        # WriteSearchInformationPlain
        si = []

        def over(delta):
            sz = len("".join(si))
            if TMPBUF < sz + delta:
                if sz + 5 < TMPBUF:
                    si.append("...\n\n")
                return True
            return False
        done = False
        if over(30):
            done = True
        if not done:
            si.append("\n\n Database(s):\n")
            for nm in db_names:
                szn = min(len(nm), 100)
                if over(szn + 2):
                    done = True
                    break
                t = list(nm[:szn])
                if szn < len(nm) and 3 < szn:
                    t[-3:] = "..."
                si.append("".join(t) + "\n")
        if not done and over(INDENT + 40):
            done = True
        if not done:
            si.append(" " * INDENT + "%d profiles\n" % db_entries)
            if over(INDENT + 50):
                done = True
        if not done:
            si.append(" " * INDENT + "%d total positions\n\n\n" % db_size)
            if over(ANNOTLEN * 2):
                done = True
        if not done:
            if found:
                msg = " Profiles found below the e-value threshold:"
                si.append(msg + " " * max(0, ANNOTLEN - len(msg)) + " %7s %7s\n\n" % ("Score", "E-value"))
            else:
                si.append(" No profiles found below an e-value threshold of %g.\n\n\n" % math.exp(f32(logevthld)))
        o.append("".join(si))
        if found:
            o.extend(h[0] for h in hits[:nohits])
            o.append("\n\n\n")
            o.extend(h[1] for h in hits[:noalns])
        effq, effdb = _eff(query_len, db_size, db_entries, delta)
        o.append("%-20s  %-6s   %-6s\n" % ("Reference values of", "K", "Lambda"))
        o.append("%-20s  %6.4f   %6.4f\n" % ("Ungapped", f32(ref_k), f32(ref_lambda)))
        o.append("%-20s  %6.4f   %6.4f\n\n" % ("Gapped", f32(gapped_k), f32(gapped_lambda)))
        o.append("Length of query, %d\nLength of database, %d\n" % (query_len, db_size))
        o.append("Effective length of query, %d\nEffective length of database, %d\n" % (effq, effdb))
        o.append("Effective search space, %d\n\n" % int(f32(sspace)))
        return "".join(o)
    # JSON: WritePrognameJSON
    head = '{"cother_search": {\n  "program": "%s",\n  "version": "%s",\n' % (program or "", version or "")
    o.append(head)
    if WRITERBUF - len(head) - KBYTE >= 1:
        o.append('  "references": [\n')
        refs = list(references or []) + [None]
        tot, bwrt, i = 0, True, 0
        while i == 0 or (bwrt and refs[i] is not None):
            s = refs[i]
            tot += len(s) if s is not None else 0
            bwrt = tot < KBYTE - 60
            o.append('    "%s"%s\n' % (s if (bwrt and s is not None) else "",
                                       "," if (bwrt and s is not None and refs[i + 1] is not None) else ""))
            if s is None:
                break
            i += 1
        o.append("  ],\n")
    # WriteQueryDescriptionJSON
    left = min(WRITERBUF - len("".join(o)), dsclen)
    if left >= 60:
        qh = '  "query": {\n    "length": %d,\n' % query_len
        o.append(qh)
        ms = left - len(qh) - 256
        if ms >= 1:
            pre = '    "name": "' + '",\n' + '    "description": "'
            chars = []
            if query_desc is not None:
                format_description_json(chars, query_desc, ms, len(pre))
            o.append(pre + "".join(chars) + '"\n  },\n')
    # WriteSearchInformationJSON
    maxsize = TMPBUF - 40 * 7
    if maxsize >= 1:
        o.append('  "database": {\n    "names": [\n')
        for d, nm in enumerate(db_names):
            szn = min(len(nm), 99)
            maxsize -= szn + 15
            if maxsize < 1:
                o.append('      "..."\n')
                break
            chars = []
            format_description_json(chars, nm, szn + 1, 0)
            o.append('      "' + "".join(chars) + ('",\n' if d + 1 < len(db_names) else '"\n'))
        o.append('    ],\n    "number_of_profiles": %d,\n    "number_of_positions": %d\n  },\n'
                 % (db_entries, db_size))
        maxsize -= 90 * 4
        if maxsize >= 1:
            if found:
                o.append('  "message": "Profiles found below the e-value threshold:",\n')
            else:
                o.append('  "message": "No profiles found below an e-value threshold of %g",\n'
                         % math.exp(f32(logevthld)))
    o.append('  "search_summary": [\n')
    if found:
        for i, h in enumerate(hits[:nohits]):
            last = not (i + 1 < len(hits) and i + 1 < nohits)
            o.append(h[0] + ("\n" if last else ",\n"))
    o.append('  ],\n  "search_hits": [\n')
    if found:
        for i, h in enumerate(hits[:noalns]):
            last = not (i + 1 < len(hits) and i + 1 < nohits)
            o.append(h[1] + ("\n" if last else ",\n"))
    o.append("  ],\n")
    effq, effdb = _eff(query_len, db_size, db_entries, delta)
    o.append(('  "search_statistics": {\n    "reference_K_ungapped": %.4f,\n'
              '    "reference_lambda_ungapped": %.4f,\n    "reference_K_gapped": %.4f,\n'
              '    "reference_lambda_gapped": %.4f,\n    "query_length": %d,\n'
              '    "database_size": %d,\n    "effective_query_length": %d,\n'
              '    "effective_database_size": %d,\n    "effective_search_space": %d\n  }\n}}\n')
             % (f32(ref_k), f32(ref_lambda), f32(gapped_k), f32(gapped_lambda), query_len, db_size,
                effq, effdb, int(f32(sspace))))
    return "".join(o)
