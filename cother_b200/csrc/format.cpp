// Text output of the search results, plain and JSON.
//
// Two parts, as in the reference:
//  * the finalizer's per-hit text: for every reported hit an annotation line
//    (the summary list) and a hit record (description, scores, alignment,
//    statistics) -- CuBatchProcessingFinalizer::CompressResultsPlain/JSON
//    (src/libmycu/cupro/CuBatchProcessingFinalizerPlain.cpp:35-385,
//    src/libmycu/cupro/CuBatchProcessingFinalizerJSON.cpp:35-380);
//  * the writer's per-query report: program header, query, database and
//    search information, the first NOHITS annotations, the first NOALNS hit
//    records and the statistics summary -- AlnWriter::WriteResultsPlain/JSON
//    (src/libmycu/cualn/AlnWriterPlain.cpp:19-398,
//    src/libmycu/cualn/AlnWriterJSON.cpp:19-429), after the stable merge of
//    the hit lists of a query's database chunks by log E-value
//    (AlnWriter::MergeResults, src/libmycu/cualn/AlnWriter.cpp:216-256).
// The text is built in std::string instead of pre-sized raw buffers; the
// layout, number formats and truncation rules are the reference's. The
// newline is "\n" (the reference's NL outside Windows, liblib/platform.h:34).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cother_b200.h"

namespace cbp {
void set_last_error(const std::string& msg);
}

namespace {

constexpr int kIndent = 13;          // OUTPUTINDENT (liblib/mylimits.h:56)
constexpr int kAnnotLen = 75;        // ANNOTATIONLEN (liblib/mylimits.h:59)
constexpr int kBufMax = 256;         // BUF_MAX (liblib/mylimits.h:41)
constexpr int kKByte = 1024;         // KBYTE (liblib/mylimits.h:42)
constexpr int kTmpBuffer = kKByte;   // AlnWriter::szTmpBuffer (cualn/AlnWriter.h:43)
constexpr int kWriterBuffer = 4 * kKByte;   // AlnWriter::szWriterBuffer (cualn/AlnWriter.h:44)
constexpr float kLn2 = 0.69314718055994530941723212146f;   // SLC_LN2 (extsp/psl.h:29)
constexpr float kLogDpMax = 7.0978271289338397e+02f;       // SLC_LOG_DP_MAX (extsp/psl.h:49)

// record fields (TDP2OutputAlnData, src/libmycu/cuss/CuBatchSS_com.h:45-71)
enum {
    rScore = 0, rOrgProNo = 1, rNewDst = 2, rPstvs = 3, rBeg = 4, rEnd = 5, rLmbdEst = 6, rKEst = 7,
    rLogE = 8, rEpA = 9, rMin = 10, rMax = 11, rE = 12, rH = 13, rLmbd = 14, rK = 15, rIdnts = 16,
    rNGaps = 17
};
// alignment rows (TDP2OutputAlignment, CuBatchSS_com.h:73-82)
enum { aQuery = 0, aMiddle = 1, aTarget = 2, aQuerySS = 3, aTargetSS = 4 };

struct FormatError {
    int code;
    std::string msg;
};

template <class... A>
void appendf(std::string& o, const char* f, A... a)
{
    char buf[512];
    const int n = std::snprintf(buf, sizeof(buf), f, a...);
    if (n < 0) throw FormatError{CBP_ERR_ARG, "formatting failed"};
    if (n < (int)sizeof(buf)) {
        o.append(buf, (size_t)n);
    } else {
        std::vector<char> big((size_t)n + 1);
        std::snprintf(big.data(), big.size(), f, a...);
        o.append(big.data(), (size_t)n);
    }
}

int put_nl(std::string& o)
{
    o += '\n';
    return 1;
}

bool ws4(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

// FormatDescription (src/liblib/fmtdescription.h:35-86): copy a description
// with runs of blanks collapsed, wrapping at `width` with `indent` blanks
// when width < maxoutlen, stopping at maxoutlen characters (counted in
// outpos, which may arrive non-zero) and marking a cut with "...".
void format_description(std::string& o, const char* desc, int maxoutlen, int indent, int width, int& outpos,
                        int& linepos, char addsep)
{
    while (*desc && ws4(*desc)) desc++;
    if (addsep) {
        o += addsep;
        outpos++;
        linepos++;
    }
    while (*desc && outpos < maxoutlen) {
        if (*desc == ' ' || *desc == '\t') {
            while (*desc == ' ' || *desc == '\t') desc++;
            if (width < maxoutlen) {
                int loc = linepos + 1;
                for (const char* p = desc; *p && *p != ' ' && *p != '\t' && loc < width; p++, loc++) {}
                if (width <= loc) {
                    outpos += put_nl(o);
                    for (int i = 0; i < indent; i++, outpos++) o += ' ';
                    linepos = indent;
                } else {
                    o += ' ';
                    outpos++;
                    linepos++;
                }
            } else {
                o += ' ';
                outpos++;
                linepos++;
            }
            continue;
        }
        o += *desc++;
        outpos++;
        linepos++;
    }
    if (maxoutlen <= outpos && 3 < maxoutlen)
        for (int i = 1; i <= 3 && (size_t)i <= o.size(); i++) o[o.size() - i] = '.';
}

// FormatDescriptionJSON (src/liblib/fmtdescription.h:96-123): blanks
// collapsed, '"', '\' and '/' escaped, cut at maxoutlen with "..." (which
// also replaces the escape characters just before it).
void format_description_json(std::string& o, const char* desc, int maxoutlen, int& outpos)
{
    while (*desc && ws4(*desc)) desc++;
    while (*desc && outpos < maxoutlen) {
        if (*desc == ' ' || *desc == '\t') {
            while (*desc == ' ' || *desc == '\t') desc++;
            o += ' ';
            outpos++;
            continue;
        } else if (*desc == '"' || *desc == '\\' || *desc == '/') {
            o += '\\';
            outpos++;
            if (maxoutlen <= outpos) break;
        }
        o += *desc++;
        outpos++;
    }
    if (maxoutlen <= outpos && 3 < maxoutlen) {
        int i;
        for (i = 1; i <= 3 && (size_t)i <= o.size(); i++) o[o.size() - i] = '.';
        for (; i <= outpos && (size_t)i <= o.size() && o[o.size() - i] == '\\'; i++) o[o.size() - i] = '.';
    }
}

uint32_t ubits(float f)
{
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
int ibits(float f) { return (int)ubits(f); }

// CuBatchProcessingFinalizer::GetBitScore, GetEvalue, GetPvalue
// (src/libmycu/cupro/CuBatchProcessingFinalizer.h:179-188)
float bit_score(float sspace, float logeval)
{
    return sspace <= 0.0f ? 0.0f : (logf(sspace) - logeval) / kLn2;
}
double evalue_of(float logeval) { return kLogDpMax < logeval ? 1.0e+308 : std::exp((double)logeval); }
double pvalue_of(double evalue) { return evalue < 0.01 ? evalue : 1.0 - std::exp(-evalue); }

struct HitsInput {
    const float* recs;
    size_t nrecs;
    const char* rows;
    size_t row_stride, row_length;
    const int* prof_len;
    const float* prof_eno;
    const uint8_t* prof_ss;
    size_t nprof;
    const char* const* descs;
    int query_len;
    float query_eno;
    int query_ss;
    float ssswgt, logevthld, sspace;
};

// the finalizer's reported hits in its order: log E at most the threshold,
// realigned (alignment length >= 1), sorted by log E (equal values in record
// order) (CuBatchProcessingFinalizerPlain.cpp:79-92,
// CuBatchProcessingFinalizer.cpp:283-292)
std::vector<size_t> reported(const HitsInput& in)
{
    std::vector<size_t> idx;
    for (size_t k = 0; k < in.nrecs; k++) {
        const float* r = in.recs + k * CBP_REC_FLOATS;
        if (in.logevthld < r[rLogE]) continue;
        if (ibits(r[rEpA]) < 1) continue;
        idx.push_back(k);
    }
    std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
        return in.recs[a * CBP_REC_FLOATS + rLogE] < in.recs[b * CBP_REC_FLOATS + rLogE];
    });
    return idx;
}

struct HitView {
    const float* r;
    size_t k;              // record index
    uint32_t prof;         // chunk profile index
    int dbprolen;
    float dbeno;
    bool trgss;
    int alnlen;
    const char* aln[5];    // row starts of this hit's alignment
};

HitView view_of(const HitsInput& in, size_t k)
{
    HitView h;
    h.r = in.recs + k * CBP_REC_FLOATS;
    h.k = k;
    h.prof = ubits(h.r[rOrgProNo]);
    if (h.prof >= in.nprof) throw FormatError{CBP_ERR_ARG, "hit record names a profile outside the chunk"};
    h.dbprolen = in.prof_len[h.prof];
    h.dbeno = in.prof_eno[h.prof];
    h.trgss = in.prof_ss ? in.prof_ss[h.prof] != 0 : true;
    h.alnlen = ibits(h.r[rEpA]);
    const long long dst = (long long)ubits(h.r[rNewDst]);
    // the alignment is right-aligned in the hit's slot, which ends at
    // newDst + Ld - 1 + (k+1) Lq (CuBatchProcessingFinalizerPlain.cpp:252-256)
    const long long beg = dst + h.dbprolen - 1 + (long long)(k + 1) * in.query_len - h.alnlen;
    if (beg < 0 || beg + h.alnlen > (long long)in.row_length)
        throw FormatError{CBP_ERR_ARG, "alignment outside the alignment rows"};
    for (int s = 0; s < 5; s++) h.aln[s] = in.rows + (size_t)s * in.row_stride + (size_t)beg;
    return h;
}

const char* desc_of(const HitsInput& in, uint32_t p) { return in.descs ? in.descs[p] : nullptr; }

// ---- plain (CuBatchProcessingFinalizerPlain.cpp) -----------------------

// MakeAnnotationPlain (:158-181)
void annotation_plain(std::string& o, const char* desc, float score, double evalue)
{
    const size_t start = o.size();
    int outpos = 0, linepos = 0;
    if (desc) format_description(o, desc, kAnnotLen, 0, kAnnotLen, outpos, linepos, 0);
    for (size_t w = o.size() - start; w < (size_t)kAnnotLen; w++) o += ' ';
    appendf(o, " %7.0f %7.1g\n", score, evalue);
}

// FormatScoresPlain (:193-238)
void scores_plain(std::string& o, const HitsInput& in, const HitView& h, float score, float logeval,
                  double evalue)
{
    const int psts = (int)h.r[rPstvs], idts = (int)h.r[rIdnts], gaps = (int)h.r[rNGaps];
    const int alnlen = h.alnlen;
    appendf(o, "  Length/ENO: Query = %d/%.1f, Sbjct = %d/%.1f\n\n", in.query_len, in.query_eno, h.dbprolen,
            h.dbeno);
    appendf(o, " Score = %.2f (%.1f bits),  Expect = %.2g, P-value = %.2g\n", score,
            bit_score(in.sspace, logeval), evalue, pvalue_of(evalue));
    if (idts > 0) appendf(o, " Identities = %d/%d (%d%%)", idts, alnlen, idts * 100 / alnlen);
    if (psts > 0) {
        if (idts) o += ',';
        appendf(o, " Positives = %d/%d (%d%%)", psts, alnlen, psts * 100 / alnlen);
    }
    if (gaps > 0) {
        if (idts || psts) o += ',';
        appendf(o, " Gaps = %d/%d (%d%%)", gaps, alnlen, gaps * 100 / alnlen);
    }
    o += "\n\n";
}

// FormatAlignmentPlain (:250-336)
void alignment_plain(std::string& o, const HitsInput& in, const HitView& h, int width, bool printsss)
{
    const uint32_t beg = ubits(h.r[rBeg]);
    unsigned qrybeg = (beg & 0xffffu) + 1u;
    unsigned trgbeg = ((beg >> 16) & 0xffffu) + 1u;
    printsss = printsss && in.query_ss && h.trgss;
    const int alnlen = h.alnlen;
    for (int f = 0; f < alnlen; f += width) {
        const int nbytes = std::min(width, alnlen - f);
        if (printsss) {
            appendf(o, "%-13s", "struct");
            o.append(h.aln[aQuerySS] + f, (size_t)nbytes);
            put_nl(o);
        }
        {
            const char* p = h.aln[aQuery] + f;
            appendf(o, "Query: %5u ", qrybeg);
            o.append(p, (size_t)nbytes);
            const int fgaps = (int)std::count(p, p + nbytes, '-');
            qrybeg += nbytes - fgaps;
            appendf(o, " %-5d\n", nbytes <= fgaps ? (int)qrybeg : (int)qrybeg - 1);
        }
        appendf(o, "%13c", ' ');
        o.append(h.aln[aMiddle] + f, (size_t)nbytes);
        put_nl(o);
        {
            const char* p = h.aln[aTarget] + f;
            appendf(o, "Sbjct: %5u ", trgbeg);
            o.append(p, (size_t)nbytes);
            const int fgaps = (int)std::count(p, p + nbytes, '-');
            trgbeg += nbytes - fgaps;
            appendf(o, " %-5d\n", nbytes <= fgaps ? (int)trgbeg : (int)trgbeg - 1);
        }
        if (printsss) {
            appendf(o, "%-13s", "struct");
            o.append(h.aln[aTargetSS] + f, (size_t)nbytes);
            put_nl(o);
        }
        put_nl(o);
    }
}

void stat_pair(const HitView& h, float K, float lmbd, char* kbuf, char* lbuf, const char*& kp, const char*& lp,
               const char* na)
{
    kp = lp = na;
    if (h.r[rE] < 0.0f) {
        if (K > 0.0f) {
            std::snprintf(kbuf, kBufMax, "%6.4f", K);
            kp = kbuf;
        }
        if (lmbd > 0.0f) {
            std::snprintf(lbuf, kBufMax, "%6.4f", lmbd);
            lp = lbuf;
        }
    }
}

// FormatFooterPlain (:342-385)
void footer_plain(std::string& o, const HitView& h)
{
    char kbuf[kBufMax], lbuf[kBufMax];
    const char *kp, *lp;
    appendf(o, "%25c  %-6s   %-6s\n", ' ', "K", "Lambda");
    stat_pair(h, h.r[rK], h.r[rLmbd], kbuf, lbuf, kp, lp, "n/a");
    appendf(o, "%-25s  %6s   %6s\n", "Computed  ungapped,", kp, lp);
    stat_pair(h, h.r[rKEst], h.r[rLmbdEst], kbuf, lbuf, kp, lp, "n/a");
    appendf(o, "%-25s  %6s   %6s\n", "Estimated gapped,", kp, lp);
    appendf(o, "Entropy, %6.4f; Expected, %6.4f; Min/Max, %.0f/%-.0f\n\n", h.r[rH], h.r[rE], h.r[rMin],
            h.r[rMax]);
}

// CompressResultsPlain, one hit (:93-147)
void hit_plain(std::string& annot, std::string& rec, const HitsInput& in, const HitView& h,
               const cbp_format_options& fo)
{
    const float logeval = h.r[rLogE];
    const double evalue = evalue_of(logeval);
    const float score = h.r[rScore];
    const char* desc = desc_of(in, h.prof);
    annotation_plain(annot, desc, score, evalue);
    int outpos = 0, linepos = 0;
    const int width = kIndent < fo.dscwidth ? fo.dscwidth : 1;
    if (desc) format_description(rec, desc, fo.dsclen, kIndent, width, outpos, linepos, '>');
    put_nl(rec);
    scores_plain(rec, in, h, score, logeval, evalue);
    alignment_plain(rec, in, h, fo.alnwidth, in.ssswgt > 0.0f);
    if (fo.show) footer_plain(rec, h);
    rec += "\n\n";
}

// ---- JSON (CuBatchProcessingFinalizerJSON.cpp) -------------------------

// MakeAnnotationJSON (:161-187)
void annotation_json(std::string& o, const char* desc, float score, double evalue)
{
    int outpos = 0;
    o += "    {\"summary_entry\": {\n      \"description\": \"";
    if (desc) format_description_json(o, desc, kAnnotLen, outpos);
    o += "\",\n";
    appendf(o, "      \"score\": %.0f,\n      \"evalue\": %.2g\n    }}", score, evalue);
}

// FormatScoresJSON (:197-224)
void scores_json(std::string& o, const HitsInput& in, const HitView& h, float score, float logeval,
                 double evalue)
{
    const int psts = (int)h.r[rPstvs], idts = (int)h.r[rIdnts], gaps = (int)h.r[rNGaps];
    appendf(o,
            "        \"score\": %.2f,\n"
            "        \"bit_score\": %.1f,\n"
            "        \"evalue\": %.2g,\n"
            "        \"pvalue\": %.2g,\n",
            score, bit_score(in.sspace, logeval), evalue, pvalue_of(evalue));
    appendf(o,
            "        \"n_identities\": %d,\n"
            "        \"n_positives\": %d,\n"
            "        \"n_gaps\": %d,\n"
            "        \"aln_length\": %d,\n",
            idts, psts, gaps, h.alnlen);
}

// FormatAlignmentJSON (:236-316); the SS rows are shown whenever both
// profiles carry SS data (SSSWGT is not consulted here)
void alignment_json(std::string& o, const HitsInput& in, const HitView& h)
{
    const uint32_t beg = ubits(h.r[rBeg]);
    const unsigned qrybeg = (beg & 0xffffu) + 1u;
    const unsigned trgbeg = ((beg >> 16) & 0xffffu) + 1u;
    const int nbytes = h.alnlen;
    const int ngapsqry = (int)std::count(h.aln[aQuery], h.aln[aQuery] + nbytes, '-');
    const int ngapstrg = (int)std::count(h.aln[aTarget], h.aln[aTarget] + nbytes, '-');
    const unsigned qryend = qrybeg + nbytes - ngapsqry;
    const unsigned trgend = trgbeg + nbytes - ngapstrg;
    const int printsss = (in.query_ss && h.trgss) ? 1 : 0;
    // the SS rows are filled only with SSSWGT > 0; the reference copies them
    // with strncpy all the same, so an unfilled row ends at its first NUL.
    // Here that is the end of the field (the reference's writer would cut
    // the whole record there, from rows that nothing wrote).
    auto ss_field = [&](const char* p) { o.append(p, strnlen(p, (size_t)nbytes)); };
    appendf(o,
            "        \"query_from\": %u,\n"
            "        \"query_to\": %u,\n"
            "        \"target_from\": %u,\n"
            "        \"target_to\": %u,\n",
            qrybeg, nbytes <= ngapsqry ? qryend : qryend - 1, trgbeg, nbytes <= ngapstrg ? trgend : trgend - 1);
    appendf(o,
            "        \"query_secstr_available\": %d,\n"
            "        \"target_secstr_available\": %d,\n"
            "        \"query_secstr\": \"",
            printsss, printsss);
    if (printsss) ss_field(h.aln[aQuerySS]);
    o += "\",\n        \"target_secstr\": \"";
    if (printsss) ss_field(h.aln[aTargetSS]);
    o += "\",\n        \"query_aln\": \"";
    o.append(h.aln[aQuery], (size_t)nbytes);
    o += "\",\n        \"target_aln\": \"";
    o.append(h.aln[aTarget], (size_t)nbytes);
    o += "\",\n        \"middle\": \"";
    o.append(h.aln[aMiddle], (size_t)nbytes);
    o += "\",\n";
}

// FormatFooterJSON (:322-380)
void footer_json(std::string& o, const HitView& h)
{
    char kbuf[kBufMax], lbuf[kBufMax];
    const char *kp, *lp;
    stat_pair(h, h.r[rK], h.r[rLmbd], kbuf, lbuf, kp, lp, "NA");
    appendf(o,
            "        \"computed_K_ungapped\": \"%s\",\n"
            "        \"computed_lambda_ungapped\": \"%s\",\n",
            kp, lp);
    stat_pair(h, h.r[rKEst], h.r[rLmbdEst], kbuf, lbuf, kp, lp, "NA");
    appendf(o,
            "        \"estimated_K_gapped\": \"%s\",\n"
            "        \"estimated_lambda_gapped\": \"%s\",\n"
            "        \"entropy\": %.4f,\n"
            "        \"expected_score\": %.4f,\n"
            "        \"min_score\": %.0f,\n"
            "        \"max_score\": %.0f\n",
            kp, lp, h.r[rH], h.r[rE], h.r[rMin], h.r[rMax]);
}

// CompressResultsJSON, one hit (:85-148)
void hit_json(std::string& annot, std::string& rec, const HitsInput& in, const HitView& h,
              const cbp_format_options& fo)
{
    const float logeval = h.r[rLogE];
    const double evalue = evalue_of(logeval);
    const float score = h.r[rScore];
    const char* desc = desc_of(in, h.prof);
    annotation_json(annot, desc, score, evalue);
    rec += "    {\"hit_record\": {\n      \"target_description\": \"";
    int outpos = 0;
    if (desc) format_description_json(rec, desc, fo.dsclen, outpos);
    rec += "\",\n";
    appendf(rec,
            "      \"query_length\": %d,\n"
            "      \"query_eno\": %.1f,\n"
            "      \"target_length\": %d,\n"
            "      \"target_eno\": %.1f,\n"
            "      \"alignment\": {\n",
            in.query_len, in.query_eno, h.dbprolen, h.dbeno);
    scores_json(rec, in, h, score, logeval, evalue);
    alignment_json(rec, in, h);
    footer_json(rec, h);
    rec += "      }\n    }}";
}

void check_format_options(const cbp_format_options* fo)
{
    if (!fo) throw FormatError{CBP_ERR_ARG, "null format options"};
    if (fo->format != CBP_FORMAT_PLAIN && fo->format != CBP_FORMAT_JSON)
        throw FormatError{CBP_ERR_ARG, "unknown output format"};
    if (fo->dsclen < 1 || fo->dscwidth < 1 || fo->alnwidth < 1)
        throw FormatError{CBP_ERR_ARG, "description length and widths must be positive"};
}

// the packed records: annotation NUL hit-record NUL, per reported hit
std::string format_hits(const HitsInput& in, const cbp_format_options& fo, size_t* nhits,
                        const int32_t* order = nullptr, size_t norder = 0)
{
    std::string out;
    // the order given (the device's) or the finalizer's, restated
    std::vector<size_t> idx;
    if (order) {
        for (size_t i = 0; i < norder; i++) {
            if (order[i] < 0 || (size_t)order[i] >= in.nrecs)
                throw FormatError{CBP_ERR_ARG, "hit order names a record outside the records"};
            idx.push_back((size_t)order[i]);
        }
    } else {
        idx = reported(in);
    }
    for (size_t k : idx) {
        const HitView h = view_of(in, k);
        std::string annot, rec;
        if (fo.format == CBP_FORMAT_JSON) hit_json(annot, rec, in, h, fo);
        else hit_plain(annot, rec, in, h, fo);
        out += annot;
        out += '\0';
        out += rec;
        out += '\0';
    }
    *nhits = idx.size();
    return out;
}

int deliver(const std::string& s, char* buf, size_t cap, size_t* used)
{
    if (used) *used = s.size();
    if (!buf) return CBP_OK;
    if (cap < s.size()) {
        cbp::set_last_error("output buffer too small: " + std::to_string(s.size()) + " bytes needed");
        return CBP_ERR_LIMIT;
    }
    std::memcpy(buf, s.data(), s.size());
    return CBP_OK;
}

// ---- the writer (AlnWriterPlain.cpp / AlnWriterJSON.cpp) ----------------

// WritePrognamePlain (AlnWriterPlain.cpp:139-185)
void progname_plain(std::string& o, const cbp_report_info& ri, int width)
{
    const size_t start = o.size();
    if (ri.program) appendf(o, "%s", ri.program);
    if (ri.version) appendf(o, " %s", ri.version);
    if (ri.program || ri.version) o += "\n\n";
    const int maxsize = kWriterBuffer - (int)(o.size() - start) - (1 * 3 + 1);
    if (maxsize < 1) return;
    int outpos = 0, linepos = 0;
    for (int i = 0; ri.references && ri.references[i] && outpos < maxsize; i++) {
        format_description(o, ri.references[i], maxsize, 0, width, outpos, linepos, 0);
        outpos += put_nl(o);
        linepos = 0;
    }
    o += '\n';
}

// WriteQueryDescriptionPlain (AlnWriterPlain.cpp:198-240)
void query_plain(std::string& o, int maxsize, const cbp_report_info& ri, int width)
{
    if (maxsize < 40) return;
    const size_t start = o.size();
    appendf(o, "\n Query (%d positions):\n", ri.query_len);
    maxsize -= (int)(o.size() - start);
    if (maxsize < 1) return;
    int outpos = 0, linepos = 0;
    if (ri.query_desc) format_description(o, ri.query_desc, maxsize, 0, width, outpos, linepos, 0);
}

// WriteSearchInformationPlain (AlnWriterPlain.cpp:254-331)
void search_info_plain(std::string& o, const cbp_report_info& ri, bool found)
{
    const int maxsize = kTmpBuffer;
    const size_t maxszname = 100;
    const size_t start = o.size();
    auto size = [&]() { return (int)(o.size() - start); };
    auto over = [&](int delta) {
        if (maxsize < size() + delta) {
            if (size() + 5 < maxsize) o += "...\n\n";
            return true;
        }
        return false;
    };
    if (over(30)) return;
    o += "\n\n Database(s):\n";
    for (size_t d = 0; d < ri.n_db_names; d++) {
        const char* name = ri.db_names[d] ? ri.db_names[d] : "";
        const size_t full = std::strlen(name);
        const size_t szname = std::min(full, maxszname);
        if (over((int)(szname + 2))) return;
        o.append(name, szname);
        if (szname < full && 3 < szname)
            for (int i = 1; i <= 3; i++) o[o.size() - i] = '.';
        put_nl(o);
    }
    if (over(kIndent + 40)) return;
    o.append((size_t)kIndent, ' ');
    appendf(o, "%llu profiles\n", (unsigned long long)ri.db_entries);
    if (over(kIndent + 50)) return;
    o.append((size_t)kIndent, ' ');
    appendf(o, "%llu total positions\n\n\n", (unsigned long long)ri.db_size);
    if (over(kAnnotLen * 2)) return;
    if (found) {
        const char* msg = " Profiles found below the e-value threshold:";
        o += msg;
        for (int w = (int)std::strlen(msg); w < kAnnotLen; w++) o += ' ';
        appendf(o, " %7s %7s\n\n", "Score", "E-value");
    } else {
        appendf(o, " No profiles found below an e-value threshold of %g.\n\n\n", std::exp(ri.log_evalue_threshold));
    }
}

void effective_lengths(const cbp_report_info& ri, int* effq, unsigned long long* effdb)
{
    *effq = ri.query_len;
    *effdb = ri.db_size;
    const long long dl = ri.delta_length;
    if (dl < ri.query_len) *effq -= (int)dl;
    if ((unsigned long long)(ri.db_entries * (unsigned long long)dl) < ri.db_size)
        *effdb -= ri.db_entries * (unsigned long long)dl;
}

// WriteSummaryPlain (AlnWriterPlain.cpp:345-398)
void summary_plain(std::string& o, const cbp_report_info& ri)
{
    int effq;
    unsigned long long effdb;
    effective_lengths(ri, &effq, &effdb);
    appendf(o, "%-20s  %-6s   %-6s\n", "Reference values of", "K", "Lambda");
    appendf(o, "%-20s  %6.4f   %6.4f\n", "Ungapped", ri.ref_k, ri.ref_lambda);
    appendf(o, "%-20s  %6.4f   %6.4f\n\n", "Gapped", ri.gapped_k, ri.gapped_lambda);
    appendf(o, "Length of query, %d\n", ri.query_len);
    appendf(o, "Length of database, %llu\n", (unsigned long long)ri.db_size);
    appendf(o, "Effective length of query, %d\n", effq);
    appendf(o, "Effective length of database, %llu\n", effdb);
    appendf(o, "Effective search space, %llu\n\n", (unsigned long long)(size_t)ri.search_space);
}

// WritePrognameJSON (AlnWriterJSON.cpp:156-208)
void progname_json(std::string& o, const cbp_report_info& ri)
{
    const size_t start = o.size();
    appendf(o, "{\"cother_search\": {\n  \"program\": \"%s\",\n  \"version\": \"%s\",\n",
            ri.program ? ri.program : "", ri.version ? ri.version : "");
    const int maxsize = kWriterBuffer - (int)(o.size() - start) - kKByte;
    if (maxsize < 1) return;
    o += "  \"references\": [\n";
    const int maxlenrefinf = kKByte - 60;
    int totlenref = 0;
    bool bwrt = true;
    static const char* const kNone[1] = {nullptr};
    const char* const* refs = ri.references ? ri.references : kNone;
    for (int i = 0; !i || (bwrt && refs[i]); i++) {
        const char* s = refs[i];
        totlenref += s ? (int)std::strlen(s) : 0;
        bwrt = totlenref < maxlenrefinf;
        appendf(o, "    \"%s\"%s\n", (bwrt && s) ? s : "", (bwrt && s && refs[i + 1]) ? "," : "");
        if (!refs[i]) break;
    }
    o += "  ],\n";
}

// WriteQueryDescriptionJSON (AlnWriterJSON.cpp:219-275)
void query_json(std::string& o, int maxsize, const cbp_report_info& ri)
{
    if (maxsize < 60) return;
    const size_t start = o.size();
    appendf(o, "  \"query\": {\n    \"length\": %d,\n", ri.query_len);
    maxsize -= (int)(o.size() - start) + kBufMax;
    if (maxsize < 1) return;
    const char* nm = "    \"name\": \"";
    o += nm;
    int outpos = (int)std::strlen(nm);
    o += "\",\n";
    outpos += 3;
    const char* ds = "    \"description\": \"";
    o += ds;
    outpos += (int)std::strlen(ds);
    if (ri.query_desc) format_description_json(o, ri.query_desc, maxsize, outpos);
    o += "\"\n  },\n";
}

// WriteSearchInformationJSON (AlnWriterJSON.cpp:287-375)
void search_info_json(std::string& o, const cbp_report_info& ri, bool found)
{
    int maxsize = kTmpBuffer;
    auto over = [&](int delta) {
        maxsize -= delta;
        return maxsize < 1;
    };
    if (over(40 * 7)) return;
    o += "  \"database\": {\n    \"names\": [\n";
    for (size_t d = 0; d < ri.n_db_names; d++) {
        const char* name = ri.db_names[d] ? ri.db_names[d] : "";
        const size_t szname = std::min(std::strlen(name), (size_t)99);
        if (over((int)(szname + 15))) {
            o += "      \"...\"\n";
            break;
        }
        o += "      \"";
        int outpos = 0;
        format_description_json(o, name, (int)szname + 1, outpos);
        o += (d + 1 < ri.n_db_names) ? "\",\n" : "\"\n";
    }
    appendf(o,
            "    ],\n"
            "    \"number_of_profiles\": %llu,\n"
            "    \"number_of_positions\": %llu\n"
            "  },\n",
            (unsigned long long)ri.db_entries, (unsigned long long)ri.db_size);
    if (over(90 * 4)) return;
    if (found)
        o += "  \"message\": \"Profiles found below the e-value threshold:\",\n";
    else
        appendf(o, "  \"message\": \"No profiles found below an e-value threshold of %g\",\n",
                std::exp(ri.log_evalue_threshold));
}

// WriteSummaryJSON (AlnWriterJSON.cpp:389-429)
void summary_json(std::string& o, const cbp_report_info& ri)
{
    int effq;
    unsigned long long effdb;
    effective_lengths(ri, &effq, &effdb);
    appendf(o,
            "  \"search_statistics\": {\n"
            "    \"reference_K_ungapped\": %.4f,\n"
            "    \"reference_lambda_ungapped\": %.4f,\n"
            "    \"reference_K_gapped\": %.4f,\n"
            "    \"reference_lambda_gapped\": %.4f,\n"
            "    \"query_length\": %d,\n"
            "    \"database_size\": %llu,\n"
            "    \"effective_query_length\": %d,\n"
            "    \"effective_database_size\": %llu,\n"
            "    \"effective_search_space\": %llu\n"
            "  }\n}}\n",
            ri.ref_k, ri.ref_lambda, ri.gapped_k, ri.gapped_lambda, ri.query_len,
            (unsigned long long)ri.db_size, effq, effdb, (unsigned long long)(size_t)ri.search_space);
}

// WriteResultsPlain / WriteResultsJSON (AlnWriterPlain.cpp:19-124,
// AlnWriterJSON.cpp:19-145)
std::string write_report(const cbp_report_info& ri, const cbp_format_options& fo, const char* const* annots,
                         const char* const* recs, size_t nhits)
{
    std::string o;
    const bool found = nhits > 0;
    const size_t nh = (size_t)std::max(ri.nohits, 0), na = (size_t)std::max(ri.noalns, 0);
    if (fo.format == CBP_FORMAT_PLAIN) {
        progname_plain(o, ri, fo.dscwidth);
        const int left = std::min(kWriterBuffer - (int)o.size(), fo.dsclen);
        query_plain(o, left, ri, fo.dscwidth);
        search_info_plain(o, ri, found);
        if (found) {
            for (size_t i = 0; i < nhits && i < nh; i++) o += annots[i];
            o += "\n\n\n";
            for (size_t i = 0; i < nhits && i < na; i++) o += recs[i];
        }
        summary_plain(o, ri);
    } else {
        progname_json(o, ri);
        const int left = std::min(kWriterBuffer - (int)o.size(), fo.dsclen);
        query_json(o, left, ri);
        search_info_json(o, ri, found);
        o += "  \"search_summary\": [\n";
        if (found) {
            for (size_t i = 0; i < nhits && i < nh; i++) {
                o += annots[i];
                const bool last = !(i + 1 < nhits && i + 1 < nh);
                o += last ? "\n" : ",\n";
            }
        }
        o += "  ],\n  \"search_hits\": [\n";
        if (found) {
            // the reference ends this list by NOHITS as well
            for (size_t i = 0; i < nhits && i < na; i++) {
                o += recs[i];
                const bool last = !(i + 1 < nhits && i + 1 < nh);
                o += last ? "\n" : ",\n";
            }
        }
        o += "  ],\n";
        summary_json(o, ri);
    }
    return o;
}

template <class F>
int guarded_fmt(F&& f)
{
    try {
        const int rc = f();
        if (rc == CBP_OK) cbp::set_last_error("");
        return rc;
    } catch (const FormatError& e) {
        cbp::set_last_error(e.msg);
        return e.code;
    } catch (const std::exception& e) {
        cbp::set_last_error(e.what());
        return CBP_ERR_ARG;
    }
}

}  // namespace

// used by api.cu for the context's own results
namespace cbp {
int format_hits_from(const float* recs, size_t nrecs, const int32_t* order, size_t norder, const char* rows,
                     size_t row_stride, size_t row_length,
                     const int* prof_len, const float* prof_eno, const uint8_t* prof_ss, size_t nprof,
                     const char* const* descs, int query_len, float query_eno, int query_ss, float ssswgt,
                     float logevthld, float sspace, const cbp_format_options* fo, char* buf, size_t cap,
                     size_t* used, size_t* nhits)
{
    return guarded_fmt([&] {
        check_format_options(fo);
        HitsInput in{recs, nrecs, rows, row_stride, row_length, prof_len, prof_eno, prof_ss, nprof,
                     descs, query_len, query_eno, query_ss, ssswgt, logevthld, sspace};
        size_t n = 0;
        const std::string s = format_hits(in, *fo, &n, order, norder);
        if (nhits) *nhits = n;
        return deliver(s, buf, cap, used);
    });
}
}  // namespace cbp

extern "C" {

void cbp_default_format_options(cbp_format_options* fo)
{
    if (!fo) return;
    fo->format = CBP_FORMAT_PLAIN;
    fo->dsclen = 1024;
    fo->dscwidth = 80;
    fo->alnwidth = 60;
    fo->show = 1;
}

int cbp_format_hits_host(const cbp_hits_input* in, const cbp_format_options* fo, char* buf, size_t cap,
                         size_t* used, size_t* nhits)
{
    if (!in || (in->nrecs && (!in->recs || !in->rows || !in->prof_len || !in->prof_eno))) {
        cbp::set_last_error("cbp_format_hits_host: null input");
        return CBP_ERR_ARG;
    }
    return cbp::format_hits_from(in->recs, in->nrecs, nullptr, 0, in->rows, in->row_stride, in->row_length, in->prof_len,
                                 in->prof_eno, in->prof_ss, in->nprof, in->descs, in->query_len, in->query_eno,
                                 in->query_ss, in->ssswgt, in->log_evalue_threshold, in->search_space, fo, buf,
                                 cap, used, nhits);
}

int cbp_merge_hit_lists(size_t nparts, const float* const* log_evalues, const size_t* counts, int32_t* part,
                        int32_t* index)
{
    return guarded_fmt([&] {
        if (nparts && (!log_evalues || !counts)) throw FormatError{CBP_ERR_ARG, "null part lists"};
        std::vector<std::pair<int32_t, int32_t>> merged;
        for (size_t p = 0; p < nparts; p++) {
            if (counts[p] && !log_evalues[p]) throw FormatError{CBP_ERR_ARG, "null log E-values of a part"};
            std::vector<std::pair<int32_t, int32_t>> next(merged.size() + counts[p]);
            std::vector<std::pair<int32_t, int32_t>> add(counts[p]);
            for (size_t i = 0; i < counts[p]; i++) add[i] = {(int32_t)p, (int32_t)i};
            auto le = [&](const std::pair<int32_t, int32_t>& a) { return log_evalues[a.first][a.second]; };
            std::merge(merged.begin(), merged.end(), add.begin(), add.end(), next.begin(),
                       [&](const std::pair<int32_t, int32_t>& a, const std::pair<int32_t, int32_t>& b) {
                           return le(a) < le(b);
                       });
            merged.swap(next);
        }
        for (size_t i = 0; i < merged.size(); i++) {
            if (part) part[i] = merged[i].first;
            if (index) index[i] = merged[i].second;
        }
        return CBP_OK;
    });
}

int cbp_write_report(const cbp_report_info* info, const cbp_format_options* fo, const char* const* annotations,
                     const char* const* hit_records, size_t nhits, char* buf, size_t cap, size_t* used)
{
    return guarded_fmt([&] {
        check_format_options(fo);
        if (!info) throw FormatError{CBP_ERR_ARG, "null report information"};
        if (nhits && (!annotations || !hit_records)) throw FormatError{CBP_ERR_ARG, "null hit texts"};
        if (info->n_db_names && !info->db_names) throw FormatError{CBP_ERR_ARG, "null database names"};
        for (size_t i = 0; i < nhits; i++)
            if (!annotations[i] || !hit_records[i]) throw FormatError{CBP_ERR_ARG, "null hit text"};
        return deliver(write_report(*info, *fo, annotations, hit_records, nhits), buf, cap, used);
    });
}

}  // extern "C"
