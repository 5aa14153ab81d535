/*
 * CPU oracle for the COTHER search path -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the rules. Compiled with -ffp-contract=off.
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------
 * orc_logf: natural logarithm of a positive finite float.
 *
 * Not a restatement of any library routine: x = m * 2^e with m in
 * [sqrt(1/2), sqrt(2)), t = (m-1)/(m+1) and log(m) = 2*atanh(t) summed as
 * the odd power series 2(t + t^3/3 + ... + t^9/9) (|t| <= 0.1716, the next
 * term is below 1e-9 relative). Every operation is an IEEE single-precision
 * add, multiply, divide or fused multiply-add, so the CUDA kernels compute
 * bit-identical values with the same sequence.
 * The reference takes __logf() of the same argument
 * (src/libmycu/cusco/CuBatchScoreMatrix_Init.cu:180).
 */
float orc_logf(float x)
{
    union { float f; uint32_t u; } v = {x};
    int e = 0;
    if (v.u < 0x00800000u) {          /* subnormal: scale by 2^23 */
        v.f = x * 8388608.0f;
        e = -23;
    }
    e += (int)((v.u >> 23) & 0xffu) - 127;
    v.u = (v.u & 0x007fffffu) | 0x3f800000u;  /* m in [1,2) */
    float m = v.f;
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float t = (m - 1.0f) / (m + 1.0f);
    float t2 = t * t;
    float p = fmaf(t2, 0.11111111f, 0.14285715f);
    p = fmaf(t2, p, 0.2f);
    p = fmaf(t2, p, 0.33333334f);
    float t2x = t + t;
    float lm = fmaf(t2x * t2, p, t2x);
    float fe = (float)e;
    return fmaf(fe, 0.693145751953125f, fmaf(fe, 1.42860677e-06f, lm));
}

/* ------------------------------------------------------------------------
 * DDMS pair score with the two-level linear interpolation of the reference
 * (src/libmycu/cupro/SerializedDstMatchScores.cuh:347-396, constants
 * src/libmycu/cupro/SerializedDstMatchScoresAttr.h:29-31 and
 * SerializedDstMatchScores.cuh:19-20): distances saturate at 20
 * (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:60), 255 scores -1;
 * with d1 >= d2: score = d1*slope + (0.35 - (d2*(-0.4))*0.05),
 * slope = (-0.4-0.35)*0.05. The reference's CUDA build contracts both
 * multiply-adds (nvcc's default --fmad=true): the intercept is
 * fma(-(d2*-0.4), 0.05, 0.35) and the score fma(d1, slope, intercept),
 * which its own CPU table (cother-scores-optimizer/dstable.h:339-365)
 * rounds separately; the GPU form is the one followed here.
 */
static float orc_dms_pair_score_ex(int d1, int d2, int fused)
{
    if (d1 == 0xff || d2 == 0xff) return -1.0f;
    if (d1 > 20) d1 = 20;
    if (d2 > 20) d2 = 20;
    if (d1 < d2) { int t = d1; d1 = d2; d2 = t; }
    float b = (float)d2 * -0.4f;
    float slope = (-0.4f - 0.35f) * 0.05f;
    if (!fused) {
        float intpt = 0.35f - b * 0.05f;
        float prod = (float)d1 * slope;
        return prod + intpt;
    }
    float intpt = fmaf(-b, 0.05f, 0.35f);
    return fmaf((float)d1, slope, intpt);
}

float orc_dms_pair_score(int d1, int d2)
{
    return orc_dms_pair_score_ex(d1, d2, 1);
}

/* ------------------------------------------------------------------------
 * Top-3 non-intersecting segment register
 * (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s.cuh:114-251).
 * Coordinates are packed [QB QE PB PE], one byte each.
 */
#define ORC_COORDS(QB, QE, PB, PE) \
    ((((uint32_t)(QB) & 0xffu) << 24) | (((uint32_t)(QE) & 0xffu) << 16) | \
     (((uint32_t)(PB) & 0xffu) << 8) | ((uint32_t)(PE) & 0xffu))

static int orc_coords_intersect(uint32_t c1, uint32_t c2)
{
    uint32_t mx = 0, mn = 0;
    for (int b = 0; b < 32; b += 8) {
        uint32_t x = (c1 >> b) & 0xffu, y = (c2 >> b) & 0xffu;
        mx |= (x > y ? x : y) << b;
        mn |= (x < y ? x : y) << b;
    }
    return ((mn >> 16) & 0xffu) >= ((mx >> 24) & 0xffu) ||
           (mn & 0xffu) >= ((mx >> 8) & 0xffu);
}

static void orc_register_max(float* ms, uint32_t* mc, float segsco, uint32_t segcoords)
{
    if (segsco == 0.0f) return;
    if (ms[0] <= segsco) {
        ms[2] = ms[1]; mc[2] = mc[1];
        ms[1] = ms[0]; mc[1] = mc[0];
        ms[0] = segsco; mc[0] = segcoords;
        if (ms[1] != 0.0f && orc_coords_intersect(mc[0], mc[1])) ms[1] = 0.0f;
        if (ms[2] != 0.0f && orc_coords_intersect(mc[0], mc[2])) ms[2] = 0.0f;
        if (ms[1] == 0.0f) {
            ms[1] = ms[2]; mc[1] = mc[2];
            ms[2] = 0.0f;
        }
    } else if (ms[1] <= segsco) {
        if (orc_coords_intersect(segcoords, mc[0])) return;
        ms[2] = ms[1]; mc[2] = mc[1];
        ms[1] = segsco; mc[1] = segcoords;
        if (orc_coords_intersect(mc[1], mc[2])) ms[2] = 0.0f;
    } else if (ms[2] <= segsco) {
        if (orc_coords_intersect(segcoords, mc[0]) || orc_coords_intersect(segcoords, mc[1]))
            return;
        ms[2] = segsco; mc[2] = segcoords;
    }
}

static inline float orc_hmax(float a, float b) { return a < b ? b : a; }

/* list value at 1-based slot k; slots past the count read as no data
 * (the reference pads its shared-memory copy with 0xff:
 * src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:91-104) */
static inline int orc_lv(const uint8_t* lst, int k)
{
    int n = lst[0];
    if (k > n || k >= ORC_NDSTSLOTS) return 0xff;
    return lst[k];
}

static inline float orc_S(const uint8_t* q, int kq, const uint8_t* d, int kd, int fused)
{
    return orc_dms_pair_score_ex(orc_lv(q, kq), orc_lv(d, kd), fused);
}

/* Upper part: diagonal j of the DP over the two lists
 * (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:288-340, segment
 * update :124-147, unrolled reads :184-198). */
static void orc_diag_upper(const uint8_t* q, const uint8_t* d, int dstsegm, int len1, int len2,
                           int j, float* ms, uint32_t* mc, int fused)
{
    float segsco;
    int segqb = 0, segpb = j;
    float s[5];
    s[0] = orc_S(q, 1, d, j + 1, fused);
    segsco = orc_hmax(s[0], 0.0f);
    for (int i = 0; i < len1 && j + i < len2; i += 4) {
        float scom = 0.0f;
        int im = 0, jim = 0, ib = 0, jib = 0;
        s[2] = orc_S(q, i + 3, d, j + i + 3, fused);
        s[4] = orc_S(q, i + 5, d, j + i + 5, fused);
        s[3] = 0.5f * (s[2] + s[4]);
        s[1] = 0.5f * (s[0] + s[2]);
        for (int k = 1; k <= 4; k++) {
            if (segsco == 0.0f) { segqb = i + k; segpb = j + i + k; }
            segsco = orc_hmax(segsco + s[k], 0.0f);
            if (segsco != 0.0f) {
                if (scom < segsco && dstsegm <= i + k - segqb + 1) {
                    scom = segsco;
                    im = i + k; jim = j + i + k;
                    ib = segqb; jib = segpb;
                }
            }
        }
        orc_register_max(ms, mc, scom, ORC_COORDS(ib, im, jib, jim));
        s[0] = s[4];
    }
}

/* Lower part: diagonal i (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:345-396,
 * segment update :153-176). */
static void orc_diag_lower(const uint8_t* q, const uint8_t* d, int dstsegm, int len1, int len2,
                           int i, float* ms, uint32_t* mc, int fused)
{
    float segsco;
    int segqb = i, segpb = 0;
    float s[5];
    s[0] = orc_S(q, i + 1, d, 1, fused);
    segsco = orc_hmax(s[0], 0.0f);
    for (int j = 0; j < len2 && i + j < len1; j += 4) {
        float scom = 0.0f;
        int ijm = 0, jm = 0, ijb = 0, jb = 0;
        s[2] = orc_S(q, i + j + 3, d, j + 3, fused);
        s[4] = orc_S(q, i + j + 5, d, j + 5, fused);
        s[3] = 0.5f * (s[2] + s[4]);
        s[1] = 0.5f * (s[0] + s[2]);
        for (int k = 1; k <= 4; k++) {
            if (segsco == 0.0f) { segqb = i + j + k; segpb = j + k; }
            segsco = orc_hmax(segsco + s[k], 0.0f);
            if (segsco != 0.0f) {
                if (scom < segsco && dstsegm <= j + k - segpb + 1) {
                    scom = segsco;
                    ijm = i + j + k; jm = j + k;
                    ijb = segqb; jb = segpb;
                }
            }
        }
        orc_register_max(ms, mc, scom, ORC_COORDS(ijb, ijm, jb, jm));
        s[0] = s[4];
    }
}

/* DDMS for one cell (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:433-500):
 * band of diagonals j = len2>>2 .. 0 step 2 (upper), i = len1>>2 .. 1 step 2
 * (lower); score = (0.053*16*sum + (-1.235)) * DDMSWGT. */
float orc_ddms_cell(const uint8_t* qlist, const uint8_t* dlist, int dstsegm,
                    float ddmswgt, float* rawsum, int* computed)
{
    return orc_ddms_cell_ex(qlist, dlist, dstsegm, ddmswgt, 1, rawsum, computed);
}

float orc_ddms_cell_ex(const uint8_t* qlist, const uint8_t* dlist, int dstsegm,
                       float ddmswgt, int fused, float* rawsum, int* computed)
{
    int len1 = qlist[0], len2 = dlist[0];
    *rawsum = 0.0f;
    *computed = 0;
    if (len1 < dstsegm || len2 < dstsegm) return 0.0f;
    *computed = 1;
    float ms[3] = {0.0f, 0.0f, 0.0f};
    uint32_t mc[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
    for (int j = len2 >> 2; 0 <= j; j -= 2)
        orc_diag_upper(qlist, dlist, dstsegm, len1, len2, j, ms, mc, fused);
    for (int i = len1 >> 2; 0 < i; i -= 2)
        orc_diag_lower(qlist, dlist, dstsegm, len1, len2, i, ms, mc, fused);
    float sum = 0.0f;
    for (int k = 0; k < 3; k++) sum = sum + ms[k];
    *rawsum = sum;
    const float slope = 0.053f * 16.0f;
    float sc = fmaf(slope, sum, -1.235f);
    return sc * ddmswgt;
}

/* ------------------------------------------------------------------------
 * Profile-profile score (src/libmycu/cusco/CuBatchScoreMatrix_Init.cu:159-186):
 * log( sum_a q_tf[a]*d_tf[a] / (0.5*(q_bkg[a]+d_bkg[a])) ) - shift.
 * SS score (src/libmycu/cusco/CuBatchScoreMatrix_ssss.cu:209-279,
 * table index CuBatchScoreMatrix_ssss.cuh:26-31).
 */
static float orc_init_score(const float* qtf, long long qstride, const float* qbk,
                            const float* dtf, long long dstride, const float* dbk, long long bstride,
                            float shift)
{
    float acc = 0.0f;
    for (int a = 0; a < 20; a++) {
        float num = qtf[a * qstride] * dtf[a * dstride];
        float den = 0.5f * (qbk[a] + dbk[a * bstride]);
        acc = acc + num / den;
    }
    return orc_logf(acc) - shift;
}

static float orc_ss_score(const float* qss, long long qstride, const float* dss, long long dstride,
                          const float* T, float ssswgt)
{
    float acc = 0.0f;
    for (int i = 0; i < 3; i++) {
        float f1 = qss[i * qstride];
        int r = i * 10 + (int)(f1 * 9.999f);
        for (int j = 0; j < 3; j++) {
            float f2 = dss[j * dstride];
            int c = j * 10 + (int)(f2 * 9.999f);
            acc = fmaf(f1 * f2, T[r * ORC_NOTABLE_SS + c], acc);
        }
    }
    float f1 = qss[2 * qstride], f2 = dss[2 * dstride];
    if (-99.0f < acc) {
        acc = fmaf((f1 + 0.1f) * (f2 + 0.1f), 0.1111111f, acc);
        acc = acc - 0.05f;
        acc = acc * ssswgt;
    }
    return acc;
}

/* Context-vector score constants (_TCTXVECT::_TCTXVECT,
 * src/libpro/srcpro/TCTXVECT.cpp:26-60): dimension 19, kappa0 0.1, nu0 19;
 * lokappa0 = 1/kappa0, pownu0 = -(nu0+2)/2 and
 * cterm = (dim/2 + pownu0)(ln kappa0 - ln(kappa0+2)) + sum_{i=1..dim} (ln(nu0+1-i) - ln 2),
 * in float with the C library's logf as the reference's host code. */
void orc_cvs_constants(float* lokappa0, float* pownu0, float* cterm)
{
    const int dim = 19;
    const float kappa0 = 0.1f;
    const float nu0 = (float)dim;
    const float pw = -0.5f * (nu0 + 2.f);
    float ct = (0.5f * dim + pw) * (logf(kappa0) - logf(kappa0 + 2.f));
    float sum = 0.0f;
    for (int i = 1; i <= dim; i++) sum += logf(nu0 + 1.0f - i) - 0.69314718055994530941723212146f;
    ct += sum;
    *lokappa0 = 1.f / kappa0;
    *pownu0 = pw;
    *cterm = ct;
}

float orc_cvs_lookup(const orc_score_params* prm, float lo)
{
    if (!(prm->cvs_key_first < lo)) return prm->cvs_scores[0];   /* NaN too */
    if (prm->cvs_key_last <= lo) return prm->cvs_scores[prm->cvs_card - 1];
    return prm->cvs_scores[prm->cvs_shift + (int)rintf(lo + lo)];
}

/* The map value of cell (r, c) (CalcCVS2ScoreSMEMUnroll2x,
 * src/libmycu/cusco/CuBatchScoreMatrix_cvs2s.cuh:47-136): the log-odds of
 * the two normal vectors, log det(C2 + H'H) from their dot product and
 * squared norms, less both log priors, translated through the map. The dot
 * product, the determinant and the log-odds are contracted into fused
 * multiply-adds as the reference's CUDA build does. The reference takes the logarithm with
 * the fast intrinsic __logf (at most 3 ulp from the true value here, since
 * the determinant is at least 21); this restatement uses logf, and flags
 * the cell when the lookup would change within 8 ulp of the logarithm. */
static float orc_cvs_cell(const orc_score_params* prm, long long r, long long Lq, long long c,
                          long long N, float lokappa0, float pownu0, float cterm, int* ambiguous)
{
    float dot = 0.0f;
    for (int i = 0; i < 19; i++)
        dot = fmaf(prm->q_cv[i * Lq + r], prm->d_cv[i * N + c], dot);
    dot = dot + lokappa0;
    const float a = prm->q_cvnorm2[r] + 1.0f + lokappa0;
    const float b = prm->d_cvnorm2[c] + 1.0f + lokappa0;
    const float det = fmaf(a, b, -(dot * dot));
    const float lg = logf(det);
    float qp = prm->q_cvprior[r], dp = prm->d_cvprior[c];
    if (prm->cvs_int_priors) { qp = (float)(int)qp; dp = (float)(int)dp; }
    const float lo = fmaf(pownu0, lg, cterm) - qp - dp;
    const float v = orc_cvs_lookup(prm, lo);
    if (ambiguous) {
        const float d8 = 8.0f * (nextafterf(fabsf(lg), INFINITY) - fabsf(lg));
        const float lo1 = fmaf(pownu0, lg - d8, cterm) - qp - dp;
        const float lo2 = fmaf(pownu0, lg + d8, cterm) - qp - dp;
        *ambiguous = orc_cvs_lookup(prm, lo1) != v || orc_cvs_lookup(prm, lo2) != v;
    }
    return v;
}

void orc_score_matrix(int Lq, const float* q_tf, const float* q_bkg, const float* q_ss,
                      const uint8_t* q_dd,
                      long long N, int P, const float* d_tf, const float* d_bkg,
                      const int32_t* d_pro, const float* d_ss, const uint8_t* d_dd,
                      const float* ss_table, const orc_score_params* prm,
                      long long col0, long long ncols,
                      float* scores, float* modscores, long long ld)
{
    float lokappa0 = 0.f, pownu0 = 0.f, cterm = 0.f;
    const int cvs = prm->cvswgt > 0.0f;
    if (cvs) orc_cvs_constants(&lokappa0, &pownu0, &cterm);
    for (int r = 0; r < Lq; r++) {
        for (long long c = col0; c < col0 + ncols; c++) {
            int p = d_pro[c];
            float s = orc_init_score(q_tf + r, Lq, q_bkg, d_tf + c, N, d_bkg + p, P, prm->initshift);
            float ms = 0.0f;
            int amb = 0;
            const float cv = cvs ? orc_cvs_cell(prm, r, Lq, c, N, lokappa0, pownu0, cterm,
                                                prm->cvs_ambiguous ? &amb : NULL)
                                 : 0.0f;
            if (prm->cvs_ambiguous) prm->cvs_ambiguous[(size_t)r * ld + (c - col0)] = (uint8_t)amb;
            if (prm->ssswgt > 0.0f) {
                /* SS, plus the weighted CVS term in one addition
                 * (CuBatchScoreMatrix_ssss_cvs2s.cu:252-270); the modular
                 * score drops 0.5*CVSWGT */
                float ss = orc_ss_score(q_ss + r, Lq, d_ss + c, N, ss_table, prm->ssswgt);
                if (cvs) {
                    /* the reference kernel computes two columns per thread,
                     * c and c+32 of each 64-column block of the chunk, and its
                     * build fuses the addition for the first (one rounding)
                     * but not for the second (the product rounded first) */
                    ss = ((c >> 5) & 1) ? ss + cv * prm->cvswgt : fmaf(cv, prm->cvswgt, ss);
                    s = s + ss;
                    ms = ss - 0.5f * prm->cvswgt;
                } else {
                    s = s + ss;
                    ms = ss;
                }
            } else if (cvs && cv != 0.0f) {
                /* CVS alone (CuBatchScoreMatrix_cvs2s.cu:286-299), added
                 * to a modular score that starts at zero */
                s = s + cv * prm->cvswgt;
                ms = ms + (cv - 0.5f) * prm->cvswgt;
            }
            if (prm->ddmswgt > 0.0f) {
                float raw; int comp;
                float dm = orc_ddms_cell(q_dd + (size_t)r * ORC_NDSTSLOTS,
                                         d_dd + (size_t)c * ORC_NDSTSLOTS,
                                         prm->dstsegm, prm->ddmswgt, &raw, &comp);
                if (comp && dm != 0.0f) {
                    /* modular score: dm - 0.2*DDMSWGT, contracted as the
                     * reference's kernel is (CuBatchScoreMatrix_ddms2s_h2.cu:171) */
                    s = s + dm;
                    ms = ms + fmaf(-0.2f, prm->ddmswgt, dm);
                }
            }
            scores[(size_t)r * ld + (c - col0)] = s;
            modscores[(size_t)r * ld + (c - col0)] = ms;
        }
    }
}

typedef struct {
    int Lq; const float *q_tf, *q_bkg, *q_ss; const uint8_t* q_dd;
    long long N; int P; const float *d_tf, *d_bkg; const int32_t* d_pro;
    const float* d_ss; const uint8_t* d_dd; const float* ss_table;
    const orc_score_params* prm; long long c0, nc; float *scores, *modscores;
    long long ld, off;
} orc_sm_job;

static void* orc_sm_thread(void* arg)
{
    orc_sm_job* j = (orc_sm_job*)arg;
    orc_score_params prm = *j->prm;   /* the flag output starts at this job's columns */
    if (prm.cvs_ambiguous) prm.cvs_ambiguous += j->off;
    orc_score_matrix(j->Lq, j->q_tf, j->q_bkg, j->q_ss, j->q_dd, j->N, j->P, j->d_tf, j->d_bkg,
                     j->d_pro, j->d_ss, j->d_dd, j->ss_table, &prm, j->c0, j->nc,
                     j->scores + j->off, j->modscores + j->off, j->ld);
    return NULL;
}

void orc_score_matrix_mt(int nthreads, int Lq, const float* q_tf, const float* q_bkg,
                         const float* q_ss, const uint8_t* q_dd,
                         long long N, int P, const float* d_tf, const float* d_bkg,
                         const int32_t* d_pro, const float* d_ss, const uint8_t* d_dd,
                         const float* ss_table, const orc_score_params* prm,
                         long long col0, long long ncols,
                         float* scores, float* modscores, long long ld)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    orc_sm_job jobs[256];
    long long per = (ncols + nthreads - 1) / nthreads;
    int nt = 0;
    for (int t = 0; t < nthreads; t++) {
        long long a = (long long)t * per, b = a + per;
        if (b > ncols) b = ncols;
        if (a >= b) break;
        orc_sm_job j = {Lq, q_tf, q_bkg, q_ss, q_dd, N, P, d_tf, d_bkg, d_pro, d_ss, d_dd,
                        ss_table, prm, col0 + a, b - a, scores, modscores, ld, a};
        jobs[nt] = j;
        pthread_create(&th[nt], NULL, orc_sm_thread, &jobs[nt]);
        nt++;
    }
    for (int t = 0; t < nt; t++) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------
 * Phase-1 DP.
 * Corner triangles (src/libmycu/cudp/CuBatchDP_init_btck.cuh:117-170): with
 * edge = min(60, rint(0.34*max(Lq,Ld))) the cells with
 * (Lq <= r+edge && c <= edge+r-Lq) or (Ld-edge+r <= c && r < edge) score -9
 * (CuBatchDP_init_btck.cu:230-245). States outside the matrix are 0
 * (DPLocInitCache, CuBatchDP_init.cuh:186-206).
 */
enum { ORC_MM = 0, ORC_MI, ORC_MD, ORC_IM, ORC_II, ORC_DM, ORC_DD };
enum { ORC_STOP = 0, ORC_LEFT = 1, ORC_UP = 2, ORC_DIAG = 3 };
/* log of zero probability in the reference's DP (CuBatchDP_init.cuh:35-38) */
#define ORC_LOG0 (-32768.0f)

static int orc_corner_edge(int Lq, int Ld)
{
    int mx = Lq > Ld ? Lq : Ld;
    int e = (int)rintf(0.34f * (float)mx);
    return e > 60 ? 60 : e;
}

static int orc_in_corner(int Lq, int Ld, int edge, int r, int c)
{
    return (Lq <= r + edge && c <= edge + r - Lq) || (Ld - edge + r <= c && r < edge);
}

float orc_dp1_profile(int Lq, int Ld, const float* S, long long lds,
                      const float* qtrn, long long qts, const float* dtrn, long long dts,
                      uint8_t* btck, int* maxr, int* maxc)
{
    const int edge = orc_corner_edge(Lq, Ld);
    /* previous row (r-1) and current row (r) states, index c+1 (0 = boundary) */
    size_t w = (size_t)Ld + 1;
    float* prv = (float*)calloc(5 * w, sizeof(float));
    float* cur = (float*)calloc(5 * w, sizeof(float));
    float best = 0.0f;
    int br = 0, bc = 0;
#define PMM(a, c) a[0 * w + (c)]
#define PMI(a, c) a[1 * w + (c)]
#define PIM(a, c) a[2 * w + (c)]
#define PDN(a, c) a[3 * w + (c)]
#define PND(a, c) a[4 * w + (c)]
    float dnv = 0.0f;   /* DN of the column -1 cell of the previous row */
    for (int r = 0; r < Lq; r++) {
        const float qMMp = qtrn[ORC_MM * qts + r], qIMp = qtrn[ORC_IM * qts + r];
        const float qDMp = qtrn[ORC_DM * qts + r], qMDp = qtrn[ORC_MD * qts + r];
        const float qDDp = qtrn[ORC_DD * qts + r];
        const float qMIc = qtrn[ORC_MI * qts + r + 1], qIIc = qtrn[ORC_II * qts + r + 1];
        /* column -1 (left boundary), as the reference's block schedule
         * leaves it (src/libmycu/cudp/CuBatchDP_init_btck.cu:93-160,
         * 190-300): within each band of 32 rows, the leftmost block
         * diagonal starts 32 columns left of the profile, and its threads
         * there compute cells with log-zero profile transitions
         * (CuBatchDP_init.cuh:35-38, -32768) and score -9: MM = 0,
         * MI = IM = ND ~ -32768, DN = max(qMD(r), DN(r-1) + qDD(r)) from
         * max(qMD, qDD) on the band's first row (zeros above it). The
         * band's last row starts the next block diagonal at column 0 with
         * zero-initialised predecessors, and the first row's diagonal
         * predecessor lies in the zeroed bottom cache. */
        if ((r & 31) == 31) {
            for (int k = 0; k < 5; k++) { cur[k * w] = 0.0f; prv[k * w] = 0.0f; }
        } else {
            float up_dn = ((r & 31) == 0) ? 0.0f : dnv;
            dnv = orc_hmax(0.0f + qMDp, up_dn + qDDp);
            cur[0 * w] = 0.0f;
            cur[1 * w] = ORC_LOG0;
            cur[2 * w] = ORC_LOG0;
            cur[3 * w] = dnv;
            cur[4 * w] = ORC_LOG0;
        }
        for (int c = 0; c < Ld; c++) {
            const float dMMp = dtrn[ORC_MM * dts + c], dIMp = dtrn[ORC_IM * dts + c];
            const float dDMp = dtrn[ORC_DM * dts + c], dMDp = dtrn[ORC_MD * dts + c];
            const float dDDp = dtrn[ORC_DD * dts + c];
            const float dMIc = dtrn[ORC_MI * dts + c + 1], dIIc = dtrn[ORC_II * dts + c + 1];
            float sc = orc_in_corner(Lq, Ld, edge, r, c) ? -9.0f : S[(size_t)r * lds + c];
            float v1, v2, mx;
            int b = ORC_STOP;
            /* MM from the diagonal predecessor */
            v1 = PMI(prv, c) + qMMp + dIMp;
            v2 = PIM(prv, c) + qIMp + dMMp;
            v1 = orc_hmax(v1, v2);
            v2 = PDN(prv, c) + qDMp + dMMp;
            v1 = orc_hmax(v1, v2);
            v2 = PND(prv, c) + qMMp + dDMp;
            v1 = orc_hmax(v1, v2);
            v2 = PMM(prv, c) + qMMp + dMMp;
            v1 = orc_hmax(v1, v2);
            v1 = orc_hmax(v1 + sc, 0.0f);
            mx = v1;
            if (mx != 0.0f) b = ORC_DIAG;
            PMM(cur, c + 1) = v1;
            if (best < v1) { best = v1; br = r; bc = c; }
            /* MI from above */
            v1 = PMM(prv, c + 1) + qMMp + dMIc;
            v2 = PMI(prv, c + 1) + qMMp + dIIc;
            v1 = orc_hmax(v1, v2);
            PMI(cur, c + 1) = v1;
            if (mx < v1) { mx = v1; b = ORC_UP; }
            /* IM from the left */
            v1 = PMM(cur, c) + qMIc + dMMp;
            v2 = PIM(cur, c) + qIIc + dMMp;
            v1 = orc_hmax(v1, v2);
            PIM(cur, c + 1) = v1;
            if (mx < v1) { mx = v1; b = ORC_LEFT; }
            /* DN from above */
            v1 = PMM(prv, c + 1) + qMDp;
            v2 = PDN(prv, c + 1) + qDDp;
            v1 = orc_hmax(v1, v2);
            PDN(cur, c + 1) = v1;
            if (mx < v1) { mx = v1; b = ORC_UP; }
            /* ND from the left */
            v1 = PMM(cur, c) + dMDp;
            v2 = PND(cur, c) + dDDp;
            v1 = orc_hmax(v1, v2);
            PND(cur, c + 1) = v1;
            if (mx < v1) { mx = v1; b = ORC_LEFT; }
            btck[(size_t)r * Ld + c] = (uint8_t)b;
        }
        float* t = prv; prv = cur; cur = t;
    }
#undef PMM
#undef PMI
#undef PIM
#undef PDN
#undef PND
    free(prv);
    free(cur);
    *maxr = br;
    *maxc = bc;
    return best;
}

/* xor-butterfly warp sum (src/libmycu/cudp/CuBatchDP_final.cu:224-228):
 * after the offsets 16,8,4,2,1 every lane holds the same value; lane 0's
 * evaluation order is reproduced here. */
static float orc_butterfly_sum32(const float* v)
{
    float a[32], b[32];
    for (int t = 0; t < 32; t++) a[t] = v[t];
    for (int off = 16; off >= 1; off >>= 1) {
        for (int t = 0; t < 32; t++) b[t] = a[t] + a[t ^ off];
        for (int t = 0; t < 32; t++) a[t] = b[t];
    }
    return a[0];
}

int orc_dp1_finalize(int Lq, int Ld, const float* S, long long lds, const uint8_t* btck,
                     float maxsc, int maxr, int maxc, float thld,
                     float* out_score, float* out_psts, uint32_t* beg, uint32_t* end)
{
    (void)Lq;
    *out_score = maxsc;
    *out_psts = 0.0f;
    *beg = *end = 0;
    if (maxsc <= thld) return 0;
    float win[36];
    for (int k = 0; k < 36; k++) win[k] = 0.0f;
    int x = maxc, y = maxr, psts = 0, b = ORC_DIAG;
    float sumcorr = 0.0f;
    while (b != ORC_STOP) {
        for (int k = 0; k < 4; k++) win[k] = win[32 + k];
        int ndx = 4;
        while (ndx < 36) {
            if (x < 0 || y < 0) { b = ORC_STOP; break; }
            b = btck[(size_t)y * Ld + x];
            if (b == ORC_STOP) break;
            if (b == ORC_UP) { y--; continue; }
            if (b == ORC_LEFT) { x--; continue; }
            win[ndx] = S[(size_t)y * lds + x];
            if (win[ndx] > 0.0f) psts++;
            x--; y--; ndx++;
        }
        float corr[32];
        for (int t = 0; t < 32; t++)
            corr[t] = (ndx <= t + 4) ? 0.0f
                                     : win[t + 4] * (((win[t] + win[t + 1]) + win[t + 2]) + win[t + 3]);
        sumcorr = sumcorr + orc_butterfly_sum32(corr);
    }
    sumcorr = sumcorr * 0.5f;
    sumcorr = sumcorr < 0.0f ? -sqrtf(-sumcorr) : sqrtf(sumcorr);
    maxsc = maxsc + sumcorr;
    *out_score = maxsc;
    *out_psts = (float)psts;
    *beg = ((uint32_t)(x + 1) << 16) | (uint32_t)(y + 1);
    *end = ((uint32_t)maxc << 16) | (uint32_t)maxr;
    return thld < maxsc;
}

void orc_score_threshold(size_t nqyposs, size_t dbsize, float evalue, float gapped_lambda,
                         float gapped_k, float* scorethld, float* logevthld)
{
    size_t sspace = nqyposs * dbsize;
    float ev = evalue;
    if (ev <= 0.0f) { *scorethld = 999.0f; *logevthld = -99.0f; return; }
    *logevthld = logf(ev);
    if (ev < 1.0f) ev *= 10.0f; else ev *= 3.0f;
    ev /= gapped_k * (float)sspace;
    if (ev <= 0.0f) { *scorethld = 999.0f; return; }
    ev = logf(ev);
    float score = -ev / gapped_lambda;
    if (score < 0.0f) score = 0.0f;
    *scorethld = score;
}
