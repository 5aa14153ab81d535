/*
 * CPU oracle, statistics and E-values -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h. Compiled with -ffp-contract=off.
 *
 * Restates the reference's per-pair statistics (src/libmycu/cuss/):
 * score histogram, expected score, min/max, lambda (Newton + bisection),
 * relative entropy, K, and the SS18 / observed-parameter E-values with the
 * incomplete beta and gamma functions of src/libmycu/cusf/. The reference
 * evaluates sums with warp shuffles on a 21 x 32 thread grid; the grid and
 * the shuffle orders are emulated here so that results are reproducible
 * bit for bit by the CUDA kernel, which runs the same sequence.
 */
#include "oracle.h"

#include <math.h>
#include <stdint.h>
#include <string.h>

#define NS 21          /* unscaled scores -10..10 */
#define SF 32          /* scale factor */
#define NSC 641        /* scaled scores -320..320 */
#define LOG_SP_MIN (-8.7336545e+01f)
#define LOG_SP_MAX (8.8722839e+01f)

/* ------------------------------------------------------------------------
 * exp restated: x = k*ln2 + r, |r| <= ln2/2 (k = rint(x*log2(e)), ln2 split
 * in a 16-bit head and a tail), exp(r) by its Taylor series to r^7/7!
 * (truncation < 6e-9 relative), times 2^k assembled from two exact powers
 * of two. Identical operation sequence on the device.
 */
float orc_expf(float x)
{
    if (x != x) return x;
    if (!(x < 88.7228f)) return INFINITY;
    if (x < -103.972f) return 0.0f;
    float kf = rintf(x * 1.44269504f);
    float r = fmaf(kf, -0.693145751953125f, x);
    r = fmaf(kf, -1.42860677e-06f, r);
    float p = 1.98412698e-04f;
    p = fmaf(p, r, 1.38888889e-03f);
    p = fmaf(p, r, 8.33333333e-03f);
    p = fmaf(p, r, 4.16666667e-02f);
    p = fmaf(p, r, 1.66666667e-01f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int k = (int)kf;
    int k1 = k / 2, k2 = k - k1;
    union { uint32_t u; float f; } s1, s2;
    s1.u = (uint32_t)(k1 + 127) << 23;
    s2.u = (uint32_t)(k2 + 127) << 23;
    return (p * s1.f) * s2.f;
}

/* log-gamma for x > 0: shift x up to >= 8 accumulating the product, then
 * Stirling's series (x-1/2)log x - x + log(2 pi)/2 + 1/(12x) - 1/(360x^3)
 * + 1/(1260x^5) - 1/(1680x^7). */
float orc_lgammaf(float x)
{
    float prod = 1.0f;
    while (x < 8.0f) { prod = prod * x; x = x + 1.0f; }
    float lx = orc_logf(x);
    float ix = 1.0f / x;
    float ix2 = ix * ix;
    float ser = fmaf(ix2, fmaf(ix2, fmaf(ix2, -5.95238095e-04f, 7.93650794e-04f), -2.77777778e-03f),
                     8.33333333e-02f) * ix;
    float r = fmaf(x - 0.5f, lx, -x);
    r = r + 0.918938533f;
    r = r + ser;
    return r - orc_logf(prod);
}

static float orc_powf(float x, float y) { return orc_expf(y * orc_logf(x)); }

/* ------------------------------------------------------------------------
 * warp reductions: lane 0's value after __shfl_down (tree t += t+off) and
 * the common value after __shfl_xor (butterfly t += t^off), offsets
 * 16,8,4,2,1 (src/libmycu/cuss/CuBatchSS_dynplm.cu:224-242)
 */
static float red_down(const float* v)
{
    float a[32], b[32];
    memcpy(a, v, sizeof(a));
    for (int off = 16; off >= 1; off >>= 1) {
        for (int t = 0; t < 32; t++) b[t] = a[t] + (t + off < 32 ? a[t + off] : a[t]);
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

static float red_xor(const float* v)
{
    float a[32], b[32];
    memcpy(a, v, sizeof(a));
    for (int off = 16; off >= 1; off >>= 1) {
        for (int t = 0; t < 32; t++) b[t] = a[t] + a[t ^ off];
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

static float min_down(const float* v)
{
    float a[32], b[32];
    memcpy(a, v, sizeof(a));
    for (int off = 16; off >= 1; off >>= 1) {
        for (int t = 0; t < 32; t++) { float o = t + off < 32 ? a[t + off] : a[t]; b[t] = a[t] < o ? a[t] : o; }
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

static float max_down(const float* v)
{
    float a[32], b[32];
    memcpy(a, v, sizeof(a));
    for (int off = 16; off >= 1; off >>= 1) {
        for (int t = 0; t < 32; t++) { float o = t + off < 32 ? a[t + off] : a[t]; b[t] = a[t] < o ? o : a[t]; }
        memcpy(a, b, sizeof(a));
    }
    return a[0];
}

/* two-level sum over the 21 x 32 grid: per row by __shfl_down, rows by
 * __shfl_down over lanes 0..20 of row 0 */
static float grid_sum(float g[NS][32])
{
    float rows[32];
    for (int y = 0; y < 32; y++) rows[y] = y < NS ? red_down(g[y]) : 0.0f;
    return red_down(rows);
}

/* interval of histogram indices held by grid row y
 * (src/libmycu/cuss/CuBatchSS_dynplm.cu:199-214) */
static void row_interval(int y, int* left, int* right)
{
    int unscaled = y - 10;
    int l = unscaled * SF - (SF >> 1) + 320;
    int r = unscaled * SF + (SF >> 1) + 320;
    if (unscaled <= 0) { l++; if (l < 0) l = 0; }
    if (0 <= unscaled) { r--; if (NSC - 1 < r) r = NSC - 1; }
    *left = l;
    *right = r;
}

/* ------------------------------------------------------------------------
 * lambda: root of sum_s p(s) exp(lambda (s - max)) - exp(-lambda max) by
 * Newton steps guarded by bisection on [1e-5, 10]
 * (src/libmycu/cuss/CuBatchSS_lambda.cuh:80-330)
 */
static void lmbd_eq(float x, float g[NS][32], const int* left, float minsc, float maxsc,
                    float* f, float* df)
{
    float lf[NS][32], ldf[NS][32];
    for (int y = 0; y < NS; y++)
        for (int t = 0; t < 32; t++) {
            float a = 0.0f, b = 0.0f;
            float sc = (float)(left[y] + t - 320);
            if (minsc <= sc && sc <= maxsc) {
                sc = sc - maxsc;
                float yy = x * sc;
                if (LOG_SP_MIN < yy) {
                    a = orc_expf(yy) * g[y][t];
                    b = a * sc;
                }
            }
            lf[y][t] = a;
            ldf[y][t] = b;
        }
    float F = grid_sum(lf), DF = grid_sum(ldf);
    float xm = x * -maxsc;
    if (LOG_SP_MIN < xm) {
        xm = orc_expf(xm);
        F = F - xm;
        DF = DF + xm * maxsc;
    }
    *f = F;
    if (df) *df = DF;
}

static float orc_lambda(float g[NS][32], const int* left, float expected, float minsc, float maxsc)
{
    const float X1 = 1.0e-5f, X2 = 10.0f;
    if (0.0f <= expected || maxsc <= 0.0f) return -1.0f;
    float f, df, fl, dx, dxold, xh, xl, rts;
    lmbd_eq(X1, g, left, minsc, maxsc, &fl, 0);
    lmbd_eq(X2, g, left, minsc, maxsc, &f, 0);
    if ((fl > 0.0f && f > 0.0f) || (fl < 0.0f && f < 0.0f)) return -1.0f;
    if (fl < 0.0f) { xl = X1; xh = X2; } else { xh = X1; xl = X2; }
    rts = 0.5f * (X1 + X2);
    dxold = fabsf(X2 - X1);
    dx = dxold;
    lmbd_eq(rts, g, left, minsc, maxsc, &f, &df);
    int n;
    for (n = 0; n < 32; n++) {
        int stop = 0;
        if ((((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0f) || (fabsf(2.0f * f) > fabsf(dxold * df))) {
            dxold = dx;
            dx = 0.5f * (xh - xl);
            rts = xl + dx;
            if (xl == rts) stop = 1;
        } else {
            dxold = dx;
            dx = f / df;
            float temp = rts;
            rts = rts - dx;
            if (temp == rts) stop = 1;
        }
        if (fabsf(dx) < 1.0e-4f) stop = 1;
        if (stop) break;
        lmbd_eq(rts, g, left, minsc, maxsc, &f, &df);
        if (f < 0.0f) xl = rts; else xh = rts;
    }
    if (n == 32) return -1.0f;
    return rts;
}

/* relative entropy on scaled scores (src/libmycu/cuss/CuBatchSS_entropy.cuh:14-70) */
static float orc_entropy(float g[NS][32], const int* left, float minsc, float maxsc, float lambda)
{
    if (lambda <= 0.0f) return -1.0f;
    float e[NS][32];
    for (int y = 0; y < NS; y++)
        for (int t = 0; t < 32; t++) {
            float v = 0.0f;
            float sc = (float)(left[y] + t - 320);
            if (minsc <= sc && sc <= maxsc) {
                float yy = lambda * sc;
                if (LOG_SP_MIN < yy && yy < LOG_SP_MAX - 3.0f) v = orc_expf(yy) * yy * g[y][t];
            }
            e[y][t] = v;
        }
    return grid_sum(e);
}

/* K (src/libmycu/cuss/CuBatchSS_K.cuh:49-320). The probabilities of
 * alignment scores of length j live on the same 21 x 32 grid (cell (y,t)
 * stands for score left[y]+t-320; a shift by i moves along the row and
 * wraps into the neighbouring row), and are convolved with the unscaled
 * score distribution. Each step reads the previous step's grid only. */
static float orc_K(float g[NS][32], const float* up, const int* left, int minu, int maxu,
                   float expected, float lambda, float relent)
{
    if (0.0f <= expected || lambda <= 0.0f || relent <= 0.0f) return -1.0f;
    if (minu == -1 && maxu == 1) {
        float minprb = up[-1 + 10], maxprb = up[1 + 10];
        float d = minprb - maxprb;
        return (d * d) / minprb;
    } else if (minu == -1 || maxu == 1) {
        if (maxu != 1) return (lambda / relent) * (1.0f - orc_expf(-lambda)) * (expected * expected);
        return (relent / lambda) * (1.0f - orc_expf(-lambda));
    }
    const int range = maxu - minu + 1;
    float sigma = 0.0f, Pj = 1.0f;
    int mins = minu, maxs = maxu;
    float nxt[NS][32], pj[NS][32];
    for (int j = 1; j <= 32 && 1.0e-4f < Pj; j++) {
        for (int y = 0; y < NS; y++)
            for (int t = 0; t < 32; t++) {
                float pji = 0.0f, p = 0.0f;
                int sc = left[y] + t - 320;
                if (mins <= sc && sc <= maxs && -32 <= sc && sc <= 32) {
                    float etols = sc < 0 ? lambda * (float)sc : 0.0f;
                    if (LOG_SP_MIN < etols) {
                        int lo = (maxs - sc < range) ? maxu - (maxs - sc) : minu;
                        int hi = (sc - mins < range) ? minu + (sc - mins) : maxu;
                        for (int i = lo; i <= hi; i++) {
                            int yy = y, xx = t - i;
                            if (32 <= xx) { xx -= 32; if (yy + 1 < NS) yy++; else continue; }
                            else if (xx < 0) { xx += 32; if (0 < yy) yy--; else continue; }
                            pji = fmaf(g[yy][xx], up[i + 10], pji);
                        }
                        p = pji * orc_expf(etols);
                    }
                }
                nxt[y][t] = pji;
                pj[y][t] = p;
            }
        memcpy(g, nxt, sizeof(nxt));
        Pj = grid_sum(pj);
        sigma = sigma + Pj / (float)j;
        mins += minu;
        maxs += maxu;
    }
    return (lambda * orc_expf(-2.0f * sigma)) / (relent * (1.0f - orc_expf(-lambda)));
}

/* ------------------------------------------------------------------------
 * Histogram of rint(32 * clamp(score, -10, 10)) over a pair's cells,
 * skipping X positions when xuninf (src/libmycu/cuss/CuBatchSS_dynplm.cu:77-180).
 */
void orc_score_histogram(int Lq, int Ld, const float* S, long long lds, const char* qaa,
                         const char* daa, int xuninf, int* counts)
{
    memset(counts, 0, NSC * sizeof(int));
    for (int r = 0; r < Lq; r++)
        for (int c = 0; c < Ld; c++) {
            if (xuninf && (qaa[r] == 'X' || daa[c] == 'X')) continue;
            float s = S[(size_t)r * lds + c];
            if (s < -10.0f) s = -10.0f; else if (s > 10.0f) s = 10.0f;
            int k = (int)rintf(s * 32.0f);
            counts[k + 320]++;
        }
}

/* statistics from the histogram (src/libmycu/cuss/CuBatchSS_dynplm.cu:190-394):
 * out[0..5] = min, max, E, H, lambda, K (unscaled min/max, rescaled E and
 * lambda), up[21] = unscaled probabilities */
void orc_stat_params(const int* counts, float* out, float* up)
{
    float g[NS][32];
    int left[NS], right[NS];
    for (int y = 0; y < NS; y++) {
        row_interval(y, &left[y], &right[y]);
        for (int t = 0; t < 32; t++)
            g[y][t] = (t + left[y] <= right[y]) ? (float)counts[left[y] + t] : 0.0f;
    }
    float rowsum[32];
    for (int y = 0; y < 32; y++) rowsum[y] = y < NS ? red_xor(g[y]) : 0.0f;
    float total = red_xor(rowsum);
    for (int y = 0; y < NS; y++) up[y] = rowsum[y] / total;
    for (int y = 0; y < NS; y++)
        for (int t = 0; t < 32; t++) g[y][t] = g[y][t] / total;

    /* expected scaled score (src/libmycu/cuss/CuBatchSS_expected.cuh:12-46) */
    float ex[NS][32];
    for (int y = 0; y < NS; y++)
        for (int t = 0; t < 32; t++) ex[y][t] = (float)(left[y] + t - 320) * g[y][t];
    float E = grid_sum(ex);
    /* min/max scaled scores, 0 included (src/libmycu/cuss/CuBatchSS_minmax.cuh:12-60) */
    float rmin[32], rmax[32];
    for (int y = 0; y < 32; y++) {
        if (y < NS) {
            float mn[32];
            for (int t = 0; t < 32; t++) mn[t] = g[y][t] != 0.0f ? (float)(left[y] + t - 320) : 0.0f;
            rmin[y] = min_down(mn);
            rmax[y] = max_down(mn);
        } else {
            rmin[y] = rmax[y] = 0.0f;
        }
    }
    float mins = min_down(rmin), maxs = max_down(rmax);
    float lambda = orc_lambda(g, left, E, mins, maxs);
    float H = orc_entropy(g, left, mins, maxs, lambda);
    /* reset row 10 (score 0) to ones: the seed of the K convolution */
    for (int t = 0; t < 32; t++) g[10][t] = 1.0f;
    lambda = lambda * 32.0f;
    E = E / 32.0f;
    /* min/max unscaled scores (src/libmycu/cuss/CuBatchSS_minmax.cuh:62-99) */
    float um[32];
    for (int t = 0; t < 32; t++) um[t] = (t < NS && up[t] != 0.0f) ? (float)(t - 10) : 0.0f;
    float minu = min_down(um), maxu = max_down(um);
    float K = orc_K(g, up, left, (int)minu, (int)maxu, E, lambda, H);
    out[0] = minu;
    out[1] = maxu;
    out[2] = E;
    out[3] = H;
    out[4] = lambda;
    out[5] = K;
}

/* ------------------------------------------------------------------------
 * The parameter fit in FP64: the same estimation as orc_stat_params (the
 * reference's equations, constants, guards and stopping rules:
 * src/libmycu/cuss/CuBatchSS_expected.cuh, CuBatchSS_lambda.cuh:80-330,
 * CuBatchSS_entropy.cuh:14-70, CuBatchSS_K.cuh:49-320) in double precision
 * with the C library's exp, sums taken in plain loop order. The checker of
 * the CUDA path's FP64 fit (the precision forms) and the FP64 side of the
 * FP32 fit's error report.
 * out[0..3] = lambda (unscaled), K, H, expected score (unscaled).
 */
static void lmbd_eq64(double x, double g[NS][32], const int* left, double minsc, double maxsc,
                      double* f, double* df)
{
    double F = 0.0, DF = 0.0;
    for (int y = 0; y < NS; y++)
        for (int t = 0; t < 32; t++) {
            double sc = (double)(left[y] + t - 320);
            if (minsc <= sc && sc <= maxsc) {
                sc = sc - maxsc;
                double yy = x * sc;
                if ((double)LOG_SP_MIN < yy) {
                    double a = exp(yy) * g[y][t];
                    F += a;
                    DF += a * sc;
                }
            }
        }
    double xm = x * -maxsc;
    if ((double)LOG_SP_MIN < xm) {
        xm = exp(xm);
        F = F - xm;
        DF = DF + xm * maxsc;
    }
    *f = F;
    if (df) *df = DF;
}

void orc_stat_params64(const int* counts, double* out)
{
    double g[NS][32], up[NS];
    int left[NS], right[NS];
    double total = 0.0;
    for (int y = 0; y < NS; y++) {
        row_interval(y, &left[y], &right[y]);
        for (int t = 0; t < 32; t++) {
            g[y][t] = (t + left[y] <= right[y]) ? (double)counts[left[y] + t] : 0.0;
            total += g[y][t];
        }
    }
    for (int y = 0; y < NS; y++) {
        double rs = 0.0;
        for (int t = 0; t < 32; t++) rs += g[y][t];
        up[y] = rs / total;
    }
    double E = 0.0, mins = 0.0, maxs = 0.0;
    for (int y = 0; y < NS; y++)
        for (int t = 0; t < 32; t++) {
            g[y][t] = g[y][t] / total;
            double sc = (double)(left[y] + t - 320);
            E += sc * g[y][t];
            if (g[y][t] != 0.0) {
                if (sc < mins) mins = sc;
                if (sc > maxs) maxs = sc;
            }
        }
    /* lambda */
    double lambda = -1.0;
    if (!(0.0 <= E || maxs <= 0.0)) {
        const double X1 = 1.0e-5, X2 = 10.0;
        double f, df, fl, dx, dxold, xh, xl, rts;
        lmbd_eq64(X1, g, left, mins, maxs, &fl, 0);
        lmbd_eq64(X2, g, left, mins, maxs, &f, 0);
        if (!((fl > 0.0 && f > 0.0) || (fl < 0.0 && f < 0.0))) {
            if (fl < 0.0) { xl = X1; xh = X2; } else { xh = X1; xl = X2; }
            rts = 0.5 * (X1 + X2);
            dxold = fabs(X2 - X1);
            dx = dxold;
            lmbd_eq64(rts, g, left, mins, maxs, &f, &df);
            int n;
            for (n = 0; n < 32; n++) {
                int stop = 0;
                if ((((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0) || (fabs(2.0 * f) > fabs(dxold * df))) {
                    dxold = dx;
                    dx = 0.5 * (xh - xl);
                    rts = xl + dx;
                    if (xl == rts) stop = 1;
                } else {
                    dxold = dx;
                    dx = f / df;
                    double temp = rts;
                    rts = rts - dx;
                    if (temp == rts) stop = 1;
                }
                if (fabs(dx) < 1.0e-4) stop = 1;
                if (stop) break;
                lmbd_eq64(rts, g, left, mins, maxs, &f, &df);
                if (f < 0.0) xl = rts; else xh = rts;
            }
            lambda = (n == 32) ? -1.0 : rts;
        }
    }
    /* relative entropy */
    double H = -1.0;
    if (lambda > 0.0) {
        H = 0.0;
        for (int y = 0; y < NS; y++)
            for (int t = 0; t < 32; t++) {
                double sc = (double)(left[y] + t - 320);
                if (mins <= sc && sc <= maxs) {
                    double yy = lambda * sc;
                    if ((double)LOG_SP_MIN < yy && yy < (double)LOG_SP_MAX - 3.0) H += exp(yy) * yy * g[y][t];
                }
            }
    }
    for (int t = 0; t < 32; t++) g[10][t] = 1.0;
    lambda = lambda * 32.0;
    E = E / 32.0;
    int minu = 0, maxu = 0;
    for (int t = 0; t < NS; t++)
        if (up[t] != 0.0) {
            if (t - 10 < minu) minu = t - 10;
            if (t - 10 > maxu) maxu = t - 10;
        }
    /* K */
    double K = -1.0;
    if (!(0.0 <= E || lambda <= 0.0 || H <= 0.0)) {
        if (minu == -1 && maxu == 1) {
            double minprb = up[-1 + 10], maxprb = up[1 + 10];
            double d = minprb - maxprb;
            K = d * d / minprb;
        } else if (minu == -1 || maxu == 1) {
            if (maxu != 1) K = (lambda / H) * (1.0 - exp(-lambda)) * (E * E);
            else K = (H / lambda) * (1.0 - exp(-lambda));
        } else {
            const int range = maxu - minu + 1;
            double sigma = 0.0, Pj = 1.0;
            int mn = minu, mx = maxu;
            double nxt[NS][32];
            for (int j = 1; j <= 32 && 1.0e-4 < Pj; j++) {
                double P = 0.0;
                for (int y = 0; y < NS; y++)
                    for (int t = 0; t < 32; t++) {
                        double pji = 0.0;
                        int sc = left[y] + t - 320;
                        if (mn <= sc && sc <= mx && -32 <= sc && sc <= 32) {
                            double etols = sc < 0 ? lambda * (double)sc : 0.0;
                            if ((double)LOG_SP_MIN < etols) {
                                int lo = (mx - sc < range) ? maxu - (mx - sc) : minu;
                                int hi = (sc - mn < range) ? minu + (sc - mn) : maxu;
                                for (int i = lo; i <= hi; i++) {
                                    int yy = y, xx = t - i;
                                    if (32 <= xx) { xx -= 32; if (yy + 1 < NS) yy++; else continue; }
                                    else if (xx < 0) { xx += 32; if (0 < yy) yy--; else continue; }
                                    pji = fma(g[yy][xx], up[i + 10], pji);
                                }
                                P += pji * exp(etols);
                            }
                        }
                        nxt[y][t] = pji;
                    }
                memcpy(g, nxt, sizeof(nxt));
                Pj = P;
                sigma = sigma + Pj / (double)j;
                mn += minu;
                mx += maxu;
            }
            K = lambda * exp(-2.0 * sigma) / (H * (1.0 - exp(-lambda)));
        }
    }
    out[0] = lambda;
    out[1] = K;
    out[2] = H;
    out[3] = E;
}

/* ------------------------------------------------------------------------
 * Incomplete beta (log) and incomplete gamma (log of the upper tail), after
 * the published Cephes single-precision algorithms (incbetf: continued
 * fractions #1/#2 and power series; igamcf/igamf), as restated in
 * src/libmycu/cusf/CuSF_betainc.cuh and CuSF_gammainc.cuh.
 */
#define MACHEPF 5.9604644775390625e-8f
#define BIGSP 16777216.0f

static float bcf1(float a, float b, float x)
{
    float xk, pk, pkm1 = 1.0f, pkm2 = 0.0f, qk, qkm1 = 1.0f, qkm2 = 1.0f;
    float k1 = a, k2 = a + b, k3 = a, k4 = a + 1.0f, k5 = 1.0f, k6 = b - 1.0f, k7 = a + 1.0f, k8 = a + 2.0f;
    float r = 0.0f, t, ans = 1.0f;
    for (int n = 0; n < 100; n++) {
        xk = -((x * k1 * k2) / (k3 * k4));
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        xk = (x * k5 * k6) / (k7 * k8);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (qk != 0.0f) r = pk / qk;
        if (r != 0.0f) { t = fabsf((ans - r) / r); ans = r; } else t = 1.0f;
        if (t < MACHEPF) break;
        k1 += 1.0f; k2 += 1.0f; k3 += 2.0f; k4 += 2.0f; k5 += 1.0f; k6 -= 1.0f; k7 += 2.0f; k8 += 2.0f;
        if ((fabsf(qk) + fabsf(pk)) > BIGSP) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
        if ((fabsf(qk) < MACHEPF) || (fabsf(pk) < MACHEPF)) { pkm2 *= BIGSP; pkm1 *= BIGSP; qkm2 *= BIGSP; qkm1 *= BIGSP; }
    }
    return ans;
}

static float bcf2(float a, float b, float x)
{
    float xk, pk, pkm1 = 1.0f, pkm2 = 0.0f, qk, qkm1 = 1.0f, qkm2 = 1.0f;
    float k1 = a, k2 = b - 1.0f, k3 = a, k4 = a + 1.0f, k5 = 1.0f, k6 = a + b, k7 = a + 1.0f, k8 = a + 2.0f;
    float r = 0.0f, t, ans = 1.0f;
    float z = x / (1.0f - x);
    for (int n = 0; n < 100; n++) {
        xk = -((z * k1 * k2) / (k3 * k4));
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        xk = (z * k5 * k6) / (k7 * k8);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (qk != 0.0f) r = pk / qk;
        if (r != 0.0f) { t = fabsf((ans - r) / r); ans = r; } else t = 1.0f;
        if (t < MACHEPF) break;
        k1 += 1.0f; k2 -= 1.0f; k3 += 2.0f; k4 += 2.0f; k5 += 1.0f; k6 += 1.0f; k7 += 2.0f; k8 += 2.0f;
        if ((fabsf(qk) + fabsf(pk)) > BIGSP) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
        if ((fabsf(qk) < MACHEPF) || (fabsf(pk) < MACHEPF)) { pkm2 *= BIGSP; pkm1 *= BIGSP; qkm2 *= BIGSP; qkm1 *= BIGSP; }
    }
    return ans;
}

static float bps(float a, float b, float x)
{
    float y = a * orc_logf(x) + (b - 1.0f) * orc_logf(1.0f - x) - orc_logf(a);
    y = y - (orc_lgammaf(a) + orc_lgammaf(b));
    y = y + orc_lgammaf(a + b);
    float t = x / (1.0f - x), s = 0.0f, u = 1.0f;
    for (int it = 0; it < 10000; it++) {
        b -= 1.0f;
        if (b == 0.0f) break;
        a += 1.0f;
        u *= (t * b) / a;
        s += u;
        if (!(fabsf(u) > MACHEPF)) break;
    }
    return y + orc_logf(1.0f + s);
}

static float lbetainc_helper(float a, float b, float x)
{
    float ans, t = 1.0f - x;
    if (b > 10.0f && fabsf((b * x) / a) < 0.3f) return bps(a, b, x);
    ans = x * ((a + b - 2.0f) / (a - 1.0f));
    if (ans < 1.0f) { ans = bcf1(a, b, x); t = b * orc_logf(t); }
    else { ans = bcf2(a, b, x); t = (b - 1.0f) * orc_logf(t); }
    t = t + (a * orc_logf(x) + orc_lgammaf(a + b) - orc_lgammaf(a) - orc_lgammaf(b));
    t = t + orc_logf(ans / a);
    return t;
}

float orc_lbetaincf(float aa, float bb, float xx)
{
    if ((xx <= 0.0f) || (xx >= 1.0f)) {
        if (xx == 0.0f) return -999.0f;
        if (xx == 1.0f) return 0.0f;
        return 999.0f;
    }
    if (aa <= 0.0f) return 999.0f;
    if (aa <= 1.0f) {
        float ans = lbetainc_helper(aa + 1.0f, bb, xx);
        ans = ans > LOG_SP_MIN ? orc_expf(ans) : 0.0f;
        float t = aa * orc_logf(xx) + bb * orc_logf(1.0f - xx) + orc_lgammaf(aa + bb) -
                  orc_lgammaf(aa + 1.0f) - orc_lgammaf(bb);
        if (t > LOG_SP_MIN) ans += orc_expf(t);
        return ans != 0.0f ? orc_logf(ans) : -999.0f;
    }
    return lbetainc_helper(aa, bb, xx);
}

static float lgammainc_P(float a, float x);

float orc_lgammainc_Qf(float a, float x)
{
    if ((x <= 0.0f) || (a <= 0.0f)) return 0.0f;
    if ((x < 1.0f) || (x < a)) {
        float ans = lgammainc_P(a, x);
        ans = ans > LOG_SP_MIN ? orc_expf(ans) : 0.0f;
        return ans < 1.0f ? orc_logf(1.0f - ans) : -999.0f;
    }
    float ax = a * orc_logf(x) - x - orc_lgammaf(a);
    float y = 1.0f - a, z = x + y + 1.0f, c = 0.0f;
    float pkm2 = 1.0f, qkm2 = x, pkm1 = x + 1.0f, qkm1 = z * x;
    float ans = pkm1 / qkm1, t, r, pk, qk, yc;
    for (int it = 0; it < 10000; it++) {
        c += 1.0f; y += 1.0f; z += 2.0f;
        yc = y * c;
        pk = pkm1 * z - pkm2 * yc;
        qk = qkm1 * z - qkm2 * yc;
        if (qk != 0.0f) { r = pk / qk; t = fabsf((ans - r) / r); ans = r; } else t = 1.0f;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (fabsf(pk) > BIGSP) { pkm2 *= MACHEPF; pkm1 *= MACHEPF; qkm2 *= MACHEPF; qkm1 *= MACHEPF; }
        if (!(t > MACHEPF)) break;
    }
    return orc_logf(ans) + ax;
}

static float lgammainc_P(float a, float x)
{
    if ((x <= 0.0f) || (a <= 0.0f)) return -999.0f;
    if ((x > 1.0f) && (x > a)) {
        float ans = orc_lgammainc_Qf(a, x);
        ans = ans > LOG_SP_MIN ? orc_expf(ans) : 0.0f;
        return ans < 1.0f ? orc_logf(1.0f - ans) : -999.0f;
    }
    float ax = a * orc_logf(x) - x - orc_lgammaf(a);
    float r = a, c = 1.0f, ans = 1.0f;
    for (int it = 0; it < 10000; it++) {
        r += 1.0f;
        c *= x / r;
        ans += c;
        if (!(c / ans > MACHEPF)) break;
    }
    return orc_logf(ans) + ax - orc_logf(a);
}

/* ------------------------------------------------------------------------
 * Significance (src/libmycu/cuss/CuBatchSS_SS18.cuh:119-360,
 * CuBatchSS_NN.cuh:24-160).
 */
static float nn_act(float v) { return 2.0f / (1.0f + orc_expf(-v)) - 1.0f; }

/* one-layer network: 4 inputs, 4 hidden units, weights row-major with the
 * bias first; w_out = [bias, 4 weights] */
static float nn_eval(const float* w, const float* in, float outfactor)
{
    float h[4];
    for (int u = 0; u < 4; u++) {
        float p0 = in[0] * w[u * 5 + 1], p1 = in[1] * w[u * 5 + 2];
        float p2 = in[2] * w[u * 5 + 3], p3 = in[3] * w[u * 5 + 4];
        float s = w[u * 5] + p0 + p1 + p2 + p3;
        h[u] = nn_act(s) * w[20 + u + 1];
    }
    float o = w[20] + h[0] + h[1] + h[2] + h[3];
    return nn_act(o) * outfactor;
}

void orc_significance(const orc_sig_params* sp, int Lq, int Ld, float qeno, float deno,
                      float score, float psts, float lambda, float K, float* out4)
{
    /* out4: lambda_est, K_est, log E, log E per pair */
    const float* W = sp->nnweights;
    float lest = 0.0f, kest = 0.0f;
    if (0.0f < lambda) lest = lambda * (sp->exp_gapped_lambda / sp->ref_lambda);
    if (0.0f < K) kest = K * (sp->exp_gapped_K / sp->ref_K);
    float l1l2 = (float)((unsigned)Lq * (unsigned)Ld);
    float epa;
    if (lambda <= 0.0f || K <= 0.0f) epa = orc_logf(sp->ref_K * l1l2) - sp->ref_lambda * score;
    else epa = orc_logf(K * l1l2) - lambda * score;
    float logE;
    if (sp->ssemodel == 0) {
        logE = orc_logf(sp->exp_gapped_K * sp->searchspace) - sp->exp_gapped_lambda * score;
    } else {
        /* EVD parameters predicted by the networks */
        float in[4];
        unsigned n1 = (unsigned)Lq, n2 = (unsigned)Ld;
        float e1 = qeno, e2 = deno;
        if (e1 < e2) { float t = e1; e1 = e2; e2 = t; unsigned u = n1; n1 = n2; n2 = u; }
        else if (e1 == e2 && n1 < n2) { unsigned u = n1; n1 = n2; n2 = u; }
        const float LN1K = 6.90775527898f;
        in[0] = 0.05f * e1;
        in[1] = orc_logf((float)n1) / LN1K;
        in[2] = 0.05f * e2;
        in[3] = orc_logf((float)n2) / LN1K;
        float muE = nn_eval(W, in, 30.0f);
        float lm = rintf(lambda * 10.0f) / 10.0f;
        if (lm <= 0.0f) lm = 0.1f;
        if (10.0f < lm) lm = 10.0f;
        n1 = (unsigned)Lq; n2 = (unsigned)Ld;
        if (n1 < n2) { unsigned u = n1; n1 = n2; n2 = u; }
        in[0] = 0.2f * lm;
        in[1] = orc_logf((float)n1) / LN1K;
        in[2] = orc_logf((float)n2) / LN1K;
        in[3] = 0.0f;
        float muL = nn_eval(W + 25, in, 30.0f);
        float scL = nn_eval(W + 50, in, 5.0f);
        const float* adj = W + 75 + (sp->ssemodel == 2 ? 9 : 0);
        if (muE < 3.0f) muE = 3.0f;
        if (muL < 3.0f) muL = 3.0f;
        if (scL < 0.1f) scL = 0.1f;
        scL = adj[6] * (orc_expf(scL) - 1.0f);
        if (scL < 0.1f) scL = 0.1f;
        if (5.0f < scL) scL = 5.0f;
        float scaleE = adj[4] * muE + adj[5];
        if (scaleE < 0.1f) scaleE = 0.1f;
        if (5.0f < scaleE) scaleE = 5.0f;
        muE = adj[0] * muE + adj[1];
        muL = adj[2] * muL + adj[3];
        float alpha = adj[7], ibeta = adj[8];
        if (0.0f < lambda) {
            float rcp = 1.0f / lambda;
            float m = rcp < 10.0f ? rcp : 10.0f;
            alpha = alpha - alpha * 0.1f * m;
            ibeta = ibeta + (1.0f - ibeta) * 0.1f * m;
        }
        float mu = alpha * muE + (1.0f - alpha) * muL;
        float scale = (1.0f - ibeta) * scaleE + ibeta * scL;
        if (mu <= 0.0f || scale <= 0.0f) {
            logE = orc_logf(sp->exp_gapped_K * sp->searchspace) - sp->exp_gapped_lambda * score;
        } else {
            float logKmn = mu / scale;
            if (K > sp->ref_K && 0.0f < K && K < 1.0f && 0.0f < sp->ref_K && sp->ref_K < 1.0f)
                logKmn = logKmn + orc_logf(K / sp->ref_K);
            float logexpect = logKmn - score / scale;
            if (sp->ssemodel == 2) logexpect = logexpect + -9.210340372f;
            float logp = logexpect;
            if (-4.605170186f <= logexpect) {
                if (LOG_SP_MAX - 3.0f < logexpect) logp = 0.0f;
                else {
                    logp = orc_expf(logexpect);
                    if (LOG_SP_MAX - 3.0f < logp) logp = 0.0f;
                    else logp = orc_logf(1.0f - orc_expf(-logp));
                }
            }
            float lp = l1l2 > 625.0f ? l1l2 : 625.0f;
            float pn = rintf((100000.0f * psts) / orc_powf(lp, 1.5f));
            float logpp = orc_lbetaincf(pn + 1.0f, 0.1f, 0.757213f);
            logp = orc_lgammainc_Qf(1.346206f, (-logp - logpp) / 1.485656f);
            logexpect = logp;
            if (-4.605170186f <= logp) {
                logp = orc_expf(logp);
                logexpect = 77.0f;
                if (logp < 1.0f) {
                    logexpect = -orc_logf(1.0f - logp);
                    logexpect = orc_logf(logexpect);
                }
            }
            logexpect = logexpect + orc_logf(sp->searchspace / l1l2);
            logE = logexpect;
        }
    }
    out4[0] = lest;
    out4[1] = kest;
    out4[2] = logE;
    out4[3] = epa;
}

/* Length adjustment for edge effects and the effective search space
 * (src/libpro/srcsco/AbstractScoreMatrix.cpp:303-393; Altschul et al. 2001,
 * solved as in Gertz 2005), with the gapped lambda, K, alpha, beta. */
void orc_length_adjustment(float lambda, float K, float alpha, float beta, size_t m,
                           unsigned long long n, size_t N, unsigned long long* sspace_out,
                           size_t* delta_out)
{
    *sspace_out = (unsigned long long)m * n;
    *delta_out = 0;
    if (lambda <= 0.0f || K <= 0.0f || N < 1) return;
    const float logK = logf(K);
    const float alratio = alpha / lambda;
    const float max_mn = (float)(m > n ? m : n);
    float length = 0.0f, min_length = 0.0f, max_length, nxt_length = 0.0f, sspace = 0.0f, space2;
    int converged = 0;
    float a = (float)N;
    float b = (float)(n + (unsigned long long)m * N);
    float c = (float)((unsigned long long)m * n) - max_mn / K;
    if (c < 0.0f) return;
    max_length = 2.0f * c / (b + sqrtf(b * b - 4.0f * a * c));
    for (int j = 0; j < 20; j++) {
        length = nxt_length;
        sspace = ((float)m - length) * ((float)n - (float)N * length);
        nxt_length = alratio * (logK + logf(sspace)) + beta;
        if (length <= nxt_length) {
            min_length = length;
            if (nxt_length - length <= 1.0f) { converged = 1; break; }
            if (min_length == max_length) break;
        } else
            max_length = length;
        if (nxt_length < min_length || max_length < nxt_length)
            nxt_length = (!j) ? max_length : (min_length + max_length) * 0.5f;
    }
    if (converged) {
        length = ceilf(min_length);
        if (length <= max_length) {
            space2 = ((float)m - length) * ((float)n - (float)N * length);
            nxt_length = alratio * (logK + logf(space2)) + beta;
            if (length <= nxt_length) { min_length = length; sspace = space2; }
        }
    }
    *sspace_out = (unsigned long long)sspace;
    *delta_out = (size_t)min_length;
}
