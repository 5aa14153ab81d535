// Alignment statistics and E-values of the pairs that passed phase 1.
//
// Reference: CalcStatisticsDynPlm and its children
// (src/libmycu/cuss/CuBatchSS_dynplm.cu:61-830) -- one parent thread per
// pair launching four child grids through dynamic parallelism: histogram
// with float atomicAdd, statistical parameters on a 32 x 21 block,
// significance by model SS18 (src/libmycu/cuss/CuBatchSS_SS18.cuh) or from
// observed parameters.
//
// Here one 672-thread block per pair does all of it in one launch for all
// pairs of a slab: an integer shared-memory histogram (exact, order-free),
// then the parameter estimation on the same 21 x 32 thread grid the
// reference uses -- grid row y holds the scaled scores rounding to the
// unscaled score y-10 -- with the reference's shuffle reduction orders, so
// every value is reproducible operation by operation on the CPU.
// Differences from the reference, all deliberate:
//  * exp/log/lgamma/pow are the bit-reproducible restatements of cbmath.cuh
//    (the reference uses __expf/__logf/__powf/lgammaf);
//  * divisions are IEEE (the reference uses __fdividef);
//  * the K convolution reads the previous step's grid only (the reference
//    overwrites the grid while other warps may still read it);
//  * lambda_est and K_est are 0 when lambda or K failed (left unset there).
#include "common.cuh"
#include "cbmath.cuh"
#include "stats_kernel.cuh"

namespace cbp {

namespace {

constexpr int NS = 21;          // unscaled scores -10..10
constexpr int NSC = 641;        // scaled scores -320..320
constexpr int kThreads = NS * 32;
constexpr float kLogSpMin = -8.7336545e+01f;
constexpr float kLogSpMax = 8.8722839e+01f;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float wsum_down(float v)
{
    v += __shfl_down_sync(kFull, v, 16);
    v += __shfl_down_sync(kFull, v, 8);
    v += __shfl_down_sync(kFull, v, 4);
    v += __shfl_down_sync(kFull, v, 2);
    v += __shfl_down_sync(kFull, v, 1);
    return v;
}
__device__ __forceinline__ float wsum_xor(float v)
{
    v += __shfl_xor_sync(kFull, v, 16);
    v += __shfl_xor_sync(kFull, v, 8);
    v += __shfl_xor_sync(kFull, v, 4);
    v += __shfl_xor_sync(kFull, v, 2);
    v += __shfl_xor_sync(kFull, v, 1);
    return v;
}
__device__ __forceinline__ float wmin_down(float v)
{
    for (int o = 16; o >= 1; o >>= 1) v = hmin(v, __shfl_down_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ float wmax_down(float v)
{
    for (int o = 16; o >= 1; o >>= 1) v = hmax(v, __shfl_down_sync(kFull, v, o));
    return v;
}

// Sum over the grid: per row (warp) by the shuffle-down tree, then the row
// sums by the same tree in warp 0. Result valid in thread 0; all threads
// must call (contains barriers).
__device__ __forceinline__ float grid_sum(float v, float* tmp)
{
    const int y = threadIdx.x >> 5, x = threadIdx.x & 31;
    v = wsum_down(v);
    if (x == 0) tmp[y] = v;
    __syncthreads();
    float t = 0.f;
    if (y == 0) {
        t = (x < NS) ? tmp[x] : 0.0f;
        t = wsum_down(t);
    }
    __syncthreads();
    return t;
}

// ---- incomplete beta / gamma (logs), Cephes single-precision algorithms
// as restated in src/libmycu/cusf/CuSF_betainc.cuh and CuSF_gammainc.cuh;
// every loop is bounded.
constexpr float kMachEp = 5.9604644775390625e-8f;
constexpr float kBig = 16777216.0f;

__device__ float bcf(float a, float b, float x, bool second)
{
    float pkm1 = 1.0f, pkm2 = 0.0f, qkm1 = 1.0f, qkm2 = 1.0f;
    float k1, k2, k3 = a, k4 = a + 1.0f, k5 = 1.0f, k6, k7 = a + 1.0f, k8 = a + 2.0f;
    float z;
    if (!second) { k1 = a; k2 = a + b; k6 = b - 1.0f; z = x; }
    else { k1 = a; k2 = b - 1.0f; k6 = a + b; z = __fdiv_rn(x, 1.0f - x); }
    float r = 0.0f, t, ans = 1.0f;
    for (int n = 0; n < 100; n++) {
        float xk = -__fdiv_rn(z * k1 * k2, k3 * k4);
        float pk = pkm1 + pkm2 * xk, qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        xk = __fdiv_rn(z * k5 * k6, k7 * k8);
        pk = pkm1 + pkm2 * xk; qk = qkm1 + qkm2 * xk;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (qk != 0.0f) r = __fdiv_rn(pk, qk);
        if (r != 0.0f) { t = fabsf(__fdiv_rn(ans - r, r)); ans = r; } else t = 1.0f;
        if (t < kMachEp) break;
        k1 += 1.0f;
        if (!second) { k2 += 1.0f; k6 -= 1.0f; } else { k2 -= 1.0f; k6 += 1.0f; }
        k3 += 2.0f; k4 += 2.0f; k5 += 1.0f; k7 += 2.0f; k8 += 2.0f;
        if ((fabsf(qk) + fabsf(pk)) > kBig) { pkm2 *= kMachEp; pkm1 *= kMachEp; qkm2 *= kMachEp; qkm1 *= kMachEp; }
        if ((fabsf(qk) < kMachEp) || (fabsf(pk) < kMachEp)) { pkm2 *= kBig; pkm1 *= kBig; qkm2 *= kBig; qkm1 *= kBig; }
    }
    return ans;
}

__device__ float bps(float a, float b, float x)
{
    float y = a * cb_logf(x) + (b - 1.0f) * cb_logf(1.0f - x) - cb_logf(a);
    y = y - (cb_lgammaf(a) + cb_lgammaf(b));
    y = y + cb_lgammaf(a + b);
    const float t = __fdiv_rn(x, 1.0f - x);
    float s = 0.0f, u = 1.0f;
    for (int it = 0; it < 10000; it++) {
        b -= 1.0f;
        if (b == 0.0f) break;
        a += 1.0f;
        u *= __fdiv_rn(t * b, a);
        s += u;
        if (!(fabsf(u) > kMachEp)) break;
    }
    return y + cb_logf(1.0f + s);
}

__device__ float lbetainc_helper(float a, float b, float x)
{
    float t = 1.0f - x;
    if (b > 10.0f && fabsf(__fdiv_rn(b * x, a)) < 0.3f) return bps(a, b, x);
    float ans = x * __fdiv_rn(a + b - 2.0f, a - 1.0f);
    if (ans < 1.0f) { ans = bcf(a, b, x, false); t = b * cb_logf(t); }
    else { ans = bcf(a, b, x, true); t = (b - 1.0f) * cb_logf(t); }
    t = t + (a * cb_logf(x) + cb_lgammaf(a + b) - cb_lgammaf(a) - cb_lgammaf(b));
    t = t + cb_logf(__fdiv_rn(ans, a));
    return t;
}

__device__ float lbetaincf(float aa, float bb, float xx)
{
    if ((xx <= 0.0f) || (xx >= 1.0f)) {
        if (xx == 0.0f) return -999.0f;
        if (xx == 1.0f) return 0.0f;
        return 999.0f;
    }
    if (aa <= 0.0f) return 999.0f;
    if (aa <= 1.0f) {
        float ans = lbetainc_helper(aa + 1.0f, bb, xx);
        ans = ans > kLogSpMin ? cb_expf(ans) : 0.0f;
        const float t = aa * cb_logf(xx) + bb * cb_logf(1.0f - xx) + cb_lgammaf(aa + bb) -
                        cb_lgammaf(aa + 1.0f) - cb_lgammaf(bb);
        if (t > kLogSpMin) ans += cb_expf(t);
        return ans != 0.0f ? cb_logf(ans) : -999.0f;
    }
    return lbetainc_helper(aa, bb, xx);
}

__device__ float lgammainc_Q(float a, float x);

__device__ float lgammainc_P(float a, float x)
{
    if ((x <= 0.0f) || (a <= 0.0f)) return -999.0f;
    if ((x > 1.0f) && (x > a)) {
        float ans = lgammainc_Q(a, x);
        ans = ans > kLogSpMin ? cb_expf(ans) : 0.0f;
        return ans < 1.0f ? cb_logf(1.0f - ans) : -999.0f;
    }
    const float ax = a * cb_logf(x) - x - cb_lgammaf(a);
    float r = a, c = 1.0f, ans = 1.0f;
    for (int it = 0; it < 10000; it++) {
        r += 1.0f;
        c *= __fdiv_rn(x, r);
        ans += c;
        if (!(__fdiv_rn(c, ans) > kMachEp)) break;
    }
    return cb_logf(ans) + ax - cb_logf(a);
}

__device__ float lgammainc_Q(float a, float x)
{
    if ((x <= 0.0f) || (a <= 0.0f)) return 0.0f;
    if ((x < 1.0f) || (x < a)) {
        float ans = lgammainc_P(a, x);
        ans = ans > kLogSpMin ? cb_expf(ans) : 0.0f;
        return ans < 1.0f ? cb_logf(1.0f - ans) : -999.0f;
    }
    const float ax = a * cb_logf(x) - x - cb_lgammaf(a);
    float y = 1.0f - a, z = x + y + 1.0f, c = 0.0f;
    float pkm2 = 1.0f, qkm2 = x, pkm1 = x + 1.0f, qkm1 = z * x;
    float ans = __fdiv_rn(pkm1, qkm1);
    for (int it = 0; it < 10000; it++) {
        c += 1.0f; y += 1.0f; z += 2.0f;
        const float yc = y * c;
        const float pk = pkm1 * z - pkm2 * yc;
        const float qk = qkm1 * z - qkm2 * yc;
        float t;
        if (qk != 0.0f) { const float r = __fdiv_rn(pk, qk); t = fabsf(__fdiv_rn(ans - r, r)); ans = r; }
        else t = 1.0f;
        pkm2 = pkm1; pkm1 = pk; qkm2 = qkm1; qkm1 = qk;
        if (fabsf(pk) > kBig) { pkm2 *= kMachEp; pkm1 *= kMachEp; qkm2 *= kMachEp; qkm1 *= kMachEp; }
        if (!(t > kMachEp)) break;
    }
    return cb_logf(ans) + ax;
}

// significance networks (src/libmycu/cuss/CuBatchSS_NN.cuh:24-160)
__device__ __forceinline__ float nn_act(float v) { return __fdiv_rn(2.0f, 1.0f + cb_expf(-v)) - 1.0f; }

__device__ float nn_eval(const float* w, const float* in, float outfactor)
{
    float h[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const float p0 = in[0] * w[u * 5 + 1], p1 = in[1] * w[u * 5 + 2];
        const float p2 = in[2] * w[u * 5 + 3], p3 = in[3] * w[u * 5 + 4];
        const float s = w[u * 5] + p0 + p1 + p2 + p3;
        h[u] = nn_act(s) * w[20 + u + 1];
    }
    const float o = w[20] + h[0] + h[1] + h[2] + h[3];
    return nn_act(o) * outfactor;
}

// E-values of one pair (src/libmycu/cuss/CuBatchSS_SS18.cuh:119-360)
__device__ void significance(const StatsArgs& a, int Lq, int Ld, float qeno, float deno, float score,
                             float psts, float lambda, float K, float* out4)
{
    const float* W = a.nnweights;
    float lest = 0.0f, kest = 0.0f;
    if (0.0f < lambda) lest = lambda * __fdiv_rn(a.exp_gapped_lambda, a.ref_lambda);
    if (0.0f < K) kest = K * __fdiv_rn(a.exp_gapped_K, a.ref_K);
    const float l1l2 = (float)((unsigned)Lq * (unsigned)Ld);
    float epa;
    if (lambda <= 0.0f || K <= 0.0f) epa = cb_logf(a.ref_K * l1l2) - a.ref_lambda * score;
    else epa = cb_logf(K * l1l2) - lambda * score;
    float logE;
    if (a.ssemodel == 0) {
        logE = cb_logf(a.exp_gapped_K * a.searchspace) - a.exp_gapped_lambda * score;
    } else {
        float in[4];
        unsigned n1 = (unsigned)Lq, n2 = (unsigned)Ld;
        float e1 = qeno, e2 = deno;
        if (e1 < e2) { float t = e1; e1 = e2; e2 = t; unsigned u = n1; n1 = n2; n2 = u; }
        else if (e1 == e2 && n1 < n2) { unsigned u = n1; n1 = n2; n2 = u; }
        const float LN1K = 6.90775527898f;
        in[0] = 0.05f * e1;
        in[1] = __fdiv_rn(cb_logf((float)n1), LN1K);
        in[2] = 0.05f * e2;
        in[3] = __fdiv_rn(cb_logf((float)n2), LN1K);
        float muE = nn_eval(W, in, 30.0f);
        float lm = __fdiv_rn(rintf(lambda * 10.0f), 10.0f);
        if (lm <= 0.0f) lm = 0.1f;
        if (10.0f < lm) lm = 10.0f;
        n1 = (unsigned)Lq; n2 = (unsigned)Ld;
        if (n1 < n2) { unsigned u = n1; n1 = n2; n2 = u; }
        in[0] = 0.2f * lm;
        in[1] = __fdiv_rn(cb_logf((float)n1), LN1K);
        in[2] = __fdiv_rn(cb_logf((float)n2), LN1K);
        in[3] = 0.0f;
        float muL = nn_eval(W + 25, in, 30.0f);
        float scL = nn_eval(W + 50, in, 5.0f);
        const float* adj = W + 75 + (a.ssemodel == 2 ? 9 : 0);
        if (muE < 3.0f) muE = 3.0f;
        if (muL < 3.0f) muL = 3.0f;
        if (scL < 0.1f) scL = 0.1f;
        scL = adj[6] * (cb_expf(scL) - 1.0f);
        if (scL < 0.1f) scL = 0.1f;
        if (5.0f < scL) scL = 5.0f;
        float scaleE = adj[4] * muE + adj[5];
        if (scaleE < 0.1f) scaleE = 0.1f;
        if (5.0f < scaleE) scaleE = 5.0f;
        muE = adj[0] * muE + adj[1];
        muL = adj[2] * muL + adj[3];
        float alpha = adj[7], ibeta = adj[8];
        if (0.0f < lambda) {
            const float rcp = __fdiv_rn(1.0f, lambda);
            const float m = rcp < 10.0f ? rcp : 10.0f;
            alpha = alpha - alpha * 0.1f * m;
            ibeta = ibeta + (1.0f - ibeta) * 0.1f * m;
        }
        const float mu = alpha * muE + (1.0f - alpha) * muL;
        const float scale = (1.0f - ibeta) * scaleE + ibeta * scL;
        if (mu <= 0.0f || scale <= 0.0f) {
            logE = cb_logf(a.exp_gapped_K * a.searchspace) - a.exp_gapped_lambda * score;
        } else {
            float logKmn = __fdiv_rn(mu, scale);
            if (K > a.ref_K && 0.0f < K && K < 1.0f && 0.0f < a.ref_K && a.ref_K < 1.0f)
                logKmn = logKmn + cb_logf(__fdiv_rn(K, a.ref_K));
            float logexpect = logKmn - __fdiv_rn(score, scale);
            if (a.ssemodel == 2) logexpect = logexpect + -9.210340372f;
            float logp = logexpect;
            if (-4.605170186f <= logexpect) {
                if (kLogSpMax - 3.0f < logexpect) logp = 0.0f;
                else {
                    logp = cb_expf(logexpect);
                    if (kLogSpMax - 3.0f < logp) logp = 0.0f;
                    else logp = cb_logf(1.0f - cb_expf(-logp));
                }
            }
            const float lp = l1l2 > 625.0f ? l1l2 : 625.0f;
            const float pn = rintf(__fdiv_rn(100000.0f * psts, cb_powf(lp, 1.5f)));
            const float logpp = lbetaincf(pn + 1.0f, 0.1f, 0.757213f);
            logp = lgammainc_Q(1.346206f, __fdiv_rn(-logp - logpp, 1.485656f));
            logexpect = logp;
            if (-4.605170186f <= logp) {
                logp = cb_expf(logp);
                logexpect = 77.0f;
                if (logp < 1.0f) {
                    logexpect = -cb_logf(1.0f - logp);
                    logexpect = cb_logf(logexpect);
                }
            }
            logexpect = logexpect + cb_logf(__fdiv_rn(a.searchspace, l1l2));
            logE = logexpect;
        }
    }
    out4[0] = lest;
    out4[1] = kest;
    out4[2] = logE;
    out4[3] = epa;
}

// ---- the parameter fit in FP64 (the precision forms)
//
// The same estimation as the FP32 steps below -- expected score, lambda by
// Newton steps guarded by bisection, relative entropy, K by convolution on
// the 21 x 32 grid, with the reference's constants, guards and stopping
// rules -- restated in double precision from the pair's integer histogram.
// exp is the CUDA double-precision exp. Block-wide sums are per row by the
// shuffle-down tree and then over the rows, as in FP32.
struct Fit64 {
    double lambda, K, H, E;   // lambda unscaled, E unscaled
};

__device__ __forceinline__ double wsum_down64(double v)
{
    for (int o = 16; o >= 1; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    return v;
}

// valid in thread 0; all threads call (barriers)
__device__ __forceinline__ double grid_sum64(double v, double* tmp)
{
    const int y = threadIdx.x >> 5, x = threadIdx.x & 31;
    v = wsum_down64(v);
    if (x == 0) tmp[y] = v;
    __syncthreads();
    double t = 0.0;
    if (y == 0) {
        t = (x < NS) ? tmp[x] : 0.0;
        t = wsum_down64(t);
    }
    __syncthreads();
    return t;
}

__device__ Fit64 fit64(const int* cnt, int left, int right, float minscf, float maxscf, int minu, int maxu,
                       double (*g)[33], double* up, double* tmp, double* sh, int* flag)
{
    const int tid = threadIdx.x;
    const int y = tid >> 5, x = tid & 31;
    const double LSMIN = (double)kLogSpMin, LSMAX = (double)kLogSpMax;
    double gv = (x + left <= right) ? (double)cnt[left + x] : 0.0;
    const double scx = (double)(left + x - 320);
    const double minsc = (double)minscf, maxsc = (double)maxscf;
    // probabilities
    {
        const double rs = wsum_down64(gv);
        if (x == 0) tmp[y] = rs;
        __syncthreads();
        if (y == 0) {
            double t = (x < NS) ? tmp[x] : 0.0;
            t = wsum_down64(t);
            if (x == 0) sh[0] = t;
        }
        __syncthreads();
        if (y == 0 && x < NS) up[x] = tmp[x] / sh[0];
        gv = gv / sh[0];
        __syncthreads();
    }
    g[y][x] = gv;
    double E = grid_sum64(scx * gv, tmp);
    if (tid == 0) sh[1] = E;
    __syncthreads();
    E = sh[1];
    // lambda (CuBatchSS_lambda.cuh:80-330)
    double lambda = -1.0;
    if (!(0.0 <= E || maxsc <= 0.0)) {
        auto eq = [&](double lx, double& f, double& df) {
            double lf = 0.0, ldf = 0.0;
            if (minsc <= scx && scx <= maxsc) {
                const double s = scx - maxsc;
                const double yy = lx * s;
                if (LSMIN < yy) { lf = exp(yy) * gv; ldf = lf * s; }
            }
            double F = grid_sum64(lf, tmp);
            double D = grid_sum64(ldf, tmp + 32);
            double xm = lx * -maxsc;
            if (LSMIN < xm) { xm = exp(xm); F = F - xm; D = D + xm * maxsc; }
            f = F;
            df = D;
        };
        const double X1 = 1.0e-5, X2 = 10.0;
        double f, df, fl, dd, dx, dxold, xh, xl, rts;
        eq(X1, fl, dd);
        eq(X2, f, dd);
        if (tid == 0) *flag = (fl > 0.0 && f > 0.0) || (fl < 0.0 && f < 0.0);
        __syncthreads();
        if (!*flag) {
            if (fl < 0.0) { xl = X1; xh = X2; } else { xh = X1; xl = X2; }
            rts = 0.5 * (X1 + X2);
            dxold = fabs(X2 - X1);
            dx = dxold;
            eq(rts, f, df);
            int n;
            for (n = 0; n < 32; n++) {
                __syncthreads();
                if (tid == 0) {
                    int stop = 0;
                    if ((((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0) || (fabs(2.0 * f) > fabs(dxold * df))) {
                        dxold = dx;
                        dx = 0.5 * (xh - xl);
                        rts = xl + dx;
                        if (xl == rts) stop = 1;
                    } else {
                        dxold = dx;
                        dx = f / df;
                        const double temp = rts;
                        rts = rts - dx;
                        if (temp == rts) stop = 1;
                    }
                    if (fabs(dx) < 1.0e-4) stop = 1;
                    *flag = stop;
                    sh[2] = rts;
                }
                __syncthreads();
                rts = sh[2];
                const int stop = *flag;
                __syncthreads();
                if (stop) break;
                eq(rts, f, df);
                if (f < 0.0) xl = rts; else xh = rts;
            }
            lambda = (n == 32) ? -1.0 : rts;
        }
        if (tid == 0) sh[3] = lambda;
        __syncthreads();
        lambda = sh[3];
    }
    // relative entropy (CuBatchSS_entropy.cuh:14-70)
    double H = -1.0;
    if (lambda > 0.0) {
        double e = 0.0;
        if (minsc <= scx && scx <= maxsc) {
            const double yy = lambda * scx;
            if (LSMIN < yy && yy < LSMAX - 3.0) e = exp(yy) * yy * gv;
        }
        H = grid_sum64(e, tmp);
        if (tid == 0) sh[4] = H;
        __syncthreads();
        H = sh[4];
    }
    if (y == 0) g[10][x] = 1.0;
    lambda = lambda * 32.0;
    E = E / 32.0;
    __syncthreads();
    // K (CuBatchSS_K.cuh:49-320)
    double K = -1.0;
    if (!(0.0 <= E || lambda <= 0.0 || H <= 0.0)) {
        if (minu == -1 && maxu == 1) {
            const double minprb = up[-1 + 10], maxprb = up[1 + 10];
            const double d = minprb - maxprb;
            K = d * d / minprb;
        } else if (minu == -1 || maxu == 1) {
            if (maxu != 1) K = (lambda / H) * (1.0 - exp(-lambda)) * (E * E);
            else K = (H / lambda) * (1.0 - exp(-lambda));
        } else {
            const int range = maxu - minu + 1;
            const int isc = left + x - 320;
            double sigma = 0.0, Pj = 1.0;
            int mins = minu, maxs = maxu;
            for (int j = 1; j <= 32 && 1.0e-4 < Pj; j++) {
                double pji = 0.0, pv = 0.0;
                if (mins <= isc && isc <= maxs && -32 <= isc && isc <= 32) {
                    const double etols = isc < 0 ? lambda * (double)isc : 0.0;
                    if (LSMIN < etols) {
                        const int lo = (maxs - isc < range) ? maxu - (maxs - isc) : minu;
                        const int hi = (isc - mins < range) ? minu + (isc - mins) : maxu;
                        for (int i = lo; i <= hi; i++) {
                            int yy = y, xx = x - i;
                            if (32 <= xx) { xx -= 32; if (yy + 1 < NS) yy++; else continue; }
                            else if (xx < 0) { xx += 32; if (0 < yy) yy--; else continue; }
                            pji = fma(g[yy][xx], up[i + 10], pji);
                        }
                        pv = pji * exp(etols);
                    }
                }
                __syncthreads();       // every read of the previous grid is done
                g[y][x] = pji;
                const double P = grid_sum64(pv, tmp);
                if (tid == 0) {
                    sigma = sigma + P / (double)j;
                    sh[5] = P;
                }
                __syncthreads();
                Pj = sh[5];
                mins += minu;
                maxs += maxu;
            }
            if (tid == 0) K = lambda * exp(-2.0 * sigma) / (H * (1.0 - exp(-lambda)));
        }
    }
    return Fit64{lambda, K, H, E};
}

__global__ void __launch_bounds__(kThreads)
stats_kernel(const StatsArgs a)
{
    __shared__ int cnt[NSC];
    __shared__ float g[NS][33];
    __shared__ float up[NS];
    __shared__ float tmp[2 * 32];
    __shared__ float sh[8];
    __shared__ int flag;

    const int tid = threadIdx.x;
    const int y = tid >> 5, x = tid & 31;
    const int k = blockIdx.x;
    const int pl = a.pass_idx[k];
    const int p = a.p0 + pl;
    const int Ld = a.db.plen[p];
    const long long pstart = a.db.pstart[p];
    const long long colb = pstart - a.col0;
    const int Lq = a.Lq;

    // 1. histogram of rint(32 * clamp(score,-10,10)) over the pair's cells
    //    (src/libmycu/cuss/CuBatchSS_dynplm.cu:77-180)
    for (int i = tid; i < NSC; i += kThreads) cnt[i] = 0;
    __syncthreads();
    const long long ncell = (long long)Lq * Ld;
    for (long long idx = tid; idx < ncell; idx += kThreads) {
        const int r = (int)(idx / Ld), c = (int)(idx - (long long)r * Ld);
        if (a.x_uninf && (a.qaa[r] == 'X' || a.db.aa[pstart + c] == 'X')) continue;
        float s = a.scores[(long long)r * a.ld + colb + c];
        s = s < -10.0f ? -10.0f : (s > 10.0f ? 10.0f : s);
        const int bin = (int)rintf(s * 32.0f) + 320;
        atomicAdd(&cnt[bin], 1);
    }
    __syncthreads();

    // 2. grid row y holds histogram indices [left, right]
    //    (src/libmycu/cuss/CuBatchSS_dynplm.cu:199-214)
    const int unscaled = y - 10;
    int left = unscaled * 32 - 16 + 320, right = unscaled * 32 + 16 + 320;
    if (unscaled <= 0) { left++; if (left < 0) left = 0; }
    if (0 <= unscaled) { right--; if (NSC - 1 < right) right = NSC - 1; }
    float gv = (x + left <= right) ? (float)cnt[left + x] : 0.0f;
    const float scx = (float)(left + x - 320);   // scaled score of this cell

    // totals by the xor butterfly (dynplm.cu:224-260)
    float rs = wsum_xor(gv);
    if (x == 0) tmp[y] = rs;
    __syncthreads();
    if (y == 0) {
        float t = (x < NS) ? tmp[x] : 0.0f;
        t = wsum_xor(t);
        if (x < NS) up[x] = __fdiv_rn(tmp[x], t);
        if (x == 0) sh[0] = t;
    }
    __syncthreads();
    gv = __fdiv_rn(gv, sh[0]);
    g[y][x] = gv;
    __syncthreads();

    // 3. expected scaled score (src/libmycu/cuss/CuBatchSS_expected.cuh)
    float E = grid_sum(scx * gv, tmp);
    // 4. min/max scaled score, 0 included (src/libmycu/cuss/CuBatchSS_minmax.cuh)
    {
        const float mn = gv != 0.0f ? scx : 0.0f;
        const float vmin = wmin_down(mn), vmax = wmax_down(mn);
        if (x == 0) { tmp[y] = vmin; tmp[y + 32] = vmax; }
        __syncthreads();
        if (y == 0) {
            float a1 = (x < NS) ? tmp[x] : 0.0f, a2 = (x < NS) ? tmp[x + 32] : 0.0f;
            a1 = wmin_down(a1);
            a2 = wmax_down(a2);
            if (x == 0) { sh[1] = a1; sh[2] = a2; sh[3] = E; }
        }
        __syncthreads();
    }
    const float minsc = sh[1], maxsc = sh[2];
    E = sh[3];

    // 5. lambda by Newton + bisection (src/libmycu/cuss/CuBatchSS_lambda.cuh)
    float lambda = -1.0f;
    if (!(0.0f <= E || maxsc <= 0.0f)) {
        auto eq = [&](float lx, float& f, float& df) {
            float lf = 0.0f, ldf = 0.0f;
            if (minsc <= scx && scx <= maxsc) {
                const float s = scx - maxsc;
                const float yy = lx * s;
                if (kLogSpMin < yy) { lf = cb_expf(yy) * gv; ldf = lf * s; }
            }
            const float F0 = grid_sum(lf, tmp);
            const float D0 = grid_sum(ldf, tmp + 32);
            float F = F0, D = D0;
            float xm = lx * -maxsc;
            if (kLogSpMin < xm) { xm = cb_expf(xm); F = F - xm; D = D + xm * maxsc; }
            f = F;
            df = D;
        };
        const float X1 = 1.0e-5f, X2 = 10.0f;
        float f, df, fl, dfdummy, dx, dxold, xh, xl, rts;
        eq(X1, fl, dfdummy);
        eq(X2, f, dfdummy);
        if (tid == 0) {
            flag = (fl > 0.0f && f > 0.0f) || (fl < 0.0f && f < 0.0f);
            sh[4] = X1;
        }
        __syncthreads();
        if (!flag) {
            if (fl < 0.0f) { xl = X1; xh = X2; } else { xh = X1; xl = X2; }
            rts = 0.5f * (X1 + X2);
            dxold = fabsf(X2 - X1);
            dx = dxold;
            eq(rts, f, df);
            int n;
            for (n = 0; n < 32; n++) {
                if (tid == 0) {
                    int stop = 0;
                    if ((((rts - xh) * df - f) * ((rts - xl) * df - f) > 0.0f) ||
                        (fabsf(2.0f * f) > fabsf(dxold * df))) {
                        dxold = dx;
                        dx = 0.5f * (xh - xl);
                        rts = xl + dx;
                        if (xl == rts) stop = 1;
                    } else {
                        dxold = dx;
                        dx = __fdiv_rn(f, df);
                        const float temp = rts;
                        rts = rts - dx;
                        if (temp == rts) stop = 1;
                    }
                    if (fabsf(dx) < 1.0e-4f) stop = 1;
                    flag = stop;
                    sh[4] = rts;
                }
                __syncthreads();
                rts = sh[4];
                const int stop = flag;
                __syncthreads();
                if (stop) break;
                eq(rts, f, df);
                if (f < 0.0f) xl = rts; else xh = rts;
            }
            lambda = (n == 32) ? -1.0f : rts;
        }
        // broadcast thread 0's value
        if (tid == 0) sh[5] = lambda;
        __syncthreads();
        lambda = sh[5];
    }

    // 6. relative entropy on scaled scores (src/libmycu/cuss/CuBatchSS_entropy.cuh)
    float H = -1.0f;
    if (lambda > 0.0f) {
        float e = 0.0f;
        if (minsc <= scx && scx <= maxsc) {
            const float yy = lambda * scx;
            if (kLogSpMin < yy && yy < kLogSpMax - 3.0f) e = cb_expf(yy) * yy * gv;
        }
        H = grid_sum(e, tmp);
        if (tid == 0) sh[6] = H;
        __syncthreads();
        H = sh[6];
    }

    // rescale; row 10 (score 0) becomes the seed of the K convolution
    if (y == 0) g[10][x] = 1.0f;
    lambda = lambda * 32.0f;
    E = __fdiv_rn(E, 32.0f);
    __syncthreads();

    // 7. unscaled min/max (minmax.cuh:62-99) and K (src/libmycu/cuss/CuBatchSS_K.cuh)
    if (y == 0) {
        const float um = (x < NS && up[x] != 0.0f) ? (float)(x - 10) : 0.0f;
        const float v1 = wmin_down(um), v2 = wmax_down(um);
        if (x == 0) { sh[1] = v1; sh[2] = v2; }
    }
    __syncthreads();
    const float minuf = sh[1], maxuf = sh[2];
    const int minu = (int)minuf, maxu = (int)maxuf;
    float K = -1.0f;
    if (!(0.0f <= E || lambda <= 0.0f || H <= 0.0f)) {
        if (minu == -1 && maxu == 1) {
            const float minprb = up[-1 + 10], maxprb = up[1 + 10];
            const float d = minprb - maxprb;
            K = __fdiv_rn(d * d, minprb);
        } else if (minu == -1 || maxu == 1) {
            if (maxu != 1) K = __fdiv_rn(lambda, H) * (1.0f - cb_expf(-lambda)) * (E * E);
            else K = __fdiv_rn(H, lambda) * (1.0f - cb_expf(-lambda));
        } else {
            const int range = maxu - minu + 1;
            const int isc = left + x - 320;
            float sigma = 0.0f, Pj = 1.0f;
            int mins = minu, maxs = maxu;
            for (int j = 1; j <= 32 && 1.0e-4f < Pj; j++) {
                float pji = 0.0f, pv = 0.0f;
                if (mins <= isc && isc <= maxs && -32 <= isc && isc <= 32) {
                    const float etols = isc < 0 ? lambda * (float)isc : 0.0f;
                    if (kLogSpMin < etols) {
                        const int lo = (maxs - isc < range) ? maxu - (maxs - isc) : minu;
                        const int hi = (isc - mins < range) ? minu + (isc - mins) : maxu;
                        for (int i = lo; i <= hi; i++) {
                            int yy = y, xx = x - i;
                            if (32 <= xx) { xx -= 32; if (yy + 1 < NS) yy++; else continue; }
                            else if (xx < 0) { xx += 32; if (0 < yy) yy--; else continue; }
                            pji = __fmaf_rn(g[yy][xx], up[i + 10], pji);
                        }
                        pv = pji * cb_expf(etols);
                    }
                }
                __syncthreads();       // every read of the previous grid is done
                g[y][x] = pji;
                const float P = grid_sum(pv, tmp);
                if (tid == 0) {
                    sigma = sigma + __fdiv_rn(P, (float)j);
                    sh[7] = P;
                }
                __syncthreads();
                Pj = sh[7];
                mins += minu;
                maxs += maxu;
            }
            if (tid == 0)
                K = __fdiv_rn(lambda * cb_expf(-2.0f * sigma), H * (1.0f - cb_expf(-lambda)));
        }
    }

    // 7b. the precision forms: the fit again in FP64, used for the E-value
    if (a.fits) {
        __shared__ double g64[NS][33];
        __shared__ double up64[NS];
        __shared__ double tmp64[64];
        __shared__ double sh64[8];
        __syncthreads();
        const Fit64 f = fit64(cnt, left, right, minsc, maxsc, minu, maxu, g64, up64, tmp64, sh64, &flag);
        if (tid == 0) {
            double* o = a.fits + (long long)k * kFitDoubles;
            o[0] = f.lambda; o[1] = f.K; o[2] = f.H; o[3] = f.E;
            o[4] = lambda; o[5] = K; o[6] = H; o[7] = E;
            if (a.use_fit64) {
                lambda = (float)f.lambda;
                K = (float)f.K;
                H = (float)f.H;
                E = (float)f.E;
            }
        }
    }

    // 8. significance and the output record (thread 0)
    if (tid == 0) {
        const Dp1Rec r1 = a.recs[pl];
        float o4[4];
        significance(a, Lq, Ld, a.qeno, a.db.eno[p], r1.score, r1.psts, lambda, K, o4);
        float* out = a.out + (long long)k * kRecFloats;
        out[0] = r1.score;
        out[1] = __int_as_float(p);
        out[2] = __int_as_float((int)a.pass_dst[k]);
        out[3] = r1.psts;
        out[4] = __int_as_float((int)r1.beg);
        out[5] = __int_as_float((int)r1.end);
        out[6] = o4[0];
        out[7] = o4[1];
        out[8] = o4[2];
        out[9] = o4[3];
        out[10] = minuf;
        out[11] = maxuf;
        out[12] = E;
        out[13] = H;
        out[14] = lambda;
        out[15] = K;
        out[16] = 0.0f;
        out[17] = 0.0f;
    }
}

}  // namespace

void launch_stats(const StatsArgs& a, int npass, cudaStream_t stream)
{
    if (npass <= 0) return;
    stats_kernel<<<npass, kThreads, 0, stream>>>(a);
    CBP_CHECK_LAUNCH();
}

}  // namespace cbp
