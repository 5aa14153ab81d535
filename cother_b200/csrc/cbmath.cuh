// Arithmetic shared by the kernels that must agree with the CPU oracle
// operation by operation. The library is compiled with --fmad=false, so a
// multiply-add is fused only where __fmaf_rn is written.
#pragma once

#include <stdint.h>

namespace cbp {

// Natural logarithm of a positive finite float: x = m * 2^e with m in
// [sqrt(1/2), sqrt(2)), t = (m-1)/(m+1), log(m) = 2*atanh(t) summed as the
// odd series 2(t + t^3/3 + t^5/5 + t^7/7 + t^9/9) (|t| <= 0.1716; the first
// omitted term is below 1e-9 relative); log(x) = e*ln2 + log(m) with ln2
// split in a 16-bit head and a tail. Every step is a correctly rounded IEEE
// operation, so the result is identical on any IEEE machine evaluating the
// same sequence (max error measured at 1.7 ulp against a double-precision
// log).
__host__ __device__ __forceinline__ float cb_logf(float x)
{
    union { float f; uint32_t u; } v;
    v.f = x;
    int e = 0;
    if (v.u < 0x00800000u) {
        v.f = x * 8388608.0f;
        e = -23;
    }
    e += (int)((v.u >> 23) & 0xffu) - 127;
    v.u = (v.u & 0x007fffffu) | 0x3f800000u;
    float m = v.f;
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
#ifdef __CUDA_ARCH__
    float t = __fdiv_rn(m - 1.0f, m + 1.0f);
    float t2 = t * t;
    float p = __fmaf_rn(t2, 0.11111111f, 0.14285715f);
    p = __fmaf_rn(t2, p, 0.2f);
    p = __fmaf_rn(t2, p, 0.33333334f);
    float t2x = t + t;
    float lm = __fmaf_rn(t2x * t2, p, t2x);
    float fe = (float)e;
    return __fmaf_rn(fe, 0.693145751953125f, __fmaf_rn(fe, 1.42860677e-06f, lm));
#else
    float t = (m - 1.0f) / (m + 1.0f);
    float t2 = t * t;
    float p = __builtin_fmaf(t2, 0.11111111f, 0.14285715f);
    p = __builtin_fmaf(t2, p, 0.2f);
    p = __builtin_fmaf(t2, p, 0.33333334f);
    float t2x = t + t;
    float lm = __builtin_fmaf(t2x * t2, p, t2x);
    float fe = (float)e;
    return __builtin_fmaf(fe, 0.693145751953125f, __builtin_fmaf(fe, 1.42860677e-06f, lm));
#endif
}

// a < b ? b : a, the reference's max (src/libmycu/cucom/cucommon.h:62);
// written out so that signed zeros and NaNs behave as there.
__host__ __device__ __forceinline__ float hmax(float a, float b) { return a < b ? b : a; }
__host__ __device__ __forceinline__ float hmin(float a, float b) { return a < b ? a : b; }

// exp of a float: x = k*ln2 + r with k = rint(x*log2(e)) and ln2 split in
// a 16-bit head and a tail (Cody-Waite), exp(r) by its Taylor series to
// r^7/7! (|r| <= ln2/2, truncation below 6e-9 relative), scaled by 2^k
// built from two exact powers of two. Measured within 1 ulp of exp().
__device__ __forceinline__ float cb_expf(float x)
{
    if (x != x) return x;
    if (!(x < 88.7228f)) return __int_as_float(0x7f800000);
    if (x < -103.972f) return 0.0f;
    const float kf = rintf(x * 1.44269504f);
    float r = __fmaf_rn(kf, -0.693145751953125f, x);
    r = __fmaf_rn(kf, -1.42860677e-06f, r);
    float p = 1.98412698e-04f;
    p = __fmaf_rn(p, r, 1.38888889e-03f);
    p = __fmaf_rn(p, r, 8.33333333e-03f);
    p = __fmaf_rn(p, r, 4.16666667e-02f);
    p = __fmaf_rn(p, r, 1.66666667e-01f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    const int k = (int)kf;
    const int k1 = k / 2, k2 = k - k1;
    const float s1 = __int_as_float((k1 + 127) << 23);
    const float s2 = __int_as_float((k2 + 127) << 23);
    return (p * s1) * s2;
}

// log-gamma for x > 0: x shifted up to >= 8 while accumulating the product
// of the shifts, then Stirling's series (x-1/2)log x - x + log(2 pi)/2 +
// 1/(12x) - 1/(360x^3) + 1/(1260x^5) - 1/(1680x^7).
__device__ __forceinline__ float cb_lgammaf(float x)
{
    float prod = 1.0f;
    for (int i = 0; i < 64 && x < 8.0f; i++) { prod = prod * x; x = x + 1.0f; }
    const float lx = cb_logf(x);
    const float ix = __fdiv_rn(1.0f, x);
    const float ix2 = ix * ix;
    const float ser = __fmaf_rn(ix2, __fmaf_rn(ix2, __fmaf_rn(ix2, -5.95238095e-04f, 7.93650794e-04f),
                                               -2.77777778e-03f), 8.33333333e-02f) * ix;
    float r = __fmaf_rn(x - 0.5f, lx, -x);
    r = r + 0.918938533f;
    r = r + ser;
    return r - cb_logf(prod);
}

__device__ __forceinline__ float cb_powf(float x, float y) { return cb_expf(y * cb_logf(x)); }

}  // namespace cbp
