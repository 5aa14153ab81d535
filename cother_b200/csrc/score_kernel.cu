// Batch score matrix: profile-profile + secondary structure + distance
// distribution match score (DDMS) for every (query position, database
// position) cell of a slab, in ONE kernel.
//
// The reference computes the three terms in three kernels that add into the
// output with atomics (src/libmycu/cusco/CuBatchScoreMatrix.cu:236-396:
// CalcSM_Init_SMEMUnroll2x, CalcSM_SSSS_SMEMUnroll2x,
// CalcSM_DDMS2S_SMEMUnroll2x_h2). Here one thread owns one database
// position (lane) and walks a strip of query positions, adding the terms in
// the reference's order -- (init + SS) + DDMS -- and writing each cell once.
//
// DDMS dominates the cost (~550 segment-DP steps per cell for 99-distance
// lists); it is CUDA-core ALU-bound, so the kernel is shaped for issue
// efficiency: byte-packed distance lists brought in by bulk copies and kept
// in shared memory at an odd word stride (conflict-free for lanes in step),
// a 22x22 pair-score table in shared memory, one code path for upper and
// lower diagonals, and the step loop unrolled by four with DSTSEGM as
// compile-time cases.
#include <cmath>
#include "cother_b200.h"
#include "common.cuh"
#include "cbmath.cuh"
#include "layout.h"
#include "score_kernel.cuh"
#include "bulkcopy.cuh"

namespace cbp {

namespace {

constexpr int kCols = 32;          // database positions per block (one per lane)
constexpr int kWarps = 4;
constexpr int kThreads = kCols * kWarps;
constexpr int kElems = 104;        // list elements held per position (99 + overrun)
constexpr int kDbStride = 108;     // bytes per database list in shared memory (27 words)
constexpr int kDbCopy = 112;       // bytes of a list brought in by one bulk copy (and its packed stride)
constexpr int kDbWords = kDbStride / 4;
constexpr unsigned long long kListWaitNs = 1000000000ull;   // the lists' copies: a wait gives up after 1 s

// Top-3 register of non-intersecting segments
// (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s.cuh:182-251). The reference
// packs a segment's coordinates into one word [QB QE PB PE] and tests
// intersection with per-byte SIMD min/max. Here a segment is two words,
// begins (QB<<16 | PB) and ends (QE<<16 | PE), so that the test uses the
// native halfword SIMD min/max of sm_90+: two segments intersect when their
// query OR their database ranges overlap (ddms2s.cuh:162-173), i.e. when
// min(end) >= max(begin) in either halfword; adding 256 to each halfword
// before subtracting keeps both non-negative (positions < 256), so the test
// is whether bits 8..15 of either half are set. The coordinates of an empty
// entry (score 0) are never consulted for a decision, as in the reference.
__device__ __forceinline__ uint32_t vmax_u16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmin_u16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ bool seg_intersect(uint32_t b1, uint32_t e1, uint32_t b2, uint32_t e2)
{
    const uint32_t mx = vmax_u16x2(b1, b2), mn = vmin_u16x2(e1, e2);
    return ((mn + 0x01000100u - mx) & 0xff00ff00u) != 0u;
}
// The update proper, for a candidate s >= ms[2] whose intersection with the
// top entry (x0) is known and that changes the register: s >= ms[0] or not
// x0. Every case of the reference's register tests the candidate against
// the entries at ranks 0 and 1 (an empty entry's test never matters).
__device__ __forceinline__ void register_max(float (&ms)[3], uint32_t (&mb)[3], uint32_t (&me)[3],
                                             float s, uint32_t cb, uint32_t ce, bool x0)
{
    const bool x1 = seg_intersect(cb, ce, mb[1], me[1]);
    if (ms[0] <= s) {
        const float a1 = x0 ? 0.0f : ms[0];
        const float a2 = x1 ? 0.0f : ms[1];
        const bool up = (a1 == 0.0f);
        ms[2] = up ? 0.0f : a2;
        ms[1] = up ? a2 : a1;
        const uint32_t b1 = up ? mb[1] : mb[0], e1 = up ? me[1] : me[0];
        mb[2] = mb[1]; me[2] = me[1];
        mb[1] = b1; me[1] = e1;
        ms[0] = s; mb[0] = cb; me[0] = ce;
    } else if (ms[1] <= s) {          // not x0 here
        ms[2] = x1 ? 0.0f : ms[1]; mb[2] = mb[1]; me[2] = me[1];
        ms[1] = s; mb[1] = cb; me[1] = ce;
    } else if (!x1) {                 // ms[2] <= s, not x0
        ms[2] = s; mb[2] = cb; me[2] = ce;
    }
}

// Saturating add/multiply: the result clamped to [0, 1] in one FMA-pipe
// instruction.
__device__ __forceinline__ float sat_add(float a, float b)
{
    float r;
    asm("add.sat.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float sat_mul(float a, float b)
{
    float r;
    asm("mul.sat.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float sat_fma(float a, float b, float c)
{
    float r;
    asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// smallest positive float: the register filter's threshold while its third
// entry is empty (every positive candidate is at least this)
constexpr float kTiny = 0x1p-149f;

// One diagonal of the DDMS segment DP. Elements e = 0,1,... pair query list
// element oq+e with database list element od+e (upper diagonals: oq = 0,
// od = j; lower: oq = i, od = 0). The lists hold their codes pre-multiplied
// into byte offsets of the pair-score table T (query: code x 88, a row of
// 22 floats; database: code x 4), so a pair score is one add and one load. Pair scores at even offsets within each
// 4-step are table values, odd ones the mean of their neighbours
// (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:184-198); a segment
// restarts when the running sum has fallen to zero, and the best segment of
// length >= DSTSEGM ending in each 4-step is offered to the top-3 register
// (ddms2s_h2.cuh:124-176, 288-396).
//
// The pair scores come pre-scaled by 2^-7, so every running sum stays in
// [0, 1) and max(sum, 0) is one saturating add; scaling by a power of two
// commutes exactly with IEEE rounding, so the sums are the reference's
// times 2^-7, bit for bit. An odd element's mean 0.5*(a+b) is exact once a+b
// is rounded, so adding it is one saturating fma(0.5, a+b, sum). The segment length is a small exact float:
// len_k = len_{k-1} * [sum_{k-1} > 0] + 1, the indicator being
// sat(sum * 2^100) (every positive sum here is far above 2^-100). A step's
// candidate is max_k sum_k * [len_k >= DSTSEGM] and sits at the first k that
// attains it, which is the reference's strict "<" scan. `thr` is
// max(third entry's score, kTiny): a candidate below it changes nothing.
// kLongSegments: DSTSEGM >= 5 (the default is 6), a compile-time case so
// that the candidate's begin needs no run-time test in the step loop
// (measured 1.9 % faster than the uniform branch).
template <bool kLongSegments>
__device__ __forceinline__ void ddms_diagonal(
    const uint16_t* __restrict__ q, const uint8_t* __restrict__ d,
    const char* __restrict__ T, int lim, int oq, int od, float nsegm1,
    float (&ms)[3], uint32_t (&mb)[3], uint32_t (&me)[3], float& thr)
{
    constexpr float kBig = 0x1p100f;
    float s0 = *reinterpret_cast<const float*>(T + q[0] + d[0]);
    float t = sat_add(s0, 0.0f);
    float ls = 1.0f;
    const uint32_t cbase = ((uint32_t)oq << 16) | (uint32_t)od;
    // four steps per iteration (measured: 2.2 % faster than the compiler's
    // own choice, 3.6 % slower with two, 12 % slower with eight)
#pragma unroll 4
    for (int x = 0; x < lim; x += 4) {
        const float s2 = *reinterpret_cast<const float*>(T + q[x + 2] + d[x + 2]);
        const float s4 = *reinterpret_cast<const float*>(T + q[x + 4] + d[x + 4]);
        const float l1 = __fmaf_rn(ls, sat_mul(t, kBig), 1.0f);
        const float t1 = sat_fma(0.5f, s0 + s2, t);
        const float l2 = __fmaf_rn(l1, sat_mul(t1, kBig), 1.0f);
        const float t2 = sat_add(t1, s2);
        const float l3 = __fmaf_rn(l2, sat_mul(t2, kBig), 1.0f);
        const float t3 = sat_fma(0.5f, s2 + s4, t2);
        const float l4 = __fmaf_rn(l3, sat_mul(t3, kBig), 1.0f);
        const float t4 = sat_add(t3, s4);
        const float v1 = t1 * sat_add(l1, nsegm1);
        const float v2 = t2 * sat_add(l2, nsegm1);
        const float v3 = t3 * sat_add(l3, nsegm1);
        const float v4 = t4 * sat_add(l4, nsegm1);
        const float scom = fmaxf(fmaxf(v1, v2), fmaxf(v3, v4));
        // the register is sorted by score, so a candidate below its third
        // entry changes nothing (every branch of register_max fails)
        if (thr <= scom) {
            const int k = (v1 == scom) ? 1 : (v2 == scom) ? 2 : (v3 == scom) ? 3 : 4;
            const uint32_t be = (uint32_t)(x + k);
            uint32_t bb;
            if (kLongSegments) {
                // DSTSEGM >= 5: the candidate, at least 5 long and ending at
                // x+k <= x+4, contains element x, so it is the segment running
                // at x, which began at x + 1 - ls
                bb = (uint32_t)(x + 1) - (uint32_t)ls;
            } else {
                const float lk = (v1 == scom) ? l1 : (v2 == scom) ? l2 : (v3 == scom) ? l3 : l4;
                bb = be + 1u - (uint32_t)lk;
            }
            const uint32_t cb = cbase + bb * 0x00010001u, ce = cbase + be * 0x00010001u;
            // below the top entry and intersecting it, a candidate changes
            // nothing (the reference's second and third cases both require
            // no intersection with the top); most candidates end here
            const bool x0 = seg_intersect(cb, ce, mb[0], me[0]);
            if (ms[0] <= scom || !x0) {
                register_max(ms, mb, me, scom, cb, ce, x0);
                thr = fmaxf(ms[2], kTiny);
            }
        }
        s0 = s4;
        t = t4;
        ls = l4;
    }
}

// DDMS of one cell (src/libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh:433-500).
// Returns the top-3 sum in the reference's scale.
__device__ __forceinline__ float ddms_cell(const uint16_t* __restrict__ q, int len1,
                                           const uint8_t* __restrict__ d, int len2,
                                           const char* __restrict__ T, int dstsegm)
{
    float ms[3] = {0.0f, 0.0f, 0.0f};
    uint32_t mb[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
    uint32_t me[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
    const float nsegm1 = -(float)(dstsegm - 1);
    float thr = kTiny;
    if (dstsegm == 6) {
        // the default DSTSEGM with its constant in the instructions (0.8 % faster)
        for (int j = len2 >> 2; 0 <= j; j -= 2)
            ddms_diagonal<true>(q, d + j, T, min(len1, len2 - j), 0, j, -5.0f, ms, mb, me, thr);
        for (int i = len1 >> 2; 0 < i; i -= 2)
            ddms_diagonal<true>(q + i, d, T, min(len2, len1 - i), i, 0, -5.0f, ms, mb, me, thr);
    } else if (dstsegm >= 5) {
        for (int j = len2 >> 2; 0 <= j; j -= 2)
            ddms_diagonal<true>(q, d + j, T, min(len1, len2 - j), 0, j, nsegm1, ms, mb, me, thr);
        for (int i = len1 >> 2; 0 < i; i -= 2)
            ddms_diagonal<true>(q + i, d, T, min(len2, len1 - i), i, 0, nsegm1, ms, mb, me, thr);
    } else {
        for (int j = len2 >> 2; 0 <= j; j -= 2)
            ddms_diagonal<false>(q, d + j, T, min(len1, len2 - j), 0, j, nsegm1, ms, mb, me, thr);
        for (int i = len1 >> 2; 0 < i; i -= 2)
            ddms_diagonal<false>(q + i, d, T, min(len2, len1 - i), i, 0, nsegm1, ms, mb, me, thr);
    }
    float sum = 0.0f;
    sum = sum + ms[0];
    sum = sum + ms[1];
    sum = sum + ms[2];
    return sum * 128.0f;
}

// Context-vector term of one cell (CalcCVS2ScoreSMEMUnroll2x,
// src/libmycu/cusco/CuBatchScoreMatrix_cvs2s.cuh:47-136): the log-odds of
// the two normal vectors, log det(C2 + H'H) from their dot product and
// squared norms less both log priors, translated through the map
// (SerializedCVS2Scores::GetScoreE1S1Step2Boundary,
// src/libmycu/cupro/SerializedCVS2Scores.cuh:377-410). The dot product, the
// determinant and the log-odds are fused multiply-adds and the logarithm is
// the __logf intrinsic, as in the reference's build. A log-odds that is
// not above the first key (a NaN included) takes the first score.
__device__ __forceinline__ float cvs_cell(const ScoreArgs& a, const float* __restrict__ qcv, float qprior,
                                          float qnorm2, const float (*__restrict__ dcv)[kCols], int lane,
                                          float dprior, float dnorm2)
{
    float dot = 0.0f;
#pragma unroll
    for (int i = 0; i < kNCV; i++) dot = __fmaf_rn(qcv[i], dcv[i][lane], dot);
    dot = dot + a.cvs_lokappa0;
    const float qa = qnorm2 + 1.0f + a.cvs_lokappa0;
    const float da = dnorm2 + 1.0f + a.cvs_lokappa0;
    const float det = __fmaf_rn(qa, da, -(dot * dot));
    if (a.cvs_int_priors) {   // FtorRoundMAPALN0 (CuBatchScoreMatrix_cvs2s.cuh:38-41)
        qprior = (float)(int)qprior;
        dprior = (float)(int)dprior;
    }
    const float lo = __fmaf_rn(a.cvs_pownu0, __logf(det), a.cvs_cterm) - qprior - dprior;
    if (!(a.cvs_key_first < lo)) return __ldg(a.cvs_scores);
    if (a.cvs_key_last <= lo) return __ldg(a.cvs_scores + a.cvs_card - 1);
    return __ldg(a.cvs_scores + a.cvs_shift + (int)rintf(lo + lo));
}

// kRows query positions per block (8, 16 or 32; each warp takes every
// kWarps-th of them), chosen by the tuner. kStacked: the rows belong to
// several queries (cbp_process_batch), each with its own background; a
// separate instantiation, so that the single-query kernel is unchanged.
template <int kRows, bool kStacked>
__global__ void __launch_bounds__(kThreads, 10)
score_matrix_kernel(const ScoreArgs a)
{
    __shared__ float s_dms[kDstCard * kDstCard];
    __shared__ float s_sst[kSSCard * kSSCard];
    // the distance lists: first packed at kDbCopy bytes as the bulk copies
    // leave them, then at the odd stride kDbStride with the codes times 4
    __shared__ __align__(16) uint8_t s_dbe[kCols * kDbCopy];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ __align__(16) uint16_t s_qe[kRows * kElems];
    __shared__ float s_dtf[kNAA][kCols];
    __shared__ float s_dbg[kNAA][kCols];
    __shared__ float s_dss[kNSS][kCols];
    __shared__ float s_qtf[kRows][kNAA + 1];
    __shared__ float s_qss[kRows][kNSS];
    __shared__ int s_dlen[kCols];
    __shared__ int s_qlen[kRows];
    // context vectors and their log priors and squared norms (CVSWGT > 0):
    // dynamic shared memory, absent otherwise, so that ten blocks fit an SM
    extern __shared__ float s_cvsdyn[];
    float (*s_dcv)[kCols] = reinterpret_cast<float (*)[kCols]>(s_cvsdyn);
    float (*s_dcvpn)[kCols] = reinterpret_cast<float (*)[kCols]>(s_cvsdyn + kNCV * kCols);
    float (*s_qcv)[kNCV + 1] = reinterpret_cast<float (*)[kNCV + 1]>(s_cvsdyn + (kNCV + 2) * kCols);
    float (*s_qcvpn)[kRows] =
        reinterpret_cast<float (*)[kRows]>(s_cvsdyn + (kNCV + 2) * kCols + kRows * (kNCV + 1));
    __shared__ int s_col[kCols];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int colb = blockIdx.x * kCols;
    const int rowb = blockIdx.y * kRows;
    const long long N = a.db.N;

    if (tid < kCols) {
        const int slot = colb + tid;
        s_col[tid] = slot < a.ncols ? (a.colorder ? a.colorder[slot] : slot) : -1;
    }
    const bool ddms = a.ddmswgt > 0.0f;
    for (int i = tid; ddms && i < kDstCard * kDstCard; i += kThreads) s_dms[i] = a.dmstab[i] * 0x1p-7f;
    for (int i = tid; i < kSSCard * kSSCard; i += kThreads) s_sst[i] = a.sstab[i];
    if (ddms && tid == 0) {
        mbar_init(&s_bar);
        mbar_init_fence();
    }
    __syncthreads();

    // the block's distance lists (DDMS only): one bulk copy per column,
    // bytes 0..111 of its 128-byte list (this GPU's memory, 128-byte
    // aligned) into s_dbe at a 112-byte stride, in flight while the
    // column fields and the query rows below are read
    if (ddms && warp == 0) {
        const int cc = s_col[lane];
        const unsigned ncopy = __popc(__ballot_sync(0xffffffffu, cc >= 0));
        if (lane == 0) mbar_expect_tx(&s_bar, ncopy * (unsigned)kDbCopy);
        __syncwarp();
        if (cc >= 0) bulk_load(s_dbe + lane * kDbCopy, a.db.dst + (a.col0 + cc) * kDstStride, kDbCopy, &s_bar);
    }

    // database columns of this block: lane l takes slab column s_col[l]
    const int col = s_col[lane];
    const bool cvalid = col >= 0;
    const long long gpos = a.col0 + col;
    if (cvalid) {
        const int p = a.db.pro[gpos];
        for (int k = warp; k < kNAA; k += kWarps) {
            s_dtf[k][lane] = a.db.tf[(long long)k * N + gpos];
            // one query: the denominator 0.5*(query bkg + profile bkg) of
            // the column, rounded as in the cell loop; stacked queries: the
            // profile's background alone
            const float b = a.db.bkg[(long long)k * a.db.P + p];
            s_dbg[k][lane] = kStacked ? b : 0.5f * (__ldg(a.q.bkg + k) + b);
        }
        if (warp < kNSS) s_dss[warp][lane] = a.db.ss[(long long)warp * N + gpos];
        if (warp == kNSS) s_dlen[lane] = a.db.dstlen[gpos];
    } else if (warp == kNSS) {
        s_dlen[lane] = 0;
    }
    // query rows of this block
    for (int idx = tid; idx < kRows * kNAA; idx += kThreads) {
        const int r = idx / kNAA, k = idx - r * kNAA;
        const int row = rowb + r;
        s_qtf[r][k] = row < a.Lq ? a.q.tf[(long long)k * a.q.N + row] : 0.0f;
    }
    for (int idx = tid; idx < kRows * kNSS; idx += kThreads) {
        const int r = idx / kNSS, k = idx - r * kNSS;
        const int row = rowb + r;
        s_qss[r][k] = row < a.Lq ? a.q.ss[(long long)k * a.q.N + row] : 0.0f;
    }
    if (a.cvswgt > 0.0f) {
        if (cvalid) {
            for (int k = warp; k < kNCV; k += kWarps) s_dcv[k][lane] = a.db.cv[(long long)k * N + gpos];
            if (warp == 0) {
                s_dcvpn[0][lane] = a.db.cvprior[gpos];
                s_dcvpn[1][lane] = a.db.cvnorm2[gpos];
            }
        }
        for (int idx = tid; idx < kRows * kNCV; idx += kThreads) {
            const int r = idx / kNCV, k = idx - r * kNCV;
            const int row = rowb + r;
            s_qcv[r][k] = row < a.Lq ? a.q.cv[(long long)k * a.q.N + row] : 0.0f;
        }
        if (tid < kRows) {
            const int row = rowb + tid;
            s_qcvpn[0][tid] = row < a.Lq ? a.q.cvprior[row] : 0.0f;
            s_qcvpn[1][tid] = row < a.Lq ? a.q.cvnorm2[row] : 0.0f;
        }
    }
    if (tid < kRows) s_qlen[tid] = (rowb + tid < a.Lq) ? a.q.dstlen[rowb + tid] : 0;
    // query lists: each code times 88, the byte offset of its table row
    for (int idx = tid; ddms && idx < kRows * (kElems / 4); idx += kThreads) {
        const int r = idx / (kElems / 4), w = idx - r * (kElems / 4);
        const int row = rowb + r;
        uint32_t v = 0x15151515u;
        if (row < a.Lq) v = *reinterpret_cast<const uint32_t*>(a.q.dst + (long long)row * kDstStride + 4 * w);
        uint16_t* o = s_qe + r * kElems + 4 * w;
        o[0] = (uint16_t)((v & 0xffu) * (kDstCard * 4));
        o[1] = (uint16_t)(((v >> 8) & 0xffu) * (kDstCard * 4));
        o[2] = (uint16_t)(((v >> 16) & 0xffu) * (kDstCard * 4));
        o[3] = (uint16_t)((v >> 24) * (kDstCard * 4));
    }
    if (ddms) {
        // the lists' copies: a wait that gives up flags the launch, waits
        // once more for the copies still in flight into this block's
        // shared memory, and ends the block without writing
        const bool got = mbar_wait_for(&s_bar, 0, kListWaitNs);
        if (__syncthreads_or(!got)) {
            if (tid == 0 && a.err) atomicExch(a.err, 2);
            (void)mbar_wait_for(&s_bar, 0, kListWaitNs);
            return;
        }
        // to the odd stride, each code times 4 (a byte offset in a row of
        // the pair-score table; codes <= 21, so the shift never carries
        // across bytes); a slot without a column reads as no data
        constexpr int kPer = (kCols * kDbWords + kThreads - 1) / kThreads;
        const uint32_t* src = reinterpret_cast<const uint32_t*>(s_dbe);
        uint32_t w[kPer];
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const int idx = tid + k * kThreads;
            const int c = idx / kDbWords, wd = idx - c * kDbWords;
            w[k] = 0x15151515u;   // kDstNoData in every byte
            if (idx < kCols * kDbWords && s_col[c] >= 0) w[k] = src[c * (kDbCopy / 4) + wd];
        }
        __syncthreads();
        uint32_t* dstw = reinterpret_cast<uint32_t*>(s_dbe);
#pragma unroll
        for (int k = 0; k < kPer; k++) {
            const int idx = tid + k * kThreads;
            if (idx < kCols * kDbWords) dstw[idx] = w[k] << 2;
        }
    }
    __syncthreads();

    if (!cvalid) return;  // no block-wide synchronisation below

    const int dlen = s_dlen[lane];
    const uint8_t* de = s_dbe + lane * kDbStride;
    const float dss0 = s_dss[0][lane], dss1 = s_dss[1][lane], dss2 = s_dss[2][lane];

    for (int r = warp; r < kRows; r += kWarps) {
        const int row = rowb + r;
        if (row >= a.Lq) break;

        // profile-profile term (CuBatchScoreMatrix_Init.cu:159-186)
        float acc = 0.0f;
        if (a.dots_in_scores) {
            acc = a.scores[(long long)row * a.ld + col];
        } else if (!kStacked) {
#pragma unroll
            for (int k = 0; k < kNAA; k++) {
                const float num = s_qtf[r][k] * s_dtf[k][lane];
                acc = acc + __fdiv_rn(num, s_dbg[k][lane]);
            }
        } else {
            // stacked queries: the background of this row's query
            const float* __restrict__ qbg = a.q.bkg + a.q.pro[row];
#pragma unroll
            for (int k = 0; k < kNAA; k++) {
                const float num = s_qtf[r][k] * s_dtf[k][lane];
                const float den = 0.5f * (__ldg(qbg + (long long)k * a.q.P) + s_dbg[k][lane]);
                acc = acc + __fdiv_rn(num, den);
            }
        }
        float s = cb_logf(acc) - a.initshift;
        float mod = 0.0f;
        const float cvs = (a.cvswgt > 0.0f)
                              ? cvs_cell(a, s_qcv[r], s_qcvpn[0][r], s_qcvpn[1][r], s_dcv, lane,
                                         s_dcvpn[0][lane], s_dcvpn[1][lane])
                              : 0.0f;

        // SS term (CuBatchScoreMatrix_ssss.cu:209-279)
        if (a.ssswgt > 0.0f) {
            float ss = 0.0f;
            const float dsv[3] = {dss0, dss1, dss2};
#pragma unroll
            for (int i = 0; i < kNSS; i++) {
                const float f1 = s_qss[r][i];
                const int ri = i * 10 + (int)(f1 * 9.999f);
#pragma unroll
                for (int j = 0; j < kNSS; j++) {
                    const float f2 = dsv[j];
                    const int cj = j * 10 + (int)(f2 * 9.999f);
                    ss = __fmaf_rn(f1 * f2, s_sst[ri * kSSCard + cj], ss);
                }
            }
            if (-99.0f < ss) {
                ss = __fmaf_rn((s_qss[r][2] + 0.1f) * (dss2 + 0.1f), 0.1111111f, ss);
                ss = ss - 0.05f;
                ss = ss * a.ssswgt;
            }
            if (a.cvswgt > 0.0f) {
                // SS plus the weighted CVS term, the modular score 0.5*CVSWGT
                // lower (CuBatchScoreMatrix_ssss_cvs2s.cu:252-270). That
                // kernel computes chunk columns c and c+32 of each 64-column
                // block in one thread, and its build fuses the addition for
                // the first (one rounding) but not for the second.
                ss = ((gpos >> 5) & 1) ? ss + cvs * a.cvswgt : __fmaf_rn(cvs, a.cvswgt, ss);
                s = s + ss;
                mod = ss - 0.5f * a.cvswgt;
            } else {
                s = s + ss;
                mod = ss;
            }
        } else if (a.cvswgt > 0.0f && cvs != 0.0f) {
            // CVS alone (CuBatchScoreMatrix_cvs2s.cu:286-299); the modular
            // score starts at zero
            s = s + cvs * a.cvswgt;
            mod = mod + (cvs - 0.5f) * a.cvswgt;
        }

        // DDMS term (CuBatchScoreMatrix_ddms2s_h2.cu:158-186)
        if (a.ddmswgt > 0.0f) {
            const int qlen = s_qlen[r];
            if (qlen >= a.dstsegm && dlen >= a.dstsegm) {
                const float sum = ddms_cell(s_qe + r * kElems, qlen, de, dlen,
                                            reinterpret_cast<const char*>(s_dms), a.dstsegm);
                const float dm = __fmaf_rn(0.053f * 16.0f, sum, -1.235f) * a.ddmswgt;
                if (dm != 0.0f) {
                    // the modular score drops 0.2*DDMSWGT, in the contracted
                    // form of CuBatchScoreMatrix_ddms2s_h2.cu:171
                    s = s + dm;
                    mod = mod + __fmaf_rn(-0.2f, a.ddmswgt, dm);
                }
            }
        }
        const long long o = (long long)row * a.ld + col;
        a.scores[o] = s;
        a.modscores[o] = mod;
    }
}

}  // namespace

// One block per window: a counting sort of the window's columns by
// descending list length (0..kMaxDst). The order within one length is
// arbitrary: it decides only which lane computes a cell, never its value.
__global__ void __launch_bounds__(256)
column_order_kernel(const uint8_t* __restrict__ dstlen, long long col0, int ncols, long long ld, int window,
                    int* __restrict__ order)
{
    __shared__ int s_cnt[kMaxDst + 1];
    const int w0 = blockIdx.x * window;
    const int n = min(window, ncols - w0);
    for (int i = threadIdx.x; i <= kMaxDst; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        atomicAdd(&s_cnt[kMaxDst - min((int)dstlen[col0 + w0 + i], kMaxDst)], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int b = 0; b <= kMaxDst; b++) {
            const int c = s_cnt[b];
            s_cnt[b] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int b = kMaxDst - min((int)dstlen[col0 + w0 + i], kMaxDst);
        order[w0 + atomicAdd(&s_cnt[b], 1)] = w0 + i;
    }
    // slots past the last column (the final window only)
    for (long long i = (long long)w0 + n + threadIdx.x; i < min(ld, (long long)w0 + window);
         i += blockDim.x)
        order[i] = -1;
}

void launch_column_order(const uint8_t* dstlen, long long col0, int ncols, long long ld, int window, int* order,
                         cudaStream_t stream)
{
    if (ncols <= 0) return;
    if (window < 32 || window > kMaxOrderWindow || window % 32)
        throw Error(CBP_ERR_ARG, "column order window must be a multiple of 32 in [32, 4096]");
    column_order_kernel<<<(unsigned)ceil_div(ncols, window), 256, 0, stream>>>(dstlen, col0, ncols, ld, window,
                                                                               order);
    CBP_CHECK_LAUNCH();
}

template <int kRows>
void launch_score_rows(const ScoreArgs& a, cudaStream_t stream)
{
    dim3 grid((unsigned)ceil_div(a.ncols, kCols), (unsigned)ceil_div(a.Lq, kRows));
    const size_t cvs_smem =
        a.cvswgt > 0.0f ? sizeof(float) * ((kNCV + 2) * kCols + kRows * (kNCV + 1) + 2 * kRows) : 0;
    if (a.q.P > 1) score_matrix_kernel<kRows, true><<<grid, kThreads, cvs_smem, stream>>>(a);
    else score_matrix_kernel<kRows, false><<<grid, kThreads, cvs_smem, stream>>>(a);
    CBP_CHECK_LAUNCH();
}

void launch_score_matrix(const ScoreArgs& a, cudaStream_t stream)
{
    if (a.ncols <= 0 || a.Lq <= 0) return;
    switch (a.rows) {
    case 8: launch_score_rows<8>(a, stream); break;
    case 16: launch_score_rows<16>(a, stream); break;
    case 32: launch_score_rows<32>(a, stream); break;
    default: throw Error(CBP_ERR_ARG, "score kernel rows per block must be 8, 16 or 32");
    }
}

// Pair-score table over packed distance codes (0..20 saturated, 21 = no
// data), computed on the host (constants
// src/libmycu/cupro/SerializedDstMatchScoresAttr.h:29-31, formula
// src/libmycu/cupro/SerializedDstMatchScores.cuh:347-396). With d1 >= d2 the
// reference's CUDA build evaluates intercept = 0.35 - (d2*-0.4)*0.05 and
// score = d1*slope + intercept as two fused multiply-adds (nvcc contracts
// them by default), so the table does the same with fmaf.
void build_dms_table(float* T)
{
    volatile float s00 = 0.35f, s200 = -0.4f, inv = 0.05f;
    for (int a1 = 0; a1 < kDstCard; a1++)
        for (int a2 = 0; a2 < kDstCard; a2++) {
            if (a1 == kDstNoData || a2 == kDstNoData) { T[a1 * kDstCard + a2] = -1.0f; continue; }
            int d1 = a1 > a2 ? a1 : a2, d2 = a1 > a2 ? a2 : a1;
            volatile float t = (float)d2 * s200;
            volatile float intpt = std::fmaf(-t, inv, s00);
            volatile float sl0 = s200 - s00;
            volatile float slope = sl0 * inv;
            T[a1 * kDstCard + a2] = std::fmaf((float)d1, slope, intpt);
        }
}

}  // namespace cbp
