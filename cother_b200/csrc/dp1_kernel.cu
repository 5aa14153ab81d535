// Phase-1 gapped local alignment: 5-state (MM, MI, IM, DN, ND) max-plus DP
// with one backtrack byte per cell, its finalization (maximum, backtrace,
// correlation bonus, threshold) and a deterministic pass list.
//
// Reference: ExecDP_Btck_Unroll32x (src/libmycu/cudp/CuBatchDP_init_btck.cu:65-494),
// launched once per block diagonal by the host (src/libmycu/cudp/CuBatchDP.cu:260-312);
// FinalizeDPPro (src/libmycu/cudp/CuBatchDP_final.cu:61-292) with a device
// spin-lock + atomicAdd pass list.
//
// Here one warp owns one database profile for the whole DP: it sweeps bands
// of 32 query rows, lane t holding row r0+t, along anti-diagonals (lane t is
// at column s-t at step s). "Up" and "diagonal" states arrive from lane t-1
// by shuffle; lane 0 reads the bottom row of the previous band from a
// per-profile global strip that lane 31 writes. One launch covers every
// profile of a slab (no per-diagonal launches, no grid-wide syncs).
#include "cother_b200.h"
#include "common.cuh"
#include "cbmath.cuh"
#include "dp1_kernel.cuh"

namespace cbp {

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr float kLog0 = -32768.0f;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ int corner_edge(int Lq, int Ld)
{
    const int mx = Lq > Ld ? Lq : Ld;
    const int e = (int)rintf(0.34f * (float)mx);
    return e > 60 ? 60 : e;
}

__device__ __forceinline__ bool in_corner(int Lq, int Ld, int edge, int r, int c)
{
    return (Lq <= r + edge && c <= edge + r - Lq) || (Ld - edge + r <= c && r < edge);
}

// Score tiles and backtrack codes are staged through shared memory so that
// every global access is a row segment: a band's columns are taken in
// chunks of 32; chunk k+1's 32x32 score tile is fetched with cp.async while
// the warp sweeps chunk k (a ring of three tiles: step s touches columns
// s-31..s), and chunk k's backtrack codes are written back row by row once
// lane 31 has passed the chunk. Row-major [row][32] tiles are free of bank
// conflicts both for the row-wise fill (lane t writes column t) and for the
// anti-diagonal reads (lane t reads row t, column s-t: bank (s-t) mod 32);
// so are the byte tiles of backtrack codes (bank 8*(t mod 4) + a distinct
// quarter-column per lane).
constexpr int kChunk = 32;              // columns per staged chunk
constexpr int kScoreRing = 3;           // score tiles in flight per warp
constexpr int kBtckRing = 2;            // backtrack tiles per warp

// per chunk of 32 columns: the score tile, the profile transitions of the
// chunk's columns (MI and II from the next column's entry, as the DP reads
// them) and, for bands below the first, the previous band's bottom row from
// the strip; all fetched with cp.async one chunk ahead, so that no step
// waits on a global load
struct DpStage {
    float sc[kScoreRing][32][kChunk];
    float tr[kScoreRing][kNTrn][kChunk];
    float sp[kScoreRing][5][kChunk];
    uint8_t bt[kBtckRing][32][kChunk];
};

__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = valid ? 4 : 0;   // 0: fill with zeros, read nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// issue the loads of chunk k for the band of rows r0..r0+31: its score
// tile (zero outside the matrix), the transitions of its columns and, below
// the first band, the strip (the previous band's bottom row)
__device__ __forceinline__ void fetch_chunk(DpStage& st, const float* __restrict__ S, long long ld,
                                            int r0, int Lq, int Ld, int k, int lane,
                                            const float* __restrict__ trn, long long NT, long long tb,
                                            const float* __restrict__ strip)
{
    const int c = k * kChunk + lane;
    const bool cv = c < Ld;
    const int slot = k % kScoreRing;
    float (*tile)[kChunk] = st.sc[slot];
#pragma unroll 4
    for (int i = 0; i < 32; i++) {
        const bool v = cv && (r0 + i < Lq);
        const float* src = v ? S + (long long)(r0 + i) * ld + c : S;
        cp_async4(&tile[i][lane], src, v);
    }
    const long long e = tb + c;
#pragma unroll
    for (int f = 0; f < kNTrn; f++) {
        const long long ef = (f == trMI || f == trII) ? e + 1 : e;
        cp_async4(&st.tr[slot][f][lane], cv ? trn + f * NT + ef : trn, cv);
    }
    if (r0 > 0) {
#pragma unroll
        for (int f = 0; f < 5; f++) cp_async4(&st.sp[slot][f][lane], cv ? strip + f * ld + c : strip, cv);
    }
}

// write back the backtrack codes of chunk k of rows r0..r0+31
__device__ __forceinline__ void store_btck_chunk(const DpStage& st, uint8_t* __restrict__ B, long long ld,
                                                 int r0, int Lq, int Ld, int k, int lane)
{
    const int c = k * kChunk + lane;
    if (c >= Ld) return;
    const uint8_t (*tile)[kChunk] = st.bt[k % kBtckRing];
    const int nr = min(32, Lq - r0);
    for (int i = 0; i < nr; i++) B[(long long)(r0 + i) * ld + c] = tile[i][lane];
}

// kDpWarps warps (profiles) per block: 1 or 2, chosen by the tuner (each
// warp stages 18.5 KB of tiles, so a block of 4 would exceed the 48 KB of
// static shared memory)
template <int kDpWarps>
__global__ void __launch_bounds__(32 * kDpWarps)
dp1_kernel(const Dp1Args a)
{
    __shared__ DpStage s_stage[kDpWarps];
    const int lane = threadIdx.x & 31;
    const int pl = blockIdx.x * kDpWarps + (threadIdx.x >> 5);
    if (pl >= a.nprof) return;  // whole warp
    DpStage& st = s_stage[threadIdx.x >> 5];
    const int p = a.p0 + pl;
    const int Ld = a.db.plen[p];
    const long long colb = a.db.pstart[p] - a.col0;
    if (colb < 0 || colb + Ld > a.ld || Ld >= 65536) {
        // a profile outside the slab's columns (or too long for the 16-bit
        // cell coordinates) is skipped: nothing of it is read or written,
        // and its maximum is flagged as NaN with coordinates 0xffffffff
        if (lane == 0) {
            a.maxsc[pl] = __int_as_float(0x7fc00000);
            a.maxcoords[pl] = 0xffffffffu;
        }
        return;
    }
    const long long tb = a.db.pstart[p] + p;        // beginning-transition entry
    const long long NT = a.db.N + a.db.P;
    const int Lq = a.Lq;
    const int edge = corner_edge(Lq, Ld);
    const float* __restrict__ S = a.scores + colb;
    uint8_t* __restrict__ B = a.btck + colb;
    float* __restrict__ strip = a.bandbuf + colb;  // [5][ld] rows, this profile's columns
    const long long ld = a.ld;
    const int nchunks = (Ld + kChunk - 1) / kChunk;

    float best = 0.0f;
    int bestr = 0, bestc = 0;

    for (int r0 = 0; r0 < Lq; r0 += 32) {
        const int r = r0 + lane;
        const bool rv = r < Lq;
        const long long QT = Lq + 1;
        const float qMMp = rv ? a.qtrn[trMM * QT + r] : kLog0;
        const float qIMp = rv ? a.qtrn[trIM * QT + r] : kLog0;
        const float qDMp = rv ? a.qtrn[trDM * QT + r] : kLog0;
        const float qMDp = rv ? a.qtrn[trMD * QT + r] : kLog0;
        const float qDDp = rv ? a.qtrn[trDD * QT + r] : kLog0;
        const float qMIc = rv ? a.qtrn[trMI * QT + r + 1] : kLog0;
        const float qIIc = rv ? a.qtrn[trII * QT + r + 1] : kLog0;
        // column -1 of row r, as the reference's block schedule leaves it
        // (src/libmycu/cudp/CuBatchDP_init_btck.cu:93-160, 190-300): its
        // leftmost block diagonal of each 32-row band starts 32 columns left
        // of the profile and computes cells there with log-zero profile
        // transitions and score -9, so MM = 0, MI = IM = ND ~ -32768 and
        // DN(r) = max(qMD(r), DN(r-1) + qDD(r)), from max(qMD, qDD) on the
        // band's first row. The band's last row is started by the next
        // block diagonal at column 0 with zeroed predecessors.
        float dnv = hmax(0.0f + qMDp, 0.0f + qDDp);
        for (int k = 1; k < 31; k++) {
            const float up = __shfl_up_sync(kFull, dnv, 1);
            if (lane == k) dnv = hmax(0.0f + qMDp, up + qDDp);
        }
        const bool lastrow = (lane == 31);
        // this lane's latest cell (r, c-1): the "left" states
        float lMM = 0.f;
        float lMI = lastrow ? 0.f : kLog0, lIM = lastrow ? 0.f : kLog0;
        float lDN = lastrow ? 0.f : dnv, lND = lastrow ? 0.f : kLog0;
        // the previous step's "up" = this step's "diagonal"
        float dMM = 0.f, dMI = 0.f, dIM = 0.f, dDN = 0.f, dND = 0.f;
        const bool top = (r0 == 0);
        const int nsteps = Ld + 31;
        __syncwarp();   // the previous band's tiles are no longer read
        fetch_chunk(st, S, ld, r0, Lq, Ld, 0, lane, a.db.trn, NT, tb, strip);
        cp_async_commit();
        for (int s = 0; s < nsteps; s++) {
            if ((s & 31) == 0) {
                // chunk s/32 must be resident; fetch the next one
                if ((s >> 5) + 1 < nchunks)
                    fetch_chunk(st, S, ld, r0, Lq, Ld, (s >> 5) + 1, lane, a.db.trn, NT, tb, strip);
                cp_async_commit();
                cp_async_wait1();
                __syncwarp();
            } else if ((s & 31) == 31 && s >= 63) {
                // lane 31 passed chunk (s-63)/32 at the previous step
                __syncwarp();
                store_btck_chunk(st, B, ld, r0, Lq, Ld, (s - 63) >> 5, lane);
                __syncwarp();
            }
            const int c = s - lane;
            // states of (r-1, c): from lane-1's latest cell, or the strip
            float uMM = __shfl_up_sync(kFull, lMM, 1);
            float uMI = __shfl_up_sync(kFull, lMI, 1);
            float uIM = __shfl_up_sync(kFull, lIM, 1);
            float uDN = __shfl_up_sync(kFull, lDN, 1);
            float uND = __shfl_up_sync(kFull, lND, 1);
            if (lane == 0) {
                if (!top && c < Ld) {
                    const float (*sp)[kChunk] = st.sp[(c >> 5) % kScoreRing];
                    uMM = sp[0][c & 31]; uMI = sp[1][c & 31]; uIM = sp[2][c & 31];
                    uDN = sp[3][c & 31]; uND = sp[4][c & 31];
                } else {
                    uMM = uMI = uIM = uDN = uND = 0.f;
                }
            }
            if (lastrow && c == 0) {
                // the band's last row takes zeroed predecessors at column 0
                dMM = dMI = dIM = dDN = dND = 0.f;
            }
            if (rv && c >= 0 && c < Ld) {
                const float (*tr)[kChunk] = st.tr[(c >> 5) % kScoreRing];
                const int cc = c & 31;
                const float dMMp = tr[trMM][cc], dIMp = tr[trIM][cc];
                const float dDMp = tr[trDM][cc], dMDp = tr[trMD][cc];
                const float dDDp = tr[trDD][cc];
                const float dMIc = tr[trMI][cc], dIIc = tr[trII][cc];
                const float sc = in_corner(Lq, Ld, edge, r, c) ? -9.0f
                                 : st.sc[(c >> 5) % kScoreRing][lane][c & 31];
                float v1, v2, mx;
                int b = 0;
                v1 = dMI + qMMp + dIMp;
                v2 = dIM + qIMp + dMMp;
                v1 = hmax(v1, v2);
                v2 = dDN + qDMp + dMMp;
                v1 = hmax(v1, v2);
                v2 = dND + qMMp + dDMp;
                v1 = hmax(v1, v2);
                v2 = dMM + qMMp + dMMp;
                v1 = hmax(v1, v2);
                const float nMM = hmax(v1 + sc, 0.0f);
                mx = nMM;
                if (mx != 0.0f) b = 3;
                if (best < nMM) { best = nMM; bestr = r; bestc = c; }
                v1 = uMM + qMMp + dMIc;
                v2 = uMI + qMMp + dIIc;
                const float nMI = hmax(v1, v2);
                if (mx < nMI) { mx = nMI; b = 2; }
                v1 = lMM + qMIc + dMMp;
                v2 = lIM + qIIc + dMMp;
                const float nIM = hmax(v1, v2);
                if (mx < nIM) { mx = nIM; b = 1; }
                v1 = uMM + qMDp;
                v2 = uDN + qDDp;
                const float nDN = hmax(v1, v2);
                if (mx < nDN) { mx = nDN; b = 2; }
                v1 = lMM + dMDp;
                v2 = lND + dDDp;
                const float nND = hmax(v1, v2);
                if (mx < nND) { mx = nND; b = 1; }
                st.bt[(c >> 5) % kBtckRing][lane][c & 31] = (uint8_t)b;
                lMM = nMM; lMI = nMI; lIM = nIM; lDN = nDN; lND = nND;
                if (lane == 31) {
                    strip[0 * ld + c] = nMM; strip[1 * ld + c] = nMI; strip[2 * ld + c] = nIM;
                    strip[3 * ld + c] = nDN; strip[4 * ld + c] = nND;
                }
            }
            dMM = uMM; dMI = uMI; dIM = uIM; dDN = uDN; dND = uND;
            __syncwarp();
        }
        // the steps s = 32k+63 < Ld+31 wrote back chunks 0 .. (Ld-1)/32 - 1;
        // the last chunk is complete after the final step
        __syncwarp();
        store_btck_chunk(st, B, ld, r0, Lq, Ld, nchunks - 1, lane);
        __syncwarp();
    }
    // first cell in row-major order among equal maxima
    for (int off = 16; off >= 1; off >>= 1) {
        const float ob = __shfl_xor_sync(kFull, best, off);
        const int orr = __shfl_xor_sync(kFull, bestr, off);
        const int oc = __shfl_xor_sync(kFull, bestc, off);
        if (best < ob || (best == ob && (orr < bestr || (orr == bestr && oc < bestc)))) {
            best = ob; bestr = orr; bestc = oc;
        }
    }
    if (lane == 0) {
        a.maxsc[pl] = best;
        a.maxcoords[pl] = ((uint32_t)bestc << 16) | (uint32_t)bestr;
    }
}

// Finalization: one warp per profile (CuBatchDP_final.cu:61-292). Lane 0
// walks the backtrack bytes from the maximum; the diagonal steps' scores
// are collected in windows of 32 and the correlation terms
// s[k+4]*(s[k]+...+s[k+3]) are summed by the same xor butterfly as the
// reference, so the bonus is bit-identical to it.
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
dp1_finalize_kernel(const Dp1Args a, float thld)
{
    __shared__ float win[kWarpsPerBlock][40];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pl = blockIdx.x * kWarpsPerBlock + w;
    if (pl >= a.nprof) return;
    const int p = a.p0 + pl;
    const long long colb = a.db.pstart[p] - a.col0;
    const float* __restrict__ S = a.scores + colb;
    const uint8_t* __restrict__ B = a.btck + colb;
    float maxsc = a.maxsc[pl];
    const uint32_t xx = a.maxcoords[pl];
    Dp1Rec rec;
    rec.score = maxsc;
    rec.psts = 0.f;
    rec.beg = 0;
    rec.end = 0;
    rec.passed = 0;
    if (maxsc <= thld) {
        if (lane == 0) a.recs[pl] = rec;
        return;
    }
    float* wv = win[w];
    if (lane < 4) wv[32 + lane] = 0.f;
    __syncwarp();
    int x = (int)(xx >> 16), y = (int)(xx & 0xffff);
    int psts = 0, b = 3;
    float sumcorr = 0.f;
    const long long ld = a.ld;
    while (b != 0) {
        float carry = 0.f;
        if (lane < 4) carry = wv[32 + lane];
        __syncwarp();
        if (lane < 4) wv[lane] = carry;
        int ndx = 4;
        if (lane == 0) {
            while (ndx < 36) {
                if (x < 0 || y < 0) { b = 0; break; }
                b = B[(long long)y * ld + x];
                if (b == 0) break;
                if (b == 2) { y--; continue; }
                if (b == 1) { x--; continue; }
                const float v = S[(long long)y * ld + x];
                wv[ndx] = v;
                if (v > 0.0f) psts++;
                x--; y--; ndx++;
            }
        }
        __syncwarp();
        b = __shfl_sync(kFull, b, 0);
        ndx = __shfl_sync(kFull, ndx, 0);
        float corr = 0.f;
        if (!(ndx <= lane + 4))
            corr = wv[lane + 4] * (((wv[lane] + wv[lane + 1]) + wv[lane + 2]) + wv[lane + 3]);
        corr += __shfl_xor_sync(kFull, corr, 16);
        corr += __shfl_xor_sync(kFull, corr, 8);
        corr += __shfl_xor_sync(kFull, corr, 4);
        corr += __shfl_xor_sync(kFull, corr, 2);
        corr += __shfl_xor_sync(kFull, corr, 1);
        sumcorr += corr;
        __syncwarp();
    }
    if (lane == 0) {
        sumcorr = sumcorr * 0.5f;
        sumcorr = sumcorr < 0.0f ? -sqrtf(-sumcorr) : sqrtf(sumcorr);
        maxsc = maxsc + sumcorr;
        rec.score = maxsc;
        rec.psts = (float)psts;
        rec.beg = ((uint32_t)(x + 1) << 16) | (uint32_t)(y + 1);
        rec.end = xx;
        rec.passed = thld < maxsc ? 1 : 0;
        a.recs[pl] = rec;
    }
}

// Pass list in profile order: a single-block exclusive scan over the
// passed flags (and over the passed profiles' lengths for their offsets
// in the phase-2 position space). Replaces the reference's spin-locked
// atomicAdd list (CuBatchDP_final.cu:258-270), whose order varies run to run.
__global__ void __launch_bounds__(1024)
pass_compact_kernel(const Dp1Args a, int* __restrict__ pass_idx, long long* __restrict__ pass_dst,
                    int* __restrict__ npass_out, long long* __restrict__ npos_out)
{
    __shared__ int s_cnt[1024];
    __shared__ long long s_len[1024];
    __shared__ int base_cnt;
    __shared__ long long base_len;
    const int t = threadIdx.x;
    if (t == 0) { base_cnt = 0; base_len = 0; }
    __syncthreads();
    for (int start = 0; start < a.nprof; start += 1024) {
        const int pl = start + t;
        const int passed = (pl < a.nprof) ? a.recs[pl].passed : 0;
        const long long len = passed ? (long long)a.db.plen[a.p0 + pl] : 0;
        s_cnt[t] = passed;
        s_len[t] = len;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            int vc = (t >= off) ? s_cnt[t - off] : 0;
            long long vl = (t >= off) ? s_len[t - off] : 0;
            __syncthreads();
            s_cnt[t] += vc;
            s_len[t] += vl;
            __syncthreads();
        }
        if (passed) {
            const int k = base_cnt + s_cnt[t] - 1;
            pass_idx[k] = pl;
            pass_dst[k] = base_len + s_len[t] - len;
        }
        __syncthreads();
        if (t == 1023) { base_cnt += s_cnt[1023]; base_len += s_len[1023]; }
        __syncthreads();
    }
    if (t == 0) { *npass_out = base_cnt; *npos_out = base_len; }
}

}  // namespace

void launch_dp1(const Dp1Args& a, cudaStream_t stream)
{
    if (a.nprof <= 0) return;
    switch (a.warps) {
    case 1: dp1_kernel<1><<<(unsigned)a.nprof, 32, 0, stream>>>(a); break;
    case 2: dp1_kernel<2><<<(unsigned)ceil_div(a.nprof, 2), 64, 0, stream>>>(a); break;
    default: throw Error(CBP_ERR_ARG, "phase-1 DP warps per block must be 1 or 2");
    }
    CBP_CHECK_LAUNCH();
}

void launch_dp1_finalize(const Dp1Args& a, float thld, cudaStream_t stream)
{
    if (a.nprof <= 0) return;
    const int blocks = (int)ceil_div(a.nprof, kWarpsPerBlock);
    dp1_finalize_kernel<<<blocks, 32 * kWarpsPerBlock, 0, stream>>>(a, thld);
    CBP_CHECK_LAUNCH();
}

void launch_pass_compact(const Dp1Args& a, int* pass_idx, long long* pass_dst, int* npass,
                         long long* npos, cudaStream_t stream)
{
    pass_compact_kernel<<<1, 1024, 0, stream>>>(a, pass_idx, pass_dst, npass, npos);
    CBP_CHECK_LAUNCH();
}

}  // namespace cbp
