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
// of 64 query rows, two per lane, along anti-diagonals (lane t is at column
// s-t at step s). "Up" and "diagonal" states arrive from lane t-1 by
// shuffle; lane 0 reads the bottom row of the previous band from a
// per-profile global strip that lane 31 writes. One launch covers every
// profile of a slab (no per-diagonal launches, no grid-wide syncs).
#include <cstdint>
#include <type_traits>

#include "cother_b200.h"
#include "common.cuh"
#include "cbmath.cuh"
#include "dp1_kernel.cuh"
#include "bulkcopy.cuh"

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

// The band layout. One warp owns one profile and sweeps bands of 64 query
// rows, two per lane: lane t holds rows r0+2t (row "A") and r0+2t+1 (row
// "B") and is at column s-t at step s. Row A takes its "up" states from
// lane t-1's row B by shuffle, row B from the lane's own row A; so one
// shuffle set, one read of the column's transitions and one ring index
// serve two cells. The reference computes 32-row bands
// (src/libmycu/cudp/CuBatchDP_init_btck.cu:93-160); its band boundaries
// only set the column -1 states of each row and the diagonal of a band's
// last row at column 0, which are reproduced per row (row mod 32).
//
// Steps. While every lane is inside the profile (steps 32 .. Ld-1 of a
// band whose 64 rows all exist) a step runs without predicates: no column
// or row checks and no column-0 case. The first and last 32 steps of a
// band (the wavefront filling and draining) and a last band of fewer rows
// use the checked step; a partial band ends when its last valid lane
// leaves the profile.
//
// Staging. The band's columns are staged in pieces of 16 through a ring of
// 64 columns in shared memory: piece h+1 is fetched while the warp sweeps
// piece h (lanes span 32 columns, so three pieces are in use and one is in
// flight). Score rows arrive by 1-D bulk copies (cp.async.bulk with an
// mbarrier; each lane copies its own two rows, 64 bytes each), so staging
// costs two instructions per lane per 16 steps. A bulk copy needs 16-byte
// aligned addresses, so the ring is shifted by off = (first column of the
// profile) mod 4 and a piece starts at an aligned column. The profile
// transitions and the previous band's bottom row (the strip) come by
// 4-byte cp.async into [column][4] records, zero-filled outside the
// profile and on the first band, and are read back with 16-byte loads.
// A lane's two backtrack codes share one byte of a shared tile; the band's
// bottom row goes to a shared ring too. Both are written back once lane 31
// has left a piece: four code bytes per store, the strip coalesced.
//
// Occupancy. The kernel is bound by the latency of each warp's chain of
// dependent steps, so the SM's throughput grows with the warps resident.
// The launch that finds the maxima has no backtrack tile and needs about
// 100 registers instead of about 150, so more of its warps share an SM.
constexpr int kBand = 64;              // query rows per band (two per lane)
constexpr int kRing = 64;              // staged columns
constexpr int kPiece = 16;             // columns per staged piece
constexpr int kSlots = kRing / kPiece; // ring slots
constexpr unsigned long long kWaitNs = 1000000000ull;   // a staging wait gives up after 1 s

template <bool kCodes>
struct alignas(128) DpStage {
    float sc[kBand][kRing];            // scores of the band's rows
    float4 tra[kRing];                 // transitions of the column: MM, IM, DM, MD
    float4 trb[kRing];                 // DD, and MI, II of the next column
    float4 spa[kRing];                 // previous band's bottom row: MM, MI, IM, DN
    float spb[kRing];                  // ... and ND
    float4 soa[kRing];                 // this band's bottom row, for the next band
    float sob[kRing];
    uint8_t bt[kCodes ? 32 : 1][kRing]; // codes of rows A (low nibble) and B (high nibble)
    unsigned long long bar[kSlots];    // completion of each slot's score rows
};

__device__ __forceinline__ void cp_async4(void* dst, const float* src, bool valid)
{
    const int n = valid ? 4 : 0;   // 0: fill with zeros, read nothing
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"(smem_u32(dst)), "l"(src), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
// a staging wait gives up after kWaitNs
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity)
{
    return mbar_wait_for(b, parity, kWaitNs);
}

// One cell of the 5-state DP (ExecDP_Btck_Unroll32x, CuBatchDP_init_btck.cu:
// 303-360): from the diagonal (d), up (u) and left (l) states, the query
// transitions of the row (q: MM, IM, DM, MD, DD at the row, MI, II at the
// next row) and the profile's of the column (t), the new states and the
// backtrack code (0 stop, 1 left, 2 up, 3 diagonal). The additions run in
// the reference's order, (state + query) + profile. The states, scores and
// transitions are finite and never -0 (every state starts at +0 and a sum
// is -0 only when both terms are), so fmaxf gives the same value as the
// reference's compare-and-select maximum, in any order of its operands.
// The code is that of the first state, in the order MM, MI, IM, DN, ND,
// that attains the cell's maximum -- the outcome of the reference's chain
// of strict comparisons -- computed with independent comparisons.
struct Q7 { float MM, IM, DM, MD, DD, MIc, IIc; };
struct S5 { float MM, MI, IM, DN, ND; };

__device__ __forceinline__ int dp_cell(const S5& d, const S5& u, const S5& l, const Q7& q, const Q7& t,
                                       float sc, S5& n)
{
    const float m1 = fmaxf(d.MI + q.MM + t.IM, d.IM + q.IM + t.MM);
    const float m2 = fmaxf(d.DN + q.DM + t.MM, d.ND + q.MM + t.DM);
    const float m3 = fmaxf(m1, fmaxf(m2, d.MM + q.MM + t.MM));
    n.MM = fmaxf(m3 + sc, 0.0f);
    n.MI = fmaxf(u.MM + q.MM + t.MIc, u.MI + q.MM + t.IIc);
    n.IM = fmaxf(l.MM + q.MIc + t.MM, l.IM + q.IIc + t.MM);
    n.DN = fmaxf(u.MM + q.MD, u.DN + q.DD);
    n.ND = fmaxf(l.MM + t.MD, l.ND + t.DD);
    const float M = fmaxf(fmaxf(n.MM, n.MI), fmaxf(fmaxf(n.IM, n.DN), n.ND));
    const int bmm = (n.MM != 0.0f) ? 3 : 0;
    const int bud = (n.MI == M || (n.DN == M && n.IM != M)) ? 2 : 1;
    return (n.MM == M) ? bmm : bud;
}

// The states of one cell alone (a sweep without backtrack codes).
__device__ __forceinline__ void dp_states(const S5& d, const S5& u, const S5& l, const Q7& q, const Q7& t,
                                          float sc, S5& n)
{
    const float m1 = fmaxf(d.MI + q.MM + t.IM, d.IM + q.IM + t.MM);
    const float m2 = fmaxf(d.DN + q.DM + t.MM, d.ND + q.MM + t.DM);
    const float m3 = fmaxf(m1, fmaxf(m2, d.MM + q.MM + t.MM));
    n.MM = fmaxf(m3 + sc, 0.0f);
    n.MI = fmaxf(u.MM + q.MM + t.MIc, u.MI + q.MM + t.IIc);
    n.IM = fmaxf(l.MM + q.MIc + t.MM, l.IM + q.IIc + t.MM);
    n.DN = fmaxf(u.MM + q.MD, u.DN + q.DD);
    n.ND = fmaxf(l.MM + t.MD, l.ND + t.DD);
}

__device__ __forceinline__ Q7 query_trn(const float* __restrict__ qtrn, long long QT, int r, int Lq)
{
    Q7 q;
    const bool v = r < Lq;
    q.MM = v ? qtrn[trMM * QT + r] : kLog0;
    q.IM = v ? qtrn[trIM * QT + r] : kLog0;
    q.DM = v ? qtrn[trDM * QT + r] : kLog0;
    q.MD = v ? qtrn[trMD * QT + r] : kLog0;
    q.DD = v ? qtrn[trDD * QT + r] : kLog0;
    q.MIc = v ? qtrn[trMI * QT + r + 1] : kLog0;
    q.IIc = v ? qtrn[trII * QT + r + 1] : kLog0;
    return q;
}

// kWarps warps (profiles) per block, each with its own DpStage in dynamic
// shared memory. kBulk: score rows by bulk copies (the slab width is a
// multiple of 4 floats and the buffers are aligned); otherwise by 4-byte
// cp.async with the ring unshifted.
template <int kWarps, bool kBulk, bool kCodes>
__global__ void __launch_bounds__(32 * kWarps)
dp1_kernel(const Dp1Args a)
{
    extern __shared__ __align__(128) unsigned char s_dyn[];
    const int lane = threadIdx.x & 31;
    const int pl = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (pl >= a.nprof) return;  // whole warp
    DpStage<kCodes>& st = reinterpret_cast<DpStage<kCodes>*>(s_dyn)[threadIdx.x >> 5];
    const int p = a.p0 + pl;
    const int Ld = a.db.plen[p];
    const long long colb = a.db.pstart[p] - a.col0;
    if (colb < 0 || colb + Ld > a.ld || Ld >= 65536 || Ld <= 0) {
        // a profile outside the slab's columns (or too long for the 16-bit
        // cell coordinates) is skipped: nothing of it is read or written,
        // and its maximum is flagged as NaN with coordinates 0xffffffff
        if (lane == 0) {
            a.maxsc[pl] = Ld == 0 ? 0.0f : __int_as_float(0x7fc00000);
            a.maxcoords[pl] = Ld == 0 ? 0u : 0xffffffffu;
        }
        return;
    }
    const int Lq = a.Lq;
    const long long ld = a.ld;
    const long long QT = Lq + 1;
    const long long tb = a.db.pstart[p] + p;        // beginning-transition entry
    const long long NT = a.db.N + a.db.P;
    const float* __restrict__ trn = a.db.trn;
    const float* __restrict__ S = a.scores + colb;
    uint8_t* __restrict__ B = a.btck + colb;
    float* __restrict__ strip = a.bandbuf + colb;  // [5][ld] rows, this profile's columns
    const int edge = corner_edge(Lq, Ld);
    const int off = kBulk ? (int)(colb & 3) : 0;    // ring shift: pieces start at aligned columns
    const int h_last = (Ld - 1 + off) >> 4;         // last piece holding a column of the profile

    if (kBulk) {
        if (lane == 0) {
            for (int j = 0; j < kSlots; j++) mbar_init(&st.bar[j]);
            mbar_init_fence();
        }
        __syncwarp();
    }
    unsigned phases = 0;   // per slot: parity of its next completion
    bool ok = true;

    float best = 0.0f;
    int bestr = 0, bestc = 0;

    using kTrue = std::integral_constant<bool, true>;
    using kFalse = std::integral_constant<bool, false>;
    // One sweep over the profile's DP. kCodes: with the backtrack codes and
    // the coordinates of the maximum; without them, the maximum alone.
    auto sweep = [&](auto codes_tag) {
        constexpr bool kSweepCodes = decltype(codes_tag)::value;
        best = 0.0f;
        bestr = 0;
        bestc = 0;
        for (int r0 = 0; r0 < Lq && ok; r0 += kBand) {
            const int rA = r0 + 2 * lane, rB = rA + 1;
            const bool vA = rA < Lq, vB = rB < Lq;
            const Q7 qa = query_trn(a.qtrn, QT, rA, Lq);
            const Q7 qb = query_trn(a.qtrn, QT, rB, Lq);
            const bool top = (r0 == 0);
            const bool has_next = r0 + kBand < Lq;
            const bool full = r0 + kBand <= Lq;           // all 64 rows exist
            const int nlanes = min(32, (Lq - r0 + 1) >> 1);   // lanes holding a row
            const int nsteps = Ld + nlanes - 1;
            const bool lastB = (rB & 31) == 31;  // the last row of a 32-row band of the reference
            // column -1 of each row, as the reference's block schedule leaves
            // it (CuBatchDP_init_btck.cu:93-160, 190-300): MM = 0, MI = IM = ND
            // ~ -32768 and DN(r) = max(qMD(r), DN(r-1) + qDD(r)), from
            // max(qMD, qDD) on a 32-row band's first row; a 32-row band's last
            // row starts at column 0 from zeroed predecessors
            float dnA = 0.0f, dnB = 0.0f;
            for (int k = 0; k < 16; k++) {
                const float up = __shfl_up_sync(kFull, dnB, 1);
                if ((lane & 15) == k) {
                    dnA = (k == 0) ? hmax(0.0f + qa.MD, 0.0f + qa.DD) : hmax(0.0f + qa.MD, up + qa.DD);
                    dnB = hmax(0.0f + qb.MD, dnA + qb.DD);
                }
            }
            S5 lA = {0.0f, kLog0, kLog0, dnA, kLog0};
            S5 lB = lastB ? S5{0.0f, 0.0f, 0.0f, 0.0f, 0.0f} : S5{0.0f, kLog0, kLog0, dnB, kLog0};
            S5 dg = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};       // row A's diagonal: the previous step's up
            // corner triangles (ExecDP_Btck_Unroll32x excludes them): a cell is
            // in a corner when c <= ca or c >= cb for its row
            const bool bcorner = (r0 < edge) || (r0 + kBand - 1 + edge >= Lq);
            const int caA = (Lq <= rA + edge) ? edge + rA - Lq : -1;
            const int cbA = (rA < edge) ? Ld - edge + rA : 0x7fffffff;
            const int caB = (Lq <= rB + edge) ? edge + rB - Lq : -1;
            const int cbB = (rB < edge) ? Ld - edge + rB : 0x7fffffff;
            float bstA = 0.0f, bstB = 0.0f;
            int bcA = 0, bcB = 0;

            // fetch piece h of this band into ring slot h mod 4
            auto issue = [&](int h) {
                const int slot = h & (kSlots - 1);
                const int c0 = kPiece * h - off;            // first column of the piece
                if (kBulk) {
                    const int ncol = min(kPiece, Ld - c0);   // >= 1: h <= h_last
                    const unsigned bytes = (unsigned)((ncol * 4 + 15) & ~15);
                    const int nrows = min(kBand, Lq - r0);
                    if (lane == 0) mbar_expect_tx(&st.bar[slot], bytes * (unsigned)nrows);
                    __syncwarp();
                    // the slot's earlier contents were read through the generic
                    // proxy; order those reads before the bulk copy's writes
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    if (vA) bulk_load(&st.sc[2 * lane][kPiece * slot], S + (long long)rA * ld + c0, bytes, &st.bar[slot]);
                    if (vB) bulk_load(&st.sc[2 * lane + 1][kPiece * slot], S + (long long)rB * ld + c0, bytes,
                                      &st.bar[slot]);
                } else {
#pragma unroll 4
                    for (int j = 0; j < kPiece; j++) {
                        const int c = c0 + j;
                        const bool cv = c < Ld;
                        cp_async4(&st.sc[2 * lane][kPiece * slot + j], (vA && cv) ? S + (long long)rA * ld + c : S,
                                  vA && cv);
                        cp_async4(&st.sc[2 * lane + 1][kPiece * slot + j], (vB && cv) ? S + (long long)rB * ld + c : S,
                                  vB && cv);
                    }
                }
                const int j = lane & 15;
                const int c = c0 + j;
                const bool cv = c >= 0 && c < Ld;
                const bool sv = cv && !top;                 // the strip: zeros on the first band
                const int pos = kPiece * slot + j;
                if (lane < 16) {
                    float* d = reinterpret_cast<float*>(&st.tra[pos]);
                    cp_async4(d + 0, cv ? trn + trMM * NT + tb + c : trn, cv);
                    cp_async4(d + 1, cv ? trn + trIM * NT + tb + c : trn, cv);
                    cp_async4(d + 2, cv ? trn + trDM * NT + tb + c : trn, cv);
                    cp_async4(d + 3, cv ? trn + trMD * NT + tb + c : trn, cv);
                    float* e = reinterpret_cast<float*>(&st.spa[pos]);
                    cp_async4(e + 0, sv ? strip + 0 * ld + c : trn, sv);
                    cp_async4(e + 1, sv ? strip + 1 * ld + c : trn, sv);
                } else {
                    float* d = reinterpret_cast<float*>(&st.trb[pos]);
                    cp_async4(d + 0, cv ? trn + trDD * NT + tb + c : trn, cv);
                    cp_async4(d + 1, cv ? trn + trMI * NT + tb + c + 1 : trn, cv);
                    cp_async4(d + 2, cv ? trn + trII * NT + tb + c + 1 : trn, cv);
                    float* e = reinterpret_cast<float*>(&st.spa[pos]);
                    cp_async4(e + 2, sv ? strip + 2 * ld + c : trn, sv);
                    cp_async4(e + 3, sv ? strip + 3 * ld + c : trn, sv);
                    cp_async4(&st.spb[pos], sv ? strip + 4 * ld + c : trn, sv);
                }
                cp_async_commit();
            };
            // wait until piece h is resident (piece h+1 in flight when `more`);
            // false if its score rows never arrived, after a bounded wait for
            // the copies still in flight into this warp's shared memory
            auto await = [&](int h, bool more) {
                cp_async_wait1();
                if (!kBulk) {
                    __syncwarp();
                    return true;
                }
                const int slot = h & (kSlots - 1);
                const unsigned par = (phases >> slot) & 1u;
                const bool got = __all_sync(kFull, mbar_wait(&st.bar[slot], par));
                if (got) {
                    phases ^= 1u << slot;
                    __syncwarp();
                    return true;
                }
                cp_async_wait0();
                (void)mbar_wait(&st.bar[slot], par);
                if (more) {
                    const int s1 = (h + 1) & (kSlots - 1);
                    (void)mbar_wait(&st.bar[s1], (phases >> s1) & 1u);
                }
                return false;
            };
            // write back piece h (lane 31 has left it): the backtrack codes of
            // its columns inside the profile, and the band's bottom row
            auto flush = [&](int h) {
                const int slot = h & (kSlots - 1);
                const int c0 = kPiece * h - off;
                const uint4 pk = *reinterpret_cast<const uint4*>(&st.bt[lane][kPiece * slot]);
                const uint32_t pw[4] = {pk.x, pk.y, pk.z, pk.w};
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    if (!kSweepCodes || r0 + 2 * lane + k >= Lq) continue;
                    uint8_t* dst = B + (long long)(r0 + 2 * lane + k) * ld + c0;
#pragma unroll
                    for (int wd = 0; wd < 4; wd++) {
                        const uint32_t v = (pw[wd] >> (4 * k)) & 0x0f0f0f0fu;
                        const int cw = c0 + 4 * wd;
                        if (kBulk && cw >= 0 && cw + 4 <= Ld) {
                            *reinterpret_cast<uint32_t*>(dst + 4 * wd) = v;
                        } else {
                            for (int i = 0; i < 4; i++) {
                                const int cc = cw + i;
                                if (cc >= 0 && cc < Ld) dst[4 * wd + i] = (uint8_t)(v >> (8 * i));
                            }
                        }
                    }
                }
                if (has_next && lane < kPiece) {
                    const int c = c0 + lane;
                    if (c >= 0 && c < Ld) {
                        const float4 v = st.soa[kPiece * slot + lane];
                        strip[0 * ld + c] = v.x; strip[1 * ld + c] = v.y; strip[2 * ld + c] = v.z;
                        strip[3 * ld + c] = v.w; strip[4 * ld + c] = st.sob[kPiece * slot + lane];
                    }
                }
            };

            // one step: cells (rA, c) and (rB, c) of the lane, c = s - lane.
            // kChecked: some lane may be outside the profile or below the last
            // row, or at column 0; kCorner: the band reaches a corner triangle
            auto step = [&](int s, auto checked_tag, auto corner_tag) {
                constexpr bool kChecked = decltype(checked_tag)::value;
                constexpr bool kCorner = decltype(corner_tag)::value;
                const int c = s - lane;
                S5 u;
                u.MM = __shfl_up_sync(kFull, lB.MM, 1);
                u.MI = __shfl_up_sync(kFull, lB.MI, 1);
                u.IM = __shfl_up_sync(kFull, lB.IM, 1);
                u.DN = __shfl_up_sync(kFull, lB.DN, 1);
                u.ND = __shfl_up_sync(kFull, lB.ND, 1);
                const int pos = (c + off) & (kRing - 1);
                {
                    // lane 0: the previous band's bottom row (zeros on the first
                    // band and outside the profile)
                    const float4 v = st.spa[pos];
                    const float w = st.spb[pos];
                    if (lane == 0) { u.MM = v.x; u.MI = v.y; u.IM = v.z; u.DN = v.w; u.ND = w; }
                }
                bool doA = true, doB = true;
                if (kChecked) {
                    doA = vA && c >= 0 && c < Ld;
                    doB = doA && vB;
                }
                if (doA) {
                    const float4 ta = st.tra[pos];
                    const float4 tc = st.trb[pos];
                    Q7 t;
                    t.MM = ta.x; t.IM = ta.y; t.DM = ta.z; t.MD = ta.w;
                    t.DD = tc.x; t.MIc = tc.y; t.IIc = tc.z;
                    float scA = st.sc[2 * lane][pos];
                    if (kCorner && (c <= caA || c >= cbA)) scA = -9.0f;
                    S5 nA;
                    int code = 0;
                    if (kSweepCodes) {
                        code = dp_cell(dg, u, lA, qa, t, scA, nA);
                        if (bstA < nA.MM) { bstA = nA.MM; bcA = c; }
                    } else {
                        dp_states(dg, u, lA, qa, t, scA, nA);
                        bstA = fmaxf(bstA, nA.MM);
                    }
                    if (doB) {
                        float scB = st.sc[2 * lane + 1][pos];
                        if (kCorner && (c <= caB || c >= cbB)) scB = -9.0f;
                        // diagonal of (rB, c) = (rA, c-1): row A's left state; a
                        // 32-row band's last row takes zeros at column 0
                        S5 dB = lA;
                        if (kChecked && lastB && c == 0) dB = S5{0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
                        S5 nB;
                        if (kSweepCodes) {
                            code |= dp_cell(dB, nA, lB, qb, t, scB, nB) << 4;
                            if (bstB < nB.MM) { bstB = nB.MM; bcB = c; }
                        } else {
                            dp_states(dB, nA, lB, qb, t, scB, nB);
                            bstB = fmaxf(bstB, nB.MM);
                        }
                        lB = nB;
                        if (lane == 31) {
                            st.soa[pos] = make_float4(nB.MM, nB.MI, nB.IM, nB.DN);
                            st.sob[pos] = nB.ND;
                        }
                    }
                    if (kSweepCodes) st.bt[lane][pos] = (uint8_t)code;
                    lA = nA;
                }
                dg = u;
            };

            __syncwarp();   // the previous band's tiles are no longer read
            issue(0);
            int hflushed = 0;   // pieces 0 .. hflushed-1 are written back
            // steps with every lane inside the profile and on a row (the
            // unchecked steps): [32, Ld) on a full band
            const int fast0 = full ? 32 : nsteps, fast1 = full ? Ld : nsteps;
            for (int H = 0;; H++) {
                const int sb = (H == 0) ? 0 : kPiece * H - off;   // lane 0 enters piece H
                if (sb >= nsteps) break;
                const int se = min(kPiece * H + kPiece - off, nsteps);
                __syncwarp();
                // lane 31 left piece H-3 two steps ago; its ring slot takes piece H+1
                if (H >= 3 && H - 3 <= h_last) { flush(H - 3); hflushed = H - 2; }
                if (H <= h_last) {
                    const bool more = H + 1 <= h_last;
                    if (more) issue(H + 1);
                    else cp_async_commit();   // an empty group keeps the wait accounting
                    if (!await(H, more)) { ok = false; break; }
                }
                const int f0 = max(sb, fast0), f1 = min(se, fast1);
                if (f0 < f1) {
                    for (int s = sb; s < f0; s++) step(s, kTrue(), kTrue());
                    if (bcorner) {
#pragma unroll 2
                        for (int s = f0; s < f1; s++) step(s, kFalse(), kTrue());
                    } else {
#pragma unroll 2
                        for (int s = f0; s < f1; s++) step(s, kFalse(), kFalse());
                    }
                    for (int s = f1; s < se; s++) step(s, kTrue(), kTrue());
                } else {
                    for (int s = sb; s < se; s++) step(s, kTrue(), kTrue());
                }
            }
            if (!ok) break;
            __syncwarp();
            for (int h = hflushed; h <= h_last; h++) flush(h);
            // the band's maxima into the lane's, in row-major order
            if (kSweepCodes) {
                if (best < bstA) { best = bstA; bestr = rA; bestc = bcA; }
                if (best < bstB) { best = bstB; bestr = rB; bestc = bcB; }
            } else {
                best = fmaxf(best, fmaxf(bstA, bstB));
            }
        }
    };

    // The codes are read only by the backtrace of a profile whose maximum
    // exceeds the threshold (the finalization skips the others). So a first
    // launch without them (kCodes false, a smaller stage) finds every
    // profile's maximum, and a second launch sweeps the candidates again
    // with them; code_thld = -inf: the second launch alone, for all.
    if (!kCodes) {
        sweep(kFalse());
        for (int o = 16; o >= 1; o >>= 1) best = fmaxf(best, __shfl_xor_sync(kFull, best, o));
        if (lane == 0) {
            // a staging wait that gave up flags the profile and the launch
            a.maxsc[pl] = ok ? best : __int_as_float(0x7fc00000);
            a.maxcoords[pl] = ok ? 0u : 0xffffffffu;
            if (!ok && a.err) atomicExch(a.err, 1);
        }
        return;
    }
    if (a.code_thld != -INFINITY && !(a.maxsc[pl] > a.code_thld)) return;   // not a candidate
    sweep(kTrue());
    if (!ok) {
        if (lane == 0) {
            a.maxsc[pl] = __int_as_float(0x7fc00000);
            a.maxcoords[pl] = 0xffffffffu;
            if (a.err) atomicExch(a.err, 1);
        }
        return;
    }
    // first cell in row-major order among equal maxima
    for (int o = 16; o >= 1; o >>= 1) {
        const float ob = __shfl_xor_sync(kFull, best, o);
        const int orr = __shfl_xor_sync(kFull, bestr, o);
        const int oc = __shfl_xor_sync(kFull, bestc, o);
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
    if (!(maxsc > thld)) {   // a NaN maximum (a flagged profile) never passes
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

template <int kW, bool kBulk, bool kCodes>
void launch_dp1_variant(const Dp1Args& a, cudaStream_t stream)
{
    const size_t smem = (size_t)kW * sizeof(DpStage<kCodes>);
    dp1_kernel<kW, kBulk, kCodes><<<(unsigned)ceil_div(a.nprof, kW), 32 * kW, smem, stream>>>(a);
    CBP_CHECK_LAUNCH();
}

void dp1_set_attributes()
{
    // dynamic shared memory above 48 KB (two warps per block) needs an opt-in
    CBP_CUDA(cudaFuncSetAttribute(dp1_kernel<2, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * sizeof(DpStage<true>))));
    CBP_CUDA(cudaFuncSetAttribute(dp1_kernel<2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * sizeof(DpStage<true>))));
    CBP_CUDA(cudaFuncSetAttribute(dp1_kernel<2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * sizeof(DpStage<false>))));
    CBP_CUDA(cudaFuncSetAttribute(dp1_kernel<2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * sizeof(DpStage<false>))));
}

template <bool kCodes>
void launch_dp1_pass(const Dp1Args& a, bool bulk, cudaStream_t stream)
{
    switch (a.warps) {
    case 1: bulk ? launch_dp1_variant<1, true, kCodes>(a, stream) : launch_dp1_variant<1, false, kCodes>(a, stream); break;
    case 2: bulk ? launch_dp1_variant<2, true, kCodes>(a, stream) : launch_dp1_variant<2, false, kCodes>(a, stream); break;
    default: throw Error(CBP_ERR_ARG, "phase-1 DP warps per block must be 1 or 2");
    }
}

int launch_dp1(const Dp1Args& a, cudaStream_t stream)
{
    if (a.nprof <= 0) return 0;
    // bulk copies of score rows need 16-byte aligned rows and 4-byte
    // aligned backtrack words
    const bool bulk = (a.ld % 4 == 0) && ((uintptr_t)a.scores % 16 == 0) && ((uintptr_t)a.btck % 4 == 0);
    const bool split = a.code_thld != -INFINITY;
    if (split) launch_dp1_pass<false>(a, bulk, stream);
    launch_dp1_pass<true>(a, bulk, stream);
    return split ? 2 : 1;
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
