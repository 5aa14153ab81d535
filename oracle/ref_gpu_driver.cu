// Test infrastructure: a host driver that runs the REFERENCE's own CUDA
// kernels (compiled from their sources where they lie in the reference tree
// by `make -C oracle refgpu`) on one query against one database chunk, and
// returns every intermediate result, so that golden fixtures pinning the
// CPU oracle can be generated on a GPU box. Nothing in the product links
// this; it is built into oracle/_ref/ only.
//
// The launch sequence, grid shapes and device-heap arrangement restate the
// reference's host code, not its kernels:
//   score matrix   src/libmycu/cusco/CuBatchScoreMatrix.cu:122-404
//                  (init, then SS and/or CVS, then DDMS; HDP off)
//   phase-1 DP     src/libmycu/cudp/CuBatchDP.cu:149-320 (host loop over
//                  block diagonals) and FinalizeDP, :330-380
//   statistics     src/libmycu/cuss/CuBatchSS.cu:60-160 (dynamic-parallel
//                  CalcStatisticsDynPlm, one parent thread per passed pair)
//   MAPALN=0       FinalizeDP_ALN on the phase-1 backtrack codes
//                  (src/libmycu/cudp/CuBatchDP.cu:427-530) instead of MAP
//   MAP            src/libmycu/cumapdp/CuBatchMAPDP.cu:130-330 (the host
//                  loop of its #else branch: the same kernels, in the same
//                  order, on one stream, as its parent kernel launches them)
//                  and FinalizeMAPDP_MAP, :380-470
//   sequencing     src/libmycu/cupro/CuBatchProcessing.cu:230-560
//   heap sections  src/libmycu/cupro/CuDeviceMemory.cu:548-588 with sizes
//                  from CuDeviceMemory.cuh:406-700, sized here for exactly
//                  one chunk in which every profile may pass
//   constants      dc_pm2dvfields_ (3 x 181 field addresses: query, cached
//                  DB, chunk DB) and dc_cuss_NN_weights_ (93 floats) are
//                  defined here as the reference defines them in
//                  CuDeviceMemory.cu:600-602
//   SS table       serialized as SerializedScoresCtor does
//                  (src/libmycu/cupro/SerializedScoresCtor.cuh:83-139): one
//                  probability level, one ENO level, then the packed lower
//                  triangle of the 30 x 30 table
//   DMS table      SerializedDstMatchScoresCtor<float,2> has no entries
//                  (SerializedDstMatchScores.cuh:632-645): cardinality 21.
//   CVS map        serialized as SerializedCVS2ScoresCtor does
//                  (src/libmycu/cupro/SerializedCVS2ScoresCtor.cuh:60-120) for
//                  one level: level, cardinality, shift, scale, keys,
//                  scores; attributes as CuDeviceMemory::CacheCVS2ScoresDevice
//                  (CuDeviceMemory.cu:691-740), constants as _TCTXVECT
//                  (src/libpro/srcpro/TCTXVECT.cpp:26-60).
//
// The database is passed as the chunk section (bdbC); the cached section is
// empty. Profiles should come longest first, as in a reference database:
// the phase-1 grid is sized by the first profile's length.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "liblib/mybase.h"
#include "libmycu/cucom/cucommon.h"
#include "libmycu/cupro/PM2DVectorFields.h"
#include "libmycu/cupro/CuBatchProcessing_com.cuh"
#include "libmycu/cupro/SerializedScoresAttr.h"
#include "libmycu/cupro/SerializedDstMatchScoresAttr.h"
#include "libmycu/cusco/CuBatchScoreMatrix_com.h"
#include "libmycu/cusco/CuBatchScoreMatrix_Init.cuh"
#include "libmycu/cusco/CuBatchScoreMatrix_ssss.cuh"
#include "libmycu/cusco/CuBatchScoreMatrix_ddms2s_h2.cuh"
#include "libmycu/cupro/SerializedCVS2ScoresAttr.h"
#include "libmycu/cusco/CuBatchScoreMatrix_cvs2s.cuh"
#include "libmycu/cusco/CuBatchScoreMatrix_ssss_cvs2s.cuh"
#include "libmycu/cudp/CuBatchDP_com.h"
#include "libmycu/cudp/CuBatchDP_init_btck.cuh"
#include "libmycu/cudp/CuBatchDP_final.cuh"
#include "libmycu/cudp/CuBatchDP_aln_final.cuh"
#include "libmycu/cuss/CuBatchSS_com.h"
#include "libmycu/cuss/CuBatchSS_dynplm.cuh"
#include "libmycu/cumapdp/CuBatchMAPDP_com.h"
#include "libmycu/cumapdp/CuBatchMAPDP_fwd.cuh"
#include "libmycu/cumapdp/CuBatchMAPDP_bwd.cuh"
#include "libmycu/cumapdp/CuBatchMAPDP_map_btck.cuh"
#include "libmycu/cumapdp/CuBatchMAPDP_map_final.cuh"

__constant__ char* dc_pm2dvfields_[fsg_sztotflds3];
__constant__ float dc_cuss_NN_weights_[sz_total_dc_cuss_NNwghts];

namespace {

constexpr int kFields = pmv2DTotFlds;
constexpr size_t kAlign = 256;
constexpr int kDmsCard = 21;     // DMS_MaxDst + 1
constexpr int kSsCard = 30;

size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

std::string g_err;

struct Fail {
    std::string msg;
};

void ck(cudaError_t rc, const char* what)
{
    if (rc != cudaSuccess)
        throw Fail{std::string(what) + ": " + cudaGetErrorString(rc)};
}

void ck_launch(const char* what)
{
    ck(cudaGetLastError(), what);
}

// upper bound on the number of blocks in one oblique block diagonal
// (src/libmycu/cudp/CuBatchDP.cuh:190-197)
unsigned blocks_per_diagonal(size_t dblen, size_t qlen, size_t w, size_t b)
{
    size_t along_q = (qlen + w - 1) / w;
    size_t bpw = w + b;
    size_t along_d = (dblen + bpw + bpw - 1) / bpw;
    return (unsigned)(along_q < along_d ? along_q : along_d);
}

struct Events {
    cudaEvent_t e[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    Events()
    {
        for (auto& x : e) ck(cudaEventCreate(&x), "event");
    }
    ~Events()
    {
        for (auto& x : e) if (x) cudaEventDestroy(x);
    }
};

struct DevBuf {
    char* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    char* alloc(size_t n, const char* what)
    {
        ck(cudaMalloc(&p, n), what);
        ck(cudaMemset(p, 0, n), what);
        return p;
    }
};

}  // namespace

extern "C" {

// Fixed sizes of the reference's interface records, for the caller.
void refgpu_consts(int* out)
{
    out[0] = nTDP2OutputPhase1;
    out[1] = nTDP2OutputAlnData;
    out[2] = nTDP2OutputAlignmentSSS;
    out[3] = pmv2DTotFlds;
    out[4] = CUL2CLINESIZE;
}

const char* refgpu_error() { return g_err.c_str(); }

typedef struct refgpu_job {
    // inputs: host field arrays (begin pointer and byte size per field)
    const char* q[kFields];
    size_t qsz[kFields];
    const char* d[kFields];
    size_t dsz[kFields];
    int nqyposs, ndbpros, ndbposs, dbpro1len;
    float qyeno;
    const float* sstab;        // 30 x 30
    const float* nnweights;    // sz_total_dc_cuss_NNwghts
    float ssswgt, ddmswgt, minpp, scorethld, logevthld, searchspace;
    float reflambda, refK, explambda, expK;
    int dstsegm, ssemodel, xuninf;
    // outputs (caller-allocated host memory)
    float* scores;             // [nqyposs][dblen]
    float* modscores;          // [nqyposs][dblen]
    unsigned char* btck;       // [nqyposs][dblen] phase-1 backtrack
    float* phase1;             // [ndbpros][nTDP2OutputPhase1] after FinalizeDP
    float* stats;              // [ndbpros][nTDP2OutputAlnData] after statistics
    float* final_recs;         // [ndbpros][nTDP2OutputAlnData] after MAP
    char* alns;                // [nTDP2OutputAlignmentSSS][alns_cap]
    size_t alns_cap;
    unsigned int globvars[4];  // passed profiles, their positions, max length
    int dblen;
    size_t dbalnlen2;
    // timing: with copy_matrices = 0 the score matrices and backtrack codes
    // stay on the device (their pointers may be null); stage_ms receives the
    // device time of the score matrix, phase 1 (DP + finalization),
    // statistics and MAP, measured with events around each stage's launches
    int copy_matrices;
    float stage_ms[4];
    // context-vector term: CVSWGT and the map (keys on the grid of halves,
    // smoothed scores); the profiles' CV fields are in q/d
    float cvswgt;
    const float* cvskeys;
    const float* cvsscores;
    int cvscard;
    // MAPALN=0: the phase-1 alignments (FinalizeDP_ALN) instead of MAP
    int nomapaln;
} refgpu_job;

int refgpu_run(refgpu_job* J)
{
    g_err.clear();
    try {
        const size_t Lq = (size_t)J->nqyposs;
        const size_t N = (size_t)J->ndbposs;
        const size_t P = (size_t)J->ndbpros;
        const size_t dblen = up(N, CUL2CLINESIZE);
        const size_t dbxpad = dblen - N;
        J->dblen = (int)dblen;
        if (Lq < 1 || N < 1 || P < 1)
            throw Fail{"empty query or database"};
        // the reference's kernels index a chunk's cells with 32-bit ints
        // ((y-i)*dblen + i, CuBatchDP_init_btck.cu:488); its memory planner
        // keeps chunks below INT_MAX/Lq positions
        // (CuDeviceMemory.cuh:658-690), and so must the caller
        if ((double)Lq * (double)(dblen + 64) >= 2147483647.0)
            throw Fail{"chunk too large for the reference's 32-bit cell indices: "
                       "split the database"};
        // the statistics kernels' stack size is not known statically: give
        // every thread a generous stack; the dynamic launches per passed pair
        // (a parent and six children) stay well under the pending-launch limit
        ck(cudaDeviceSetLimit(cudaLimitStackSize, 16384), "stack limit");
        ck(cudaDeviceSetLimit(cudaLimitDevRuntimePendingLaunchCount, 8192), "launch limit");

        // profile data: every field at a 256-byte boundary with slack after it
        auto pack = [](const char* const* src, const size_t* sz, DevBuf& buf,
                       std::vector<char*>& addr) {
            size_t total = 0;
            std::vector<size_t> off(kFields);
            for (int f = 0; f < kFields; f++) {
                off[f] = total;
                total += up(sz[f] + 4096, kAlign);
            }
            char* base = buf.alloc(total, "profile data");
            addr.resize(kFields);
            for (int f = 0; f < kFields; f++) {
                addr[f] = base + off[f];
                if (sz[f])
                    ck(cudaMemcpy(addr[f], src[f], sz[f], cudaMemcpyHostToDevice), "field copy");
            }
        };
        DevBuf qbuf, dbuf;
        std::vector<char*> qa, da;
        pack(J->q, J->qsz, qbuf, qa);
        pack(J->d, J->dsz, dbuf, da);
        std::vector<char*> table(fsg_sztotflds3);
        for (int f = 0; f < kFields; f++) {
            table[f] = qa[f];
            table[kFields + f] = da[f];      // cached section: unused (no profiles)
            table[2 * kFields + f] = da[f];
        }
        ck(cudaMemcpyToSymbol(dc_pm2dvfields_, table.data(), table.size() * sizeof(char*)),
           "field table");
        ck(cudaMemcpyToSymbol(dc_cuss_NN_weights_, J->nnweights,
                              sz_total_dc_cuss_NNwghts * sizeof(float)), "NN weights");

        // serialized SS table: [prob level][ENO level][lower triangle]
        std::vector<float> ssser;
        ssser.push_back(0.0f);
        ssser.push_back(1.0f);
        for (int r = 0; r < kSsCard; r++)
            for (int c = 0; c <= r; c++)
                ssser.push_back(J->sstab[r * kSsCard + c]);
        SerializedScoresAttr ssattr((int)ssser.size(), (int)(ssser.size() * sizeof(float)),
                                    1, 1, kSsCard, 1, kSsCard * (kSsCard + 1) / 2);
        SerializedDstMatchScoresAttr dmsattr(0, 0, kDmsCard, 0);
        DevBuf tabbuf;
        float* d_ss = (float*)tabbuf.alloc(up(ssser.size() * sizeof(float), kAlign) + kAlign,
                                           "tables");
        ck(cudaMemcpy(d_ss, ssser.data(), ssser.size() * sizeof(float), cudaMemcpyHostToDevice),
           "SS table");
        float* d_dms = d_ss + up(ssser.size(), 64);

        // heap sections (CuDeviceMemory.cu:548-588) for one chunk of dblen
        // positions in which all P profiles may pass
        const size_t dp2n = dblen, dp2p = P;
        const size_t szsm = up(Lq * dblen * sizeof(float), kAlign);
        const size_t diagw = (size_t)dpdssDiagM * nTDPDiagScoreSubsections + 1;
        const size_t szdpdiag = up((dblen + 64) * diagw * sizeof(float), kAlign);
        const size_t szdpbot = up((dblen + 64) * nTDPDiagScoreSubsections * sizeof(float), kAlign);
        const size_t szdpmax = up((dblen + 64) * sizeof(unsigned), kAlign);
        const size_t szdpbt = up((dblen + 64) * Lq, kAlign);
        const size_t szdp2diag = up((dp2n + 64) * diagw * sizeof(float), kAlign);
        const size_t szdp2bot = up((dp2n + 64) * nTDPDiagScoreSubsections * sizeof(float), kAlign);
        const size_t szdp2max = up((dp2n + 64) * sizeof(unsigned), kAlign);
        const size_t szdp2bt = up((dp2n + 64) * Lq, kAlign);
        const size_t szdp2fwd = up(dp2n * Lq * sizeof(float), kAlign);
        const size_t szss2 = up(dp2p * CUSS_ALIGNED_N_DIFF_TOTAL_SCORES * sizeof(float), kAlign);
        const size_t szaln = up(dp2p * nTDP2OutputAlnData * sizeof(float), kAlign);
        const size_t szalns = up((dp2n + dp2p * (Lq + 1) + 64) * nTDP2OutputAlignmentSSS, kAlign);
        const size_t szglb = up(4 * sizeof(int), kAlign);   // dgvNPassedPros..dgvMutex

        const size_t oScores = 0;
        const size_t oMod = oScores + szsm;
        const size_t oR = oMod + szsm;                      // end of modular scores
        const size_t oDPDiagEnd = oR + szdpdiag;
        const size_t oDPBotEnd = oDPDiagEnd + szdpbot;
        const size_t oDPMaxEnd = oDPBotEnd + szdpmax;
        const size_t oDPBtEnd = oDPMaxEnd + szdpbt;
        const size_t oDP2DiagEnd = oR + szdp2diag;
        const size_t oDP2BotEnd = oDP2DiagEnd + szdp2bot;
        const size_t oDP2MaxEnd = oDP2BotEnd + szdp2max;
        const size_t oDP2BtEnd = oDP2MaxEnd + szdp2bt;
        const size_t oDP2FwdEnd = oDP2BtEnd + szdp2fwd;
        const size_t oSS2End = oDP2FwdEnd + szss2;
        const size_t oAlnEnd = oSS2End + szaln;
        const size_t oAlnsEnd = oAlnEnd + szalns;
        // without MAP the SS and alignment division follows the phase-1
        // division instead of overlapping it (CuDeviceMemory.cuh:755-790)
        const size_t oSS2Base0 = oDPBtEnd;
        const size_t oSS2End0 = oSS2Base0 + szss2;
        const size_t oAlnEnd0 = oSS2End0 + szaln;
        const size_t oAlnsEnd0 = oAlnEnd0 + szalns;
        size_t oGlob = J->nomapaln ? oAlnsEnd0 : oAlnsEnd;
        if (oGlob < oDPBtEnd)
            oGlob = oDPBtEnd;
        const size_t heapsz = oGlob + szglb + (1 << 20);
        DevBuf heapbuf;
        char* H = heapbuf.alloc(heapsz, "heap");
        float* scores = (float*)(H + oScores);
        float* modscores = (float*)(H + oMod);
        unsigned* glob = (unsigned*)(H + oGlob);

        // CVS map and its attributes
        SerializedCVS2ScoresAttr cvattr;
        float* d_cvs = nullptr;
        DevBuf cvsbuf;
        if (J->cvswgt > 0.0f) {
            const int card = J->cvscard;
            int shift = 0;
            while (shift < card && J->cvskeys[shift] < 0.0f) shift++;
            std::vector<float> ser;
            ser.push_back(1.0f);              // the one level
            ser.push_back((float)card);
            ser.push_back((float)shift);
            ser.push_back(1.0f);              // scale
            for (int i = 0; i < card; i++) ser.push_back(J->cvskeys[i]);
            for (int i = 0; i < card; i++) ser.push_back(J->cvsscores[i]);
            d_cvs = (float*)cvsbuf.alloc(up(ser.size() * sizeof(float), kAlign), "CVS map");
            ck(cudaMemcpy(d_cvs, ser.data(), ser.size() * sizeof(float), cudaMemcpyHostToDevice),
               "CVS map");
            cvattr.ntotents_ = (int)ser.size();
            cvattr.szalloc_ = (int)(ser.size() * sizeof(float));
            cvattr.nenos_ = 1;
            cvattr.ntbls_ = 1;
            cvattr.card_ = card;
            cvattr.shft_ = shift;
            cvattr.key1first_ = J->cvskeys[0];
            cvattr.value1first_ = J->cvsscores[0];
            cvattr.key1last_ = J->cvskeys[card - 1];
            cvattr.value1last_ = J->cvsscores[card - 1];
            const int dim = 19;
            const float kappa0 = 0.1f, nu0 = (float)dim;
            const float pw = -0.5f * (nu0 + 2.f);
            float ct = (0.5f * dim + pw) * (logf(kappa0) - logf(kappa0 + 2.f));
            float sum = 0.0f;
            for (int i = 1; i <= dim; i++) sum += logf(nu0 + 1.0f - i) - 0.69314718055994530942f;
            ct += sum;
            cvattr.CVS_loKAPPA0_ = 1.f / kappa0;
            cvattr.CVS_PowerNU0_ = pw;
            cvattr.CVS_CTERM_ = ct;
        }

        const bool modinuse = J->ssswgt > 0.0f || J->cvswgt > 0.0f;
        const uint nq = (uint)Lq, n1 = 0, nC = (uint)N, pad = (uint)dbxpad;
        Events ev;
        for (float& t : J->stage_ms) t = 0.0f;
        ck(cudaDeviceSynchronize(), "setup");
        ck(cudaEventRecord(ev.e[0]), "event");

        // --- score matrix
        dim3 sthr(SMINIT_2DCACHE_DIM, SMINIT_2DCACHE_DIM, 1);
        dim3 sblk((unsigned)((N + 2 * sthr.x - 1) / (2 * sthr.x)),
                  (unsigned)((Lq + sthr.y - 1) / sthr.y), 1);
        CalcSM_Init_SMEMUnroll2x<<<sblk, sthr>>>(nq, n1, nC, pad, 0, 0, 0,
                                                  J->nomapaln ? CONSTINITSHIFT_MAPALN0
                                                              : CONSTINITSHIFT_MAPALN1,
                                                  scores, NULL);
        ck_launch("init scores");
        FtorRoundMAPALN1 ftor_mapaln1;
        FtorRoundMAPALN0 ftor_mapaln0;
        if (J->ssswgt > 0.0f && J->cvswgt > 0.0f) {
            if (J->nomapaln)
                CalcSM_SSSS_CVS2S_SMEMUnroll2x<<<sblk, sthr, ssattr.szalloc_ + cvattr.szalloc_>>>(
                    d_ss, ssattr, J->ssswgt, d_cvs, cvattr, J->cvswgt, nq, n1, nC, pad, 0, 0, 0,
                    ftor_mapaln0, scores, modscores);
            else
                CalcSM_SSSS_CVS2S_SMEMUnroll2x<<<sblk, sthr, ssattr.szalloc_ + cvattr.szalloc_>>>(
                    d_ss, ssattr, J->ssswgt, d_cvs, cvattr, J->cvswgt, nq, n1, nC, pad, 0, 0, 0,
                    ftor_mapaln1, scores, modscores);
            ck_launch("SS+CVS scores");
        } else if (J->ssswgt > 0.0f) {
            CalcSM_SSSS_SMEMUnroll2x<<<sblk, sthr, ssattr.szalloc_>>>(
                d_ss, ssattr, J->ssswgt, nq, n1, nC, pad, 0, 0, 0, scores, modscores);
            ck_launch("SS scores");
        } else if (J->cvswgt > 0.0f) {
            // the reference adds into modular scores it never initialised;
            // start them at zero here
            ck(cudaMemset(modscores, 0, Lq * dblen * sizeof(float)), "modscores");
            if (J->nomapaln)
                CalcSM_CVS2S_SMEMUnroll2x<<<sblk, sthr, cvattr.szalloc_>>>(
                    d_cvs, cvattr, J->cvswgt, nq, n1, nC, pad, 0, 0, 0, ftor_mapaln0, scores,
                    modscores);
            else
                CalcSM_CVS2S_SMEMUnroll2x<<<sblk, sthr, cvattr.szalloc_>>>(
                    d_cvs, cvattr, J->cvswgt, nq, n1, nC, pad, 0, 0, 0, ftor_mapaln1, scores,
                    modscores);
            ck_launch("CVS scores");
        }
        if (J->ddmswgt > 0.0f) {
            CalcSM_DDMS2S_SMEMUnroll2x_h2<DMS_STEP, DMS_LINEAR_INTERP_HALF, DMS_DSTBNDF>
                <<<sblk, sthr, dmsattr.szalloc_>>>(d_dms, dmsattr, J->ddmswgt, J->dstsegm,
                                                   nq, n1, nC, pad, 0, 0, 0, scores, modscores);
            ck_launch("DDMS scores");
        }
        ck(cudaEventRecord(ev.e[1]), "event");
        ck(cudaDeviceSynchronize(), "score matrix");
        ck(cudaEventElapsedTime(&J->stage_ms[0], ev.e[0], ev.e[1]), "event time");
        if (J->copy_matrices) {
            ck(cudaMemcpy(J->scores, scores, Lq * dblen * sizeof(float), cudaMemcpyDeviceToHost),
               "scores");
            ck(cudaMemcpy(J->modscores, modscores, Lq * dblen * sizeof(float),
                          cudaMemcpyDeviceToHost), "modscores");
        }

        // --- phase-1 DP over block diagonals
        {
            float* diag = (float*)(H + oR);
            float* bot = (float*)(H + oDPDiagEnd);
            unsigned* maxc = (unsigned*)(H + oDPBotEnd);
            char* btck = H + oDPMaxEnd;
            const uint w = CUDP_2DCACHE_DIM_D;
            const size_t len1 = (size_t)J->dbpro1len;
            dim3 thr(w, 1, 1);
            dim3 blk(blocks_per_diagonal(len1, Lq, w, CUDP_2DCACHE_DIM_X), (unsigned)P, 1);
            uint nblkdiags = (uint)(((len1 + Lq) + CUDP_2DCACHE_DIM_X - 1) / CUDP_2DCACHE_DIM_X);
            nblkdiags += (uint)(Lq - 1) / w;
            uint nintdivs = (uint)(Lq - 1) / w;
            float nsepds = (float)CUDP_2DCACHE_DIM_D / (float)CUDP_2DCACHE_DIM_X + 1.0f;
            uint lastdiag = (uint)(nsepds * (float)nintdivs) + 1 - 1;
            ck(cudaEventRecord(ev.e[1]), "event");
            for (uint dd = 0; dd < nblkdiags; dd++) {
                ExecDP_Btck_Unroll32x<<<blk, thr>>>(dd, lastdiag, 0, 0, 0, 0, nq, n1, nC, pad,
                                                     0, 0, 0, scores, diag, bot, maxc, btck);
                ck_launch("phase-1 DP");
            }
            FinalizeDP<<<1, 1>>>(J->scorethld, 0, (uint)P, 0, 0, n1, nC, pad, 0, 0, scores,
                                 diag, bot, maxc, (char*)btck, glob);
            ck_launch("FinalizeDP");
            ck(cudaEventRecord(ev.e[2]), "event");
            ck(cudaDeviceSynchronize(), "phase 1");
            ck(cudaEventElapsedTime(&J->stage_ms[1], ev.e[1], ev.e[2]), "event time");
            if (J->copy_matrices)
                ck(cudaMemcpy(J->btck, btck, Lq * dblen, cudaMemcpyDeviceToHost), "btck");
            ck(cudaMemcpy(J->phase1, diag, P * nTDP2OutputPhase1 * sizeof(float),
                          cudaMemcpyDeviceToHost), "phase-1 records");
            ck(cudaMemcpy(J->globvars, glob, 4 * sizeof(unsigned), cudaMemcpyDeviceToHost),
               "global variables");
        }

        const size_t npass = J->globvars[0];
        const size_t nposits = J->globvars[1];
        const size_t maxlen = J->globvars[2];
        J->dbalnlen2 = 0;
        if (npass < 1 || nposits < 1 || maxlen < 1)
            return 0;
        if (npass > P)
            throw Fail{"more passed profiles than profiles"};

        // --- statistics
        float* ss2 = (float*)(H + (J->nomapaln ? oSS2Base0 : oDP2FwdEnd));
        float* alndat = (float*)(H + (J->nomapaln ? oSS2End0 : oSS2End));
        ck(cudaEventRecord(ev.e[2]), "event");
        CalcStatisticsDynPlm<<<(unsigned)npass, 1>>>(
            J->xuninf != 0, 0, 0, 0, nq, n1, nC, pad, 0, 0, 0, J->ssemodel, J->qyeno,
            J->searchspace, J->reflambda, J->refK, J->explambda, J->expK, scores,
            (float*)(H + oR), ss2, alndat);
        ck_launch("statistics");
        ck(cudaEventRecord(ev.e[3]), "event");
        ck(cudaDeviceSynchronize(), "statistics");
        ck(cudaEventElapsedTime(&J->stage_ms[2], ev.e[2], ev.e[3]), "event time");
        ck(cudaMemcpy(J->stats, alndat, npass * nTDP2OutputAlnData * sizeof(float),
                      cudaMemcpyDeviceToHost), "statistics records");

        // --- MAP realignment
        const size_t dbxpad2 = up(nposits, CUL2CLINESIZE) - nposits;
        const size_t dbalnlen2 = up(nposits + npass * (Lq + 1), CUL2CLINESIZE);
        const uint dblen2 = (uint)(nposits + dbxpad2);
        J->dbalnlen2 = dbalnlen2;
        if (dbalnlen2 > J->alns_cap)
            throw Fail{"alignment buffer too small"};
        if (nposits + dbxpad2 > dp2n + 64)
            throw Fail{"phase-2 positions exceed the planned sections"};
        if (J->nomapaln) {
            // MAPALN=0 (CuBatchDP::FinalizeALNDynProgDevice, CuBatchDP.cu:427-530)
            char* outalns = H + oAlnEnd0;
            ck(cudaEventRecord(ev.e[3]), "event");
            FinalizeDP_ALN<<<(unsigned)npass, CUDP_2DCACHE_DIM_D>>>(
                J->ssswgt > 0.0f, J->logevthld, 0, 0, 0, 0, nq, n1, nC, pad, 0, 0, 0, dblen2,
                (uint)dbxpad2, (uint)dbalnlen2, scores, (const float*)(H + oR),
                (const uint*)(H + oDPBotEnd), (const char*)(H + oDPMaxEnd), alndat, outalns);
            ck_launch("ALN finalize");
            ck(cudaEventRecord(ev.e[4]), "event");
            ck(cudaDeviceSynchronize(), "ALN finalize");
            ck(cudaEventElapsedTime(&J->stage_ms[3], ev.e[3], ev.e[4]), "event time");
            ck(cudaMemcpy(J->final_recs, alndat, npass * nTDP2OutputAlnData * sizeof(float),
                          cudaMemcpyDeviceToHost), "final records");
            for (int r = 0; r < nTDP2OutputAlignmentSSS; r++)
                ck(cudaMemcpy(J->alns + (size_t)r * J->alns_cap, outalns + (size_t)r * dbalnlen2,
                              dbalnlen2, cudaMemcpyDeviceToHost), "alignments");
            return 0;
        }
        {
            float* diag = (float*)(H + oR);
            float* bot = (float*)(H + oDP2DiagEnd);
            unsigned* maxc = (unsigned*)(H + oDP2BotEnd);
            char* btck = H + oDP2MaxEnd;
            float* fwd = (float*)(H + oDP2BtEnd);
            char* outalns = H + oAlnEnd;
            const float ext = J->minpp, extgap = J->minpp * 0.5f;
            const uint w = CUMAPDP_2DCACHE_DIM_D;
            dim3 thr(w, 1, 1);
            dim3 blk(blocks_per_diagonal(maxlen, Lq, w, CUMAPDP_2DCACHE_DIM_X),
                     (unsigned)npass, 1);
            uint nblkdiags = (uint)(((maxlen + Lq) + CUMAPDP_2DCACHE_DIM_X - 1) /
                                    CUMAPDP_2DCACHE_DIM_X);
            nblkdiags += (uint)((Lq - 1) / w);
            uint nintdivs = (uint)((Lq - 1) / w);
            float nsepds = (float)CUMAPDP_2DCACHE_DIM_D / (float)CUMAPDP_2DCACHE_DIM_X + 1.0f;
            uint lastdiag = (uint)(nsepds * (float)nintdivs) + 1 - 1;
            ck(cudaEventRecord(ev.e[3]), "event");
            for (uint dd = 0; dd < nblkdiags; dd++) {
                ExecMAPDP_Fwd_Unroll32x<<<blk, thr>>>(
                    dd, lastdiag, J->logevthld, modinuse, 0, 0, 0, 0, nq, n1, nC, pad, 0, 0, 0,
                    dblen2, (uint)dbxpad2, scores, modscores, alndat, diag, bot, fwd);
                ck_launch("MAP forward");
            }
            for (int dd = (int)nblkdiags - 1; 0 <= dd; dd--) {
                ExecMAPDP_Bwd_Unroll32x<<<blk, thr>>>(
                    (uint)dd, lastdiag, J->logevthld, modinuse, 0, 0, 0, 0, nq, n1, nC, pad, 0,
                    0, 0, dblen2, (uint)dbxpad2, scores, modscores, alndat, diag, bot, fwd, ss2);
                ck_launch("MAP backward");
            }
            for (uint dd = 0; dd < nblkdiags; dd++) {
                ExecMAPDP_MAP_Btck_Unroll32x<<<blk, thr>>>(
                    ext, extgap, dd, lastdiag, J->logevthld, 0, 0, 0, 0, nq, dblen2,
                    (uint)dbxpad2, fwd, alndat, diag, bot, ss2, maxc, btck);
                ck_launch("MAP DP");
            }
            FinalizeMAPDP_MAP<<<(unsigned)npass, w>>>(
                J->ssswgt > 0.0f, J->logevthld, 0, 0, 0, 0, nq, n1, nC, pad, 0, 0, 0, dblen2,
                (uint)dbxpad2, (uint)dbalnlen2, scores, diag, maxc, btck, alndat, outalns);
            ck_launch("MAP finalize");
            ck(cudaEventRecord(ev.e[4]), "event");
            ck(cudaDeviceSynchronize(), "MAP");
            ck(cudaEventElapsedTime(&J->stage_ms[3], ev.e[3], ev.e[4]), "event time");
            ck(cudaMemcpy(J->final_recs, alndat, npass * nTDP2OutputAlnData * sizeof(float),
                          cudaMemcpyDeviceToHost), "final records");
            for (int r = 0; r < nTDP2OutputAlignmentSSS; r++)
                ck(cudaMemcpy(J->alns + (size_t)r * J->alns_cap, outalns + (size_t)r * dbalnlen2,
                              dbalnlen2, cudaMemcpyDeviceToHost), "alignments");
        }
        return 0;
    } catch (const Fail& f) {
        g_err = f.msg;
    } catch (...) {
        g_err = "unknown failure";
    }
    return 1;
}

}  // extern "C"
