// C ABI and host driver of the search path (the role of the reference's
// CuBatchProcessing, src/libmycu/cupro/CuBatchProcessing.cu:189-697, and of
// its device-memory planner CuDeviceMemory, src/libmycu/cupro/CuDeviceMemory.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cother_b200.h"
#include "common.cuh"
#include "layout.h"
#include "score_kernel.cuh"
#include "tc_kernel.cuh"
#include "dp1_kernel.cuh"
#include "hits_kernel.cuh"
#include "stats_kernel.cuh"
#include "map_kernel.cuh"

namespace cbp {

// format.cpp: the finalizer's per-hit text from host records and rows
int format_hits_from(const float* recs, size_t nrecs, const int32_t* order, size_t norder, const char* rows,
                     size_t row_stride, size_t row_length,
                     const int* prof_len, const float* prof_eno, const uint8_t* prof_ss, size_t nprof,
                     const char* const* descs, int query_len, float query_eno, int query_ss, float ssswgt,
                     float logevthld, float sspace, const cbp_format_options* fo, char* buf, size_t cap,
                     size_t* used, size_t* nhits);

// field indices (src/libmycu/cupro/PM2DVectorFields.h:51-87)
enum {
    fBkg = 0, fENO = 20, fLen = 21, fDist = 22, fTrn = 23, fTF = 30, fCV = 50,
    fDD = 71, fSS = 171, fAddrPro = 176, fAddrSS = 178, fAA = 179, fSSstate = 180, fTot = 181
};

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

// Parameters of the significance networks and of the SS18 model
// adjustments (the reference's static table SSE_NN_WEIGHTS_,
// src/libmycu/cupro/CuDeviceMemory.cu:43-80): E-network mu (4x5 + 5),
// lambda-network mu (4x5 + 5), lambda-network scale (4x5 + 5), then 9
// adjustment parameters for each of the SS18 variants 1 and 2.
static const float kNNWeightsTable[kNNWeights] = {
    3.1179029f, 0.2732032f, -1.7865388f, -2.7370650f, -2.4113938f,
    2.8802990f, -0.0845794f, 0.7335855f, -0.4155596f, -3.5943765f,
    -2.3533863f, -0.1646748f, 2.6470928f, 1.6489798f, -0.7481717f,
    -0.1763256f, 0.3270687f, 0.5918245f, 0.4900585f, 0.0253580f,
    2.0547640f, 1.4051396f, -1.7874640f, 2.0048461f, 0.6947985f,
    -0.0605839f, 0.0533123f, -1.0046299f, 0.9682557f, 0.0f,
    -0.0173019f, -0.0051053f, 0.6215832f, -0.5038284f, 0.0f,
    0.0600411f, -0.0527767f, 1.0036328f, -0.9667071f, 0.0f,
    -5.9555713f, -3.1437676f, 1.8754493f, 3.4776044f, 0.0f,
    2.8086869f, -0.5250554f, 0.3085814f, 0.5244239f, 2.4166220f,
    -4.4935289f, -11.5416831f, 0.4601384f, 4.1707612f, 0.0f,
    1.4710020f, 0.7746900f, 0.5248285f, -2.2621661f, 0.0f,
    -1.4710009f, -0.7746948f, -0.5248293f, 2.2621667f, 0.0f,
    4.8137710f, 1.0000337f, 2.0837171f, -5.3104535f, 0.0f,
    2.5137293f, 4.2316344f, -0.8620832f, 0.8620837f, 3.1901578f,
    0.1f, 12.0f, 1.0f, 4.0f, 0.05f, 1.0f, 0.1f, 0.35f, 0.65f,
    0.6f, 16.0f, 1.0f, 12.0f, 0.3f, -1.7f, 0.1f, 0.45f, 0.65f,
};

// Length adjustment for edge effects and the effective search space:
// the expected alignment length l solves l = alpha/lambda ln(K (m-l)(n-Nl))
// + beta (Altschul et al., NAR 29, 2001), found by the bracketed iteration
// of Gertz (2005) as in src/libpro/srcsco/AbstractScoreMatrix.cpp:303-393.
static void length_adjustment(float lambda, float K, float alpha, float beta, size_t m,
                              unsigned long long n, size_t N, unsigned long long* sspace_out,
                              size_t* delta_out)
{
    *sspace_out = (unsigned long long)m * n;
    *delta_out = 0;
    if (lambda <= 0.0f || K <= 0.0f || N < 1) return;
    const float logK = logf(K);
    const float alratio = alpha / lambda;
    const float max_mn = (float)(m > n ? m : n);
    float length = 0.0f, min_length = 0.0f, max_length, nxt_length = 0.0f, sspace = 0.0f;
    bool converged = false;
    const float qa = (float)N;
    const float qb = (float)(n + (unsigned long long)m * N);
    const float qc = (float)((unsigned long long)m * n) - max_mn / K;
    if (qc < 0.0f) return;
    max_length = 2.0f * qc / (qb + sqrtf(qb * qb - 4.0f * qa * qc));
    for (int j = 0; j < 20; j++) {
        length = nxt_length;
        sspace = ((float)m - length) * ((float)n - (float)N * length);
        nxt_length = alratio * (logK + logf(sspace)) + beta;
        if (length <= nxt_length) {
            min_length = length;
            if (nxt_length - length <= 1.0f) { converged = true; break; }
            if (min_length == max_length) break;
        } else {
            max_length = length;
        }
        if (nxt_length < min_length || max_length < nxt_length)
            nxt_length = (!j) ? max_length : (min_length + max_length) * 0.5f;
    }
    if (converged) {
        length = ceilf(min_length);
        if (length <= max_length) {
            const float space2 = ((float)m - length) * ((float)n - (float)N * length);
            nxt_length = alratio * (logK + logf(space2)) + beta;
            if (length <= nxt_length) { min_length = length; sspace = space2; }
        }
    }
    *sspace_out = (unsigned long long)sspace;
    *delta_out = (size_t)min_length;
}

// A device buffer that only grows.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void reserve(size_t n) {
        if (n <= bytes) return;
        if (p) CBP_CUDA(cudaFree(p));
        p = nullptr; bytes = 0;
        CBP_CUDA(cudaMalloc(&p, n));
        bytes = n;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr; bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Device copy of a packed profile set.
struct ProfilesStore {
    DevBuf tf, ss, dst, dstlen, trn, bkg, eno, plen, pstart, pro, aa, sss, cv, cvprior, cvnorm2;
    ProfilesDev view;
    std::vector<int> h_plen;
    std::vector<long long> h_pstart;
    // for the text output: ENO per profile and whether the profile carries
    // SS data (pmv2DAddrSS of its first position is not -1; empty when the
    // field was not given)
    std::vector<float> h_eno;
    std::vector<uint8_t> h_ss;
    ProfilesStore() = default;
    ProfilesStore(const ProfilesStore&) = delete;
    ProfilesStore& operator=(const ProfilesStore&) = delete;
    ~ProfilesStore() { release(); }
    size_t bytes() const {
        size_t n = 0;
        for (const DevBuf* b : {&tf, &ss, &dst, &dstlen, &trn, &bkg, &eno, &plen, &pstart, &pro, &aa,
                                &sss, &cv, &cvprior, &cvnorm2})
            n += b->bytes;
        return n;
    }
    void release() {
        for (DevBuf* b : {&tf, &ss, &dst, &dstlen, &trn, &bkg, &eno, &plen, &pstart, &pro, &aa, &sss,
                          &cv, &cvprior, &cvnorm2})
            b->release();
        view = ProfilesDev();
        h_plen.clear();
        h_pstart.clear();
        h_eno.clear();
        h_ss.clear();
    }
};

}  // namespace cbp

using namespace cbp;

namespace cbp {
// Kernel variants for one query-length bin: rows per block of the score
// kernel, the column-ordering window, warps per block of the phase-1 DP;
// and, once tuned, each candidate's time on the sample.
constexpr int kScoreCandidates = 5;
constexpr int kDpCandidates = 2;
constexpr int kScoreRowsCand[kScoreCandidates] = {16, 8, 32, 16, 16};
constexpr int kWindowCand[kScoreCandidates] = {1024, 1024, 1024, 256, 4096};
constexpr int kDpWarpsCand[kDpCandidates] = {2, 1};
constexpr int kPreferredScoreCand = 2;     // 32 rows, window 1,024
constexpr float kTuneMargin = 0.015f;      // a candidate must be this much faster to replace it
struct Tuning {
    int rows = 16, window = kOrderWindow, dp_warps = 2;
    bool tuned = false;
    float score_ms[kScoreCandidates] = {};
    float dp_ms[kDpCandidates] = {};
    long long sample_cols = 0;
};
// The results of one query of a cbp_process or cbp_process_batch call.
struct QueryResult {
    int Lq = 0;
    int row0 = 0;                    // its first row in the (stacked) score matrix
    float eno = 0.f;
    float score_thld = 0.f, logE_thld = 0.f;
    unsigned long long searchspace = 0;
    size_t delta_length = 0;
    std::vector<float> h_recs;       // hit records, all slabs
    std::vector<char> h_alns[5];     // alignment rows, all slabs
    std::vector<int32_t> h_order;    // reported hits in the finalizer's order (sorted on the device)
    long long base_len = 0, base_npass = 0;   // running phase-2 offsets over slabs
    long long last_npos2 = 0;
};
}  // namespace cbp

struct cbp_context {
    int device = 0;
    cbp_options opt{};
    cudaStream_t stream = nullptr;
    float sstab_h[kSSCard * kSSCard];
    float dmstab_h[kDstCard * kDstCard];
    DevBuf sstab, dmstab;
    // tensor-core form of the profile-profile term
    DevBuf tcq;            // the query operand image of the tensor-core form
    DevBuf tcerr;          // set by the tensor-core kernel when a wait gave up
    int h_tcerr = 0;
    // the resident database chunk; contexts on one device may share it
    // (cbp_share_database), the last owner frees it
    std::shared_ptr<ProfilesStore> db = std::make_shared<ProfilesStore>();
    ProfilesStore query;
    bool have_db = false;
    size_t mem_budget = 0;
    size_t max_slab_positions = 0;
    // settings
    uint64_t db_len = 0;
    size_t n_seqs = 0;
    size_t query_len = 0;
    float score_thld = 0.f;
    float logE_thld = 0.f;
    // Karlin-Altschul parameters (cother.par: [UNGAPPED], [GAPPED_A_1])
    float ref_lambda = 1.116276f, ref_K = 0.115812f;
    float gap_lambda = 0.561132f, gap_K = 0.001488f, gap_alpha = 0.5f, gap_beta = -1.0f;
    DevBuf nnweights;
    // context-vector score map (cbp_set_cvs2s_map)
    DevBuf cvsmap;
    bool have_cvs = false;
    int cvs_card = 0, cvs_shift = 0;
    float cvs_key_first = 0.f, cvs_key_last = 0.f;
    // working buffers
    DevBuf scores, modscores, btck, bandbuf, colorder, dpmax, dpcoords, dprecs, passidx, passdst, passcnt;
    DevBuf hitrecs, statrecs, cs2, fb2, sg2, bt2, strip2, maperr, alnbuf, dp1err;
    DevBuf hitkeys, hitcnt;    // sort keys of all records of a query, reported count
    DevBuf fits;               // the precision forms: FP64 and FP32 parameter fits per passed pair
    DevBuf qtrn;               // batches: each query's transitions as [7][Lq+1]

    int h_maperr = 0;   // set by the MAP stage when a wait between warps gave up
    // the last MAP realignment (last slab, last query of the call), for
    // cbp_read_map_fb: its pass list, phase-2 columns and band geometry
    int last_map_np = 0;
    long long last_map_nd = 0;
    int last_map_Lq = 0;
    int last_map_p0 = 0;
    const int* last_map_pass_idx = nullptr;
    const long long* last_map_pass_dst = nullptr;
    int h_dp1err = 0;   // set when a staging wait gave up: 2 by the score kernel, 1 by the phase-1 DP
    bool score_thld_set = false, logE_thld_set = false;
    // results of the last process() call, all slabs
    std::vector<QueryResult> res;   // per query of the last call
    size_t cur = 0;                 // the query the result calls read (cbp_select_query)
    // last slab
    long long last_col0 = 0;
    int last_ncols = 0;
    long long last_ld = 0;
    int last_first_profile = 0;
    int last_Lq = 0;
    long long last_row0 = 0;        // first score-matrix row of the inspected query
    long long last_dp_off = 0;      // its slot in the phase-1 buffers (profiles)
    int last_nprof = 0;
    int last_npass = 0;
    // kernel variants chosen by the tuner, per query-length bin (Lq / 64)
    std::map<int, Tuning> tuning;
    // executable CUDA graph of a slab's phase 1 (plain form)
    cudaGraphExec_t phase1_exec = nullptr;
    uint64_t graph_launches = 0;
    // instrumentation
    cudaEvent_t ev[8]{};
    float stage_ms[6] = {0, 0, 0, 0, 0, 0};
    uint64_t launches = 0;
    uint64_t stage_launches[6] = {0, 0, 0, 0, 0, 0};
};

namespace {

template <class F>
int guarded(F&& f)
{
    try {
        f();
        g_last_error.clear();
        return CBP_OK;
    } catch (const cbp::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return CBP_ERR_ARG;
    }
}

void parallel_for(long long n, const std::function<void(long long, long long)>& fn)
{
    int nt = (int)std::min<long long>(std::max(1u, std::thread::hardware_concurrency()), 32);
    if (n < 65536 || nt <= 1) { fn(0, n); return; }
    std::vector<std::thread> th;
    long long per = (n + nt - 1) / nt;
    for (int t = 0; t < nt; t++) {
        long long a = t * per, b = std::min(n, a + per);
        if (a >= b) break;
        th.emplace_back(fn, a, b);
    }
    for (auto& x : th) x.join();
}

size_t field_bytes(char* const* beg, char* const* end, int f)
{
    if (!beg[f] || !end[f] || end[f] < beg[f])
        throw Error(CBP_ERR_ARG, "field " + std::to_string(f) + ": invalid begin/end pointers");
    return (size_t)(end[f] - beg[f]);
}

// Repack 181 SoA host fields into the device layout (layout.h) and upload.
// Upload a packed profile set. With `with_cv` the context-vector fields
// (pmv2DCVentrs.., pmv2DCVprior, pmv2DCVnorm2) are uploaded too.
void upload_profiles(ProfilesStore& st, char* const* beg, char* const* end, cudaStream_t stream,
                     bool with_cv)
{
    if (!beg || !end) throw Error(CBP_ERR_ARG, "null field tables");
    const size_t P = field_bytes(beg, end, fLen) / sizeof(int);
    const size_t N = field_bytes(beg, end, fTF) / sizeof(float);
    if (P == 0 || N == 0) throw Error(CBP_ERR_ARG, "empty profile set");
    if (field_bytes(beg, end, fTrn) / sizeof(float) != N + P)
        throw Error(CBP_ERR_ARG, "transition fields must hold N+P entries");
    for (int a = 0; a < kNAA; a++) {
        if (field_bytes(beg, end, fTF + a) != N * sizeof(float))
            throw Error(CBP_ERR_ARG, "target-frequency fields of unequal size");
        if (field_bytes(beg, end, fBkg + a) != P * sizeof(float))
            throw Error(CBP_ERR_ARG, "background fields of unequal size");
    }
    for (int s = 0; s < 100; s++)
        if (field_bytes(beg, end, fDD + s) != N * sizeof(float))
            throw Error(CBP_ERR_ARG, "distance fields of unequal size");
    if (with_cv)
        for (int k = 0; k < kNCV + 2; k++)
            if (field_bytes(beg, end, fCV + k) != N * sizeof(float))
                throw Error(CBP_ERR_ARG, "context-vector fields missing or of unequal size");
    const int* lens = reinterpret_cast<const int*>(beg[fLen]);
    const uint32_t* dists = reinterpret_cast<const uint32_t*>(beg[fDist]);
    st.h_plen.assign(lens, lens + P);
    st.h_pstart.resize(P);
    long long acc = 0;
    for (size_t p = 0; p < P; p++) {
        if (lens[p] <= 0) throw Error(CBP_ERR_ARG, "profile of non-positive length");
        if (lens[p] >= 65536) throw Error(CBP_ERR_LIMIT, "profile length must be < 65536");
        if ((long long)dists[p] != acc && !(P == 1))
            throw Error(CBP_ERR_ARG, "profile offsets (pps2DDist) do not follow the lengths");
        st.h_pstart[p] = acc;
        acc += lens[p];
    }
    if ((size_t)acc != N) throw Error(CBP_ERR_ARG, "sum of profile lengths differs from #positions");
    {
        const float* eno = reinterpret_cast<const float*>(beg[fENO]);
        if (field_bytes(beg, end, fENO) != P * sizeof(float)) throw Error(CBP_ERR_ARG, "ENO field of wrong size");
        st.h_eno.assign(eno, eno + P);
        st.h_ss.clear();
        if (beg[fAddrSS] && end[fAddrSS] && (size_t)(end[fAddrSS] - beg[fAddrSS]) == N * sizeof(int)) {
            const int* addr = reinterpret_cast<const int*>(beg[fAddrSS]);
            st.h_ss.resize(P);
            for (size_t p = 0; p < P; p++) st.h_ss[p] = addr[st.h_pstart[p]] != -1 ? 1 : 0;
        }
    }

    // packed distance lists
    std::vector<uint8_t> dst((size_t)N * kDstStride);
    std::vector<uint8_t> dlen(N);
    const float* dd[100];
    for (int s = 0; s < 100; s++) dd[s] = reinterpret_cast<const float*>(beg[fDD + s]);
    std::string perr;
    std::mutex emu;
    parallel_for((long long)N, [&](long long a, long long b) {
        for (long long n = a; n < b; n++) {
            const int cnt = (int)dd[0][n];
            uint8_t* o = dst.data() + (size_t)n * kDstStride;
            if (cnt < 0 || cnt > kMaxDst) {
                std::lock_guard<std::mutex> g(emu);
                perr = "distance count out of range at position " + std::to_string(n);
                return;
            }
            dlen[n] = (uint8_t)cnt;
            int k = 0;
            for (; k < cnt; k++) {
                int v = (int)dd[k + 1][n];
                if (v < 0) {
                    std::lock_guard<std::mutex> g(emu);
                    perr = "negative distance at position " + std::to_string(n);
                    return;
                }
                o[k] = (uint8_t)(v == 255 ? kDstNoData : (v < 20 ? v : 20));
            }
            for (; k < kDstStride; k++) o[k] = (uint8_t)kDstNoData;
        }
    });
    if (!perr.empty()) throw Error(CBP_ERR_ARG, perr);

    // profile index of every position, derived from the lengths (the
    // pmv2DAddrPro field is not trusted for addressing)
    std::vector<int> pro(N);
    for (size_t p = 0; p < P; p++)
        std::fill(pro.begin() + st.h_pstart[p], pro.begin() + st.h_pstart[p] + lens[p], (int)p);

    auto up = [&](DevBuf& b, const void* src, size_t bytes) {
        b.reserve(std::max<size_t>(bytes, 16));
        CBP_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, stream));
    };
    auto up_rows = [&](DevBuf& b, int f0, int nrows, size_t row_elems, size_t esz) {
        b.reserve(std::max<size_t>(nrows * row_elems * esz, 16));
        for (int r = 0; r < nrows; r++)
            CBP_CUDA(cudaMemcpyAsync(b.as<char>() + r * row_elems * esz, beg[f0 + r], row_elems * esz,
                                     cudaMemcpyHostToDevice, stream));
    };
    up_rows(st.tf, fTF, kNAA, N, sizeof(float));
    up_rows(st.ss, fSS, kNSS, N, sizeof(float));
    up_rows(st.trn, fTrn, kNTrn, N + P, sizeof(float));
    up_rows(st.bkg, fBkg, kNAA, P, sizeof(float));
    up(st.eno, beg[fENO], P * sizeof(float));
    up(st.plen, lens, P * sizeof(int));
    up(st.pstart, st.h_pstart.data(), P * sizeof(long long));
    up(st.pro, pro.data(), N * sizeof(int));
    up(st.aa, beg[fAA], N);
    up(st.sss, beg[fSSstate], N);
    up(st.dst, dst.data(), dst.size());
    up(st.dstlen, dlen.data(), N);
    if (with_cv) {
        up_rows(st.cv, fCV, kNCV, N, sizeof(float));
        up(st.cvprior, beg[fCV + kNCV], N * sizeof(float));
        up(st.cvnorm2, beg[fCV + kNCV + 1], N * sizeof(float));
    }
    CBP_CUDA(cudaStreamSynchronize(stream));

    ProfilesDev& v = st.view;
    v.N = (long long)N; v.P = (int)P;
    v.tf = st.tf.as<float>(); v.ss = st.ss.as<float>();
    v.dst = st.dst.as<uint8_t>(); v.dstlen = st.dstlen.as<uint8_t>();
    v.trn = st.trn.as<float>(); v.bkg = st.bkg.as<float>(); v.eno = st.eno.as<float>();
    v.plen = st.plen.as<int>(); v.pstart = st.pstart.as<long long>();
    v.pro = st.pro.as<int>(); v.aa = st.aa.as<int8_t>(); v.sss = st.sss.as<int8_t>();
    v.cv = with_cv ? st.cv.as<float>() : nullptr;
    v.cvprior = with_cv ? st.cvprior.as<float>() : nullptr;
    v.cvnorm2 = with_cv ? st.cvnorm2.as<float>() : nullptr;
}

void check_ctx(cbp_context* c)
{
    if (!c) throw Error(CBP_ERR_ARG, "null context");
    CBP_CUDA(cudaSetDevice(c->device));
}

// Working bytes per slab position for a query of length Lq: score matrix,
// modular scores and phase-1 backtrack per query row (9 Lq), the score
// kernel's column order, the phase-1 band strip and per-profile records
// (172), and the phase-2 buffers for the
// worst case of every profile realigned: cell scores and forward-backward
// values per row of the padded bands (8 x 32 nb), backtrack and sign words
// per band (12 nb), band edges (4 x 48) and alignment rows (5, plus the 5 Lq
// bytes of each pair's slot, counted per position). The tensor-core form
// adds its operands.
size_t slab_bytes_per_position(const cbp_options& o, int Lq)
{
    const size_t nb = (size_t)map_bands(Lq);
    size_t b = (size_t)Lq * 9 + 172 + nb * (8 * 32 + 12) + 4 * kMapMaxWarps * kMapEdgeFields + 5 +
               (size_t)Lq * 5;
    (void)o;   // the tensor-core form needs only the query's operand image (per query, not per position)
    return b;
}

// bytes per slab independent of its size: the 31 extra diagonal rows of
// the phase-2 bands
size_t slab_fixed_bytes(int Lq)
{
    return 31 * (size_t)map_bands(Lq) * (8 * 32 + 12);
}

// Constants of the context-vector score (_TCTXVECT::_TCTXVECT,
// src/libpro/srcpro/TCTXVECT.cpp:26-60), computed in float with the host's
// logf as the reference does: dimension 19, kappa0 0.1, nu0 19;
// 1/kappa0, -(nu0+2)/2 and (dim/2 - (nu0+2)/2) (ln kappa0 - ln(kappa0+2))
// + sum_{i=1..dim} (ln(nu0+1-i) - ln 2).
const QueryResult& cur_result(const cbp_context* c)
{
    static const QueryResult kNone;
    return c->cur < c->res.size() ? c->res[c->cur] : kNone;
}

void cvs_constants(float* lokappa0, float* pownu0, float* cterm)
{
    const int dim = 19;
    const float kappa0 = 0.1f, nu0 = (float)dim;
    const float pw = -0.5f * (nu0 + 2.f);
    float ct = (0.5f * dim + pw) * (logf(kappa0) - logf(kappa0 + 2.f));
    float sum = 0.0f;
    for (int i = 1; i <= dim; i++) sum += logf(nu0 + 1.0f - i) - 0.69314718055994530942f;
    ct += sum;
    *lokappa0 = 1.f / kappa0;
    *pownu0 = pw;
    *cterm = ct;
}

// Slabs of whole profiles whose score matrices fit the working budget.
struct Slab { int p0, p1; long long col0; int ncols; };

std::vector<Slab> plan_slabs(const cbp_context* c, int Lq)
{
    const ProfilesStore& db = *c->db;
    const int P = (int)db.h_plen.size();
    const size_t per_pos = slab_bytes_per_position(c->opt, Lq);
    const size_t fixed = slab_fixed_bytes(Lq);
    size_t cap = c->mem_budget > fixed ? (c->mem_budget - fixed) / per_pos : 0;
    if (c->max_slab_positions) cap = std::min(cap, c->max_slab_positions);
    cap = std::min<size_t>(cap, (size_t)1 << 30);
    std::vector<Slab> out;
    int p = 0;
    while (p < P) {
        long long start = db.h_pstart[p];
        int q = p;
        long long n = 0;
        while (q < P && (size_t)(n + db.h_plen[q]) <= cap) { n += db.h_plen[q]; q++; }
        if (q == p) {
            if (cap < (size_t)db.h_plen[p])
                throw Error(CBP_ERR_MEMORY, "working memory too small for one profile of length " +
                                                std::to_string(db.h_plen[p]));
        }
        out.push_back({p, q, start, (int)n});
        p = q;
    }
    return out;
}

// The tuner: on the first slab of a query-length bin, time each candidate
// kernel variant on a sample of the slab (its first profiles, up to 32,768
// positions, all query rows) and keep the fastest. Every variant computes
// the same cells, so the choice changes the time, never a result; the
// sample's outputs are overwritten by the slab's own launches.
void tune_kernels(cbp_context* c, const ScoreArgs& base, int p0, int p1, Tuning& t)
{
    const ProfilesStore& db = *c->db;
    int pe = p0;
    long long ncols = 0;
    while (pe < p1 && (pe == p0 || ncols + db.h_plen[pe] <= 32768)) ncols += db.h_plen[pe++];
    ScoreArgs a = base;
    a.ncols = (int)ncols;
    a.ld = align_up(ncols, 32);
    a.dots_in_scores = false;
    cudaEvent_t e0 = c->ev[6], e1 = c->ev[7];
    auto time_it = [&](const std::function<void()>& launch) {
        float best = 0.f;
        for (int rep = 0; rep < 2; rep++) {
            CBP_CUDA(cudaEventRecord(e0, c->stream));
            launch();
            CBP_CUDA(cudaEventRecord(e1, c->stream));
            CBP_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            CBP_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (rep == 0 || ms < best) best = ms;
        }
        return best;
    };
    int bs = 0;
    for (int k = 0; k < kScoreCandidates; k++) {
        a.rows = kScoreRowsCand[k];
        t.score_ms[k] = time_it([&] {
            if (a.colorder)
                launch_column_order(db.view.dstlen, a.col0, a.ncols, a.ld, kWindowCand[k], c->colorder.as<int>(),
                                    c->stream);
            launch_score_matrix(a, c->stream);
        });
        c->launches += 4;
        if (t.score_ms[k] < t.score_ms[bs]) bs = k;
    }
    // The candidates' sample times lie within about 1 % of each other, the
    // sample's noise. Unless one is clearly faster, keep 32 rows per block
    // with the default window: the fewest re-reads of the database lists,
    // and the fastest on full-size slabs.
    if (t.score_ms[bs] > (1.0f - kTuneMargin) * t.score_ms[kPreferredScoreCand]) bs = kPreferredScoreCand;
    Dp1Args d;
    d.scores = a.scores;
    d.ld = a.ld;
    d.Lq = a.Lq;
    d.qtrn = c->query.view.trn;
    d.db = db.view;
    d.col0 = a.col0;
    d.p0 = p0;
    d.nprof = pe - p0;
    d.btck = c->btck.as<uint8_t>();
    d.bandbuf = c->bandbuf.as<float>();
    d.maxsc = c->dpmax.as<float>();
    d.maxcoords = c->dpcoords.as<uint32_t>();
    d.recs = c->dprecs.as<Dp1Rec>();
    // timed as the search runs it: the launch without backtrack codes over
    // every profile, then the codes launch, here with no candidate
    d.code_thld = INFINITY;
    int bd = 0;
    for (int k = 0; k < kDpCandidates; k++) {
        d.warps = kDpWarpsCand[k];
        int nl = 0;
        t.dp_ms[k] = time_it([&] { nl = launch_dp1(d, c->stream); });
        c->launches += 2 * (uint64_t)nl;   // two timed repetitions
        if (t.dp_ms[k] < t.dp_ms[bd]) bd = k;
    }
    t.rows = kScoreRowsCand[bs];
    t.window = kWindowCand[bs];
    t.dp_warps = kDpWarpsCand[bd];
    t.sample_cols = ncols;
    t.tuned = true;
}

}  // namespace

namespace {

// The field tables of nq single-profile queries as one profile set: each
// field's bytes in query order (per-position and per-profile fields alike),
// the profile offsets (pps2DDist) recomputed from the lengths. A field
// missing from any query is left out.
struct StackedTables {
    std::vector<std::vector<char>> bytes;
    char* beg[CBP_NFIELDS];
    char* end[CBP_NFIELDS];
};

void stack_tables(size_t nq, char* const* const* qbeg, char* const* const* qend, StackedTables& t)
{
    t.bytes.assign(CBP_NFIELDS, {});
    for (int f = 0; f < CBP_NFIELDS; f++) {
        bool all = true;
        size_t total = 0;
        for (size_t k = 0; k < nq; k++) {
            if (!qbeg[k] || !qend[k]) throw Error(CBP_ERR_ARG, "null field tables");
            if (!qbeg[k][f] || !qend[k][f] || qend[k][f] < qbeg[k][f]) { all = false; break; }
            total += (size_t)(qend[k][f] - qbeg[k][f]);
        }
        if (!all) { t.beg[f] = t.end[f] = nullptr; continue; }
        std::vector<char>& v = t.bytes[f];
        v.resize(std::max<size_t>(total, 1));
        size_t off = 0;
        for (size_t k = 0; k < nq; k++) {
            const size_t n = (size_t)(qend[k][f] - qbeg[k][f]);
            if (n) std::memcpy(v.data() + off, qbeg[k][f], n);
            off += n;
        }
        t.beg[f] = v.data();
        t.end[f] = v.data() + total;
    }
    if (!t.beg[fLen] || !t.beg[fDist] ||
        (size_t)(t.end[fLen] - t.beg[fLen]) != nq * sizeof(int) ||
        (size_t)(t.end[fDist] - t.beg[fDist]) != nq * sizeof(uint32_t))
        throw Error(CBP_ERR_ARG, "each query's field tables must hold one profile");
    const int* lens = reinterpret_cast<const int*>(t.beg[fLen]);
    uint32_t* dist = reinterpret_cast<uint32_t*>(t.beg[fDist]);
    uint32_t acc = 0;
    for (size_t k = 0; k < nq; k++) {
        dist[k] = acc;
        acc += (uint32_t)lens[k];
    }
}

// One search of nq queries against the resident chunk. The queries' rows
// are stacked into one score matrix per slab (one column-order and one
// score-kernel launch for all of them: one pass over the slab's database
// columns); phase 1 of each query follows in the same CUDA graph, each on
// its rows of the matrix and its own phase-1 buffers; statistics, MAP and
// the hit order then run per query. With nq == 1 this is the search of one
// query (CuBatchProcessing::ProcessScoreMatrix).
void process_queries(cbp_context* c, size_t nq, const size_t* qlens, char* const* const* qbeg,
                     char* const* const* qend)
{
    check_ctx(c);
    if (!c->have_db) throw Error(CBP_ERR_STATE, "no database chunk transferred");
    if (nq == 0) throw Error(CBP_ERR_ARG, "no query");
    if (c->opt.cvswgt > 0.0f) {
        if (!c->have_cvs)
            throw Error(CBP_ERR_STATE, "CVSWGT > 0 needs the context-vector map (cbp_set_cvs2s_map)");
        if (!c->db->view.cv)
            throw Error(CBP_ERR_STATE, "CVSWGT > 0 needs a database chunk with context vectors "
                                       "(transferred by a context with CVSWGT > 0)");
    }
    if (nq == 1) {
        upload_profiles(c->query, qbeg[0], qend[0], c->stream, c->opt.cvswgt > 0.0f);
        if (c->query.view.P != 1) throw Error(CBP_ERR_ARG, "the query field tables must hold one profile");
    } else {
        StackedTables t;
        stack_tables(nq, qbeg, qend, t);
        upload_profiles(c->query, t.beg, t.end, c->stream, c->opt.cvswgt > 0.0f);
    }
    const int Ltot = (int)c->query.view.N;
    std::vector<QueryResult> res(nq);
    {
        long long row = 0;
        for (size_t k = 0; k < nq; k++) {
            if ((size_t)c->query.h_plen[k] != qlens[k])
                throw Error(CBP_ERR_ARG, "query_len differs from the query profile length");
            QueryResult& r = res[k];
            r.Lq = (int)qlens[k];
            r.row0 = (int)row;
            r.eno = c->query.h_eno[k];
            row += r.Lq;
            // effective search space (AbstractScoreMatrix::ComputeLengthAdjustment);
            // the query length and the database totals default to this
            // query and this chunk when not set
            const size_t m = (nq == 1 && c->query_len) ? c->query_len : (size_t)r.Lq;
            const unsigned long long n = c->db_len ? c->db_len : (unsigned long long)c->db->view.N;
            const size_t N = c->n_seqs ? c->n_seqs : (size_t)c->db->view.P;
            length_adjustment(c->gap_lambda, c->gap_K, c->gap_alpha, c->gap_beta, m, n, N, &r.searchspace,
                              &r.delta_length);
            // thresholds not set by the caller follow from EVAL as the
            // reference's job dispatcher derives them
            float sthld = 0.f, lthld = 0.f;
            cbp_score_threshold(m, n, c->opt.eval, c->gap_lambda, c->gap_K, &sthld, &lthld);
            r.score_thld = c->score_thld_set ? c->score_thld : sthld;
            r.logE_thld = c->logE_thld_set ? c->logE_thld : lthld;
        }
    }
    c->launches = 0;
    c->last_map_np = 0;
    for (float& m : c->stage_ms) m = 0.f;
    for (uint64_t& m : c->stage_launches) m = 0;
    c->res.clear();
    c->cur = 0;

    std::vector<Slab> slabs = plan_slabs(c, Ltot);
    size_t maxcols = 0, maxprof = 0;
    for (const Slab& s : slabs) {
        maxcols = std::max(maxcols, (size_t)align_up(s.ncols, 32));
        maxprof = std::max(maxprof, (size_t)(s.p1 - s.p0));
    }
    const size_t keycap = (size_t)hit_sort_capacity(c->db->view.P);
    c->scores.reserve((size_t)Ltot * maxcols * sizeof(float));
    c->modscores.reserve((size_t)Ltot * maxcols * sizeof(float));
    c->btck.reserve((size_t)Ltot * maxcols);
    c->bandbuf.reserve(5 * maxcols * sizeof(float));
    c->colorder.reserve(maxcols * sizeof(int));
    c->dpmax.reserve(nq * maxprof * sizeof(float));
    c->dpcoords.reserve(nq * maxprof * sizeof(uint32_t));
    c->dprecs.reserve(nq * maxprof * sizeof(Dp1Rec));
    c->passidx.reserve(nq * maxprof * sizeof(int));
    c->passdst.reserve(nq * maxprof * sizeof(long long));
    c->passcnt.reserve(nq * 16);
    c->dp1err.reserve(sizeof(int));
    c->hitkeys.reserve(nq * keycap * sizeof(uint64_t));
    c->hitcnt.reserve(nq * sizeof(int));
    CBP_CUDA(cudaMemsetAsync(c->hitcnt.p, 0, nq * sizeof(int), c->stream));
    // each query's transitions as the kernels index them ([7][Lq+1])
    std::vector<const float*> qtrn(nq, c->query.view.trn);
    if (nq > 1) {
        size_t tot = 0;
        for (const QueryResult& r : res) tot += (size_t)kNTrn * (r.Lq + 1);
        c->qtrn.reserve(tot * sizeof(float));
        const long long NT = c->query.view.N + c->query.view.P;
        size_t off = 0;
        for (size_t k = 0; k < nq; k++) {
            const QueryResult& r = res[k];
            float* dst = c->qtrn.as<float>() + off;
            CBP_CUDA(cudaMemcpy2DAsync(dst, (size_t)(r.Lq + 1) * sizeof(float),
                                       c->query.view.trn + r.row0 + (long long)k, (size_t)NT * sizeof(float),
                                       (size_t)(r.Lq + 1) * sizeof(float), kNTrn, cudaMemcpyDeviceToDevice,
                                       c->stream));
            qtrn[k] = dst;
            off += (size_t)kNTrn * (r.Lq + 1);
        }
    }
    const bool tc = c->opt.tc_form != CBP_TC_PLAIN;

    for (const Slab& s : slabs) {
        ScoreArgs a;
        a.q = c->query.view;
        a.db = c->db->view;
        a.col0 = s.col0;
        a.ncols = s.ncols;
        a.ld = align_up(s.ncols, 32);
        a.Lq = Ltot;
        a.ssswgt = c->opt.ssswgt;
        a.ddmswgt = c->opt.ddmswgt;
        a.initshift = c->opt.mapaln ? 0.002f : 0.0003f;
        a.dstsegm = c->opt.dstsegm;
        if (c->opt.cvswgt > 0.0f) {
            a.cvswgt = c->opt.cvswgt;
            a.cvs_scores = c->cvsmap.as<float>();
            a.cvs_card = c->cvs_card;
            a.cvs_shift = c->cvs_shift;
            a.cvs_key_first = c->cvs_key_first;
            a.cvs_key_last = c->cvs_key_last;
            cvs_constants(&a.cvs_lokappa0, &a.cvs_pownu0, &a.cvs_cterm);
            a.cvs_int_priors = !c->opt.mapaln;
        }
        a.sstab = c->sstab.as<float>();
        a.dmstab = c->dmstab.as<float>();
        a.scores = c->scores.as<float>();
        a.modscores = c->modscores.as<float>();
        a.err = c->dp1err.as<int>();   // shared with the phase-1 DP: 2 = score kernel, 1 = DP
        // the column order only balances the DDMS loops of a warp's lanes;
        // without that term the identity keeps the stores coalesced
        a.colorder = a.ddmswgt > 0.0f ? c->colorder.as<int>() : nullptr;
        Tuning& tn = c->tuning[Ltot / 64];
        if (c->opt.autotune && !tn.tuned) tune_kernels(c, a, s.p0, s.p1, tn);
        a.rows = tn.rows;
        if (tc) {
            // the profile-profile sums on the tensor cores, per query (its
            // database operand depends on the query's background)
            CBP_CUDA(cudaEventRecord(c->ev[0], c->stream));
            const int f = c->opt.tc_form;
            size_t img = 0;
            for (const QueryResult& r : res) img = std::max(img, tc_query_image_bytes(f, r.Lq));
            c->tcq.reserve(img);
            c->tcerr.reserve(sizeof(int));
            CBP_CUDA(cudaMemsetAsync(c->tcerr.p, 0, sizeof(int), c->stream));
            for (size_t k = 0; k < nq; k++) {
                TcArgs t;
                t.q = a.q;
                t.db = a.db;
                t.col0 = a.col0;
                t.ncols = a.ncols;
                t.ld = a.ld;
                t.Lq = res[k].Lq;
                t.qrow0 = res[k].row0;
                t.qprof = (int)k;
                const int nl = tc_profile_sums(t, f, c->tcq.p, a.scores + (long long)res[k].row0 * a.ld,
                                               c->tcerr.as<int>(), c->stream);
                c->launches += nl;   // the query operand image and the tcgen05 contraction
                c->stage_launches[0] += nl;
            }
            CBP_CUDA(cudaMemcpyAsync(&c->h_tcerr, c->tcerr.p, sizeof(int), cudaMemcpyDeviceToHost,
                                     c->stream));
            a.dots_in_scores = true;
        }

        std::vector<Dp1Args> d(nq);
        for (size_t k = 0; k < nq; k++) {
            const QueryResult& r = res[k];
            d[k].scores = a.scores + (long long)r.row0 * a.ld;
            d[k].ld = a.ld;
            d[k].Lq = r.Lq;
            d[k].qtrn = qtrn[k];
            d[k].db = c->db->view;
            d[k].col0 = s.col0;
            d[k].p0 = s.p0;
            d[k].nprof = s.p1 - s.p0;
            d[k].btck = c->btck.as<uint8_t>() + (long long)r.row0 * a.ld;
            d[k].bandbuf = c->bandbuf.as<float>();
            d[k].maxsc = c->dpmax.as<float>() + k * maxprof;
            d[k].maxcoords = c->dpcoords.as<uint32_t>() + k * maxprof;
            // codes for the finalization's candidates only, unless all are asked for
            d[k].code_thld = c->opt.all_codes ? -INFINITY : r.score_thld;
            d[k].recs = c->dprecs.as<Dp1Rec>() + k * maxprof;
            d[k].warps = tn.dp_warps;
            d[k].err = c->dp1err.as<int>();
        }
        auto pass_idx = [&](size_t k) { return c->passidx.as<int>() + k * maxprof; };
        auto pass_dst = [&](size_t k) { return c->passdst.as<long long>() + k * maxprof; };
        auto pass_cnt = [&](size_t k) { return reinterpret_cast<int*>(c->passcnt.as<char>() + 16 * k); };
        auto pass_npos = [&](size_t k) { return reinterpret_cast<long long*>(c->passcnt.as<char>() + 16 * k + 8); };

        // phase 1 of the slab: column order, score matrix (all queries' rows),
        // each query's DP, finalization and pass list; with the plain form
        // one CUDA graph, captured here and swapped into the context's
        // executable graph by an update of its parameters
        int dp_launches = 0;
        auto phase1 = [&](bool capturing) {
            auto mark = [&](cudaEvent_t e) {
                if (capturing) CBP_CUDA(cudaEventRecordWithFlags(e, c->stream, cudaEventRecordExternal));
                else CBP_CUDA(cudaEventRecord(e, c->stream));
            };
            if (!tc) mark(c->ev[0]);
            CBP_CUDA(cudaMemsetAsync(c->dp1err.p, 0, sizeof(int), c->stream));
            if (a.colorder)
                launch_column_order(c->db->view.dstlen, s.col0, s.ncols, a.ld, tn.window, c->colorder.as<int>(),
                                    c->stream);
            launch_score_matrix(a, c->stream);
            mark(c->ev[1]);
            dp_launches = 0;
            for (size_t k = 0; k < nq; k++) dp_launches += launch_dp1(d[k], c->stream);
            mark(c->ev[2]);
            for (size_t k = 0; k < nq; k++) {
                launch_dp1_finalize(d[k], res[k].score_thld, c->stream);
                launch_pass_compact(d[k], pass_idx(k), pass_dst(k), pass_cnt(k), pass_npos(k), c->stream);
            }
            mark(c->ev[3]);
        };
        if (tc) {
            phase1(false);
        } else {
            CBP_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            cudaGraph_t g = nullptr;
            try {
                phase1(true);
            } catch (...) {
                cudaStreamEndCapture(c->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            CBP_CUDA(cudaStreamEndCapture(c->stream, &g));
            if (c->phase1_exec) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(c->phase1_exec, g, &info) != cudaSuccess) {
                    (void)cudaGetLastError();
                    cudaGraphExecDestroy(c->phase1_exec);
                    c->phase1_exec = nullptr;
                }
            }
            if (!c->phase1_exec) {
                const cudaError_t e = cudaGraphInstantiate(&c->phase1_exec, g, 0);
                if (e != cudaSuccess) {
                    cudaGraphDestroy(g);
                    c->phase1_exec = nullptr;
                    CBP_CUDA(e);
                }
            }
            cudaGraphDestroy(g);
            CBP_CUDA(cudaGraphLaunch(c->phase1_exec, c->stream));
            c->graph_launches += 1;
        }
        c->launches += 2 + (uint64_t)dp_launches + 2 * (uint64_t)nq;
        c->stage_launches[0] += 2;
        c->stage_launches[1] += (uint64_t)dp_launches;
        c->stage_launches[2] += 2 * (uint64_t)nq;
        std::vector<int> npass(nq, 0);
        for (size_t k = 0; k < nq; k++)
            CBP_CUDA(cudaMemcpyAsync(&npass[k], pass_cnt(k), sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CBP_CUDA(cudaMemcpyAsync(&c->h_dp1err, c->dp1err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        if (c->h_dp1err == 2)
            throw Error(CBP_ERR_CUDA, "score matrix: a wait for the bulk-copied distance lists timed out");
        if (c->h_dp1err)
            throw Error(CBP_ERR_CUDA, "phase-1 DP: a wait for staged score rows timed out");
        if (tc && c->h_tcerr)
            throw Error(CBP_ERR_CUDA, "tensor-core contraction: a wait timed out");
        float ms = 0.f;
        CBP_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
        c->stage_ms[0] += ms;
        CBP_CUDA(cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]));
        c->stage_ms[1] += ms;
        CBP_CUDA(cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]));
        c->stage_ms[2] += ms;
        // the inspection calls (cbp_read_*) see the last query of the slab
        c->last_col0 = s.col0;
        c->last_ncols = s.ncols;
        c->last_ld = a.ld;
        c->last_first_profile = s.p0;
        c->last_Lq = res[nq - 1].Lq;
        c->last_row0 = res[nq - 1].row0;
        c->last_dp_off = (long long)(nq - 1) * (long long)maxprof;
        c->last_nprof = s.p1 - s.p0;
        c->last_npass = npass[nq - 1];

        for (size_t k = 0; k < nq; k++) {
            QueryResult& r = res[k];
            const int np = npass[k];
            if (np <= 0) continue;
            const int Lq = r.Lq;
            const float* sc = a.scores + (long long)r.row0 * a.ld;
            // statistics and E-values of the passed pairs of this slab
            c->hitrecs.reserve((size_t)np * kRecFloats * sizeof(float));
            StatsArgs st;
            st.scores = sc;
            st.ld = a.ld;
            st.Lq = Lq;
            st.col0 = s.col0;
            st.p0 = s.p0;
            st.db = c->db->view;
            st.qaa = c->query.view.aa + r.row0;
            st.qeno = r.eno;
            st.x_uninf = c->opt.x_uninf;
            st.pass_idx = pass_idx(k);
            st.pass_dst = pass_dst(k);
            st.recs = d[k].recs;
            st.out = c->hitrecs.as<float>();
            st.nnweights = c->nnweights.as<float>();
            st.ssemodel = c->opt.ssemodel;
            st.searchspace = (float)r.searchspace;
            st.ref_lambda = c->ref_lambda;
            st.ref_K = c->ref_K;
            st.exp_gapped_lambda = c->gap_lambda;
            st.exp_gapped_K = c->gap_K;
            if (tc) {
                // the precision forms fit lambda, K, H in FP64 for the E-values
                c->fits.reserve((size_t)np * kFitDoubles * sizeof(double));
                st.fits = c->fits.as<double>();
                st.use_fit64 = 1;
            }
            CBP_CUDA(cudaEventRecord(c->ev[4], c->stream));
            launch_stats(st, np, c->stream);
            CBP_CUDA(cudaEventRecord(c->ev[5], c->stream));
            // the records as the statistics leave them (cbp_read_statistics)
            c->statrecs.reserve((size_t)np * kRecFloats * sizeof(float));
            CBP_CUDA(cudaMemcpyAsync(c->statrecs.p, c->hitrecs.p, (size_t)np * kRecFloats * sizeof(float),
                                     cudaMemcpyDeviceToDevice, c->stream));
            c->launches += 1;
            c->stage_launches[3] += 1;

            // phase-2 MAP realignment of the pairs within the E-value
            // threshold (in the phase-2 column space of this slab)
            long long npos2 = 0;
            CBP_CUDA(cudaMemcpyAsync(&npos2, pass_npos(k), sizeof(long long), cudaMemcpyDeviceToHost,
                                     c->stream));
            CBP_CUDA(cudaStreamSynchronize(c->stream));
            const long long nd = map_diag_rows(npos2);
            const size_t nb = (size_t)map_bands(Lq);
            const long long alnstride = align_up(npos2 + (long long)np * Lq, 32);
            c->alnbuf.reserve(5 * (size_t)alnstride);
            MapArgs mp;
            mp.scores = sc;
            mp.modscores = a.modscores + (long long)r.row0 * a.ld;
            mp.ld = a.ld;
            mp.Lq = Lq;
            mp.col0 = s.col0;
            mp.p0 = s.p0;
            mp.db = c->db->view;
            mp.qtrn = qtrn[k];
            mp.qaa = c->query.view.aa + r.row0;
            mp.qsss = c->query.view.sss + r.row0;
            mp.printsss = c->opt.ssswgt > 0.0f;
            mp.modscores_inuse = (c->opt.ssswgt > 0.0f || c->opt.cvswgt > 0.0f) ? 1 : 0;
            mp.minpp = c->opt.minpp;
            mp.logevthld = r.logE_thld;
            mp.npass = np;
            mp.pass_idx = pass_idx(k);
            mp.pass_dst = pass_dst(k);
            mp.recs = c->hitrecs.as<float>();
            mp.alns = c->alnbuf.as<char>();
            mp.alnstride = alnstride;
            CBP_CUDA(cudaMemsetAsync(c->alnbuf.p, 0, 5 * (size_t)alnstride, c->stream));
            if (c->opt.mapaln) {
                c->cs2.reserve(nb * nd * 32 * sizeof(float));
                c->fb2.reserve(nb * nd * 32 * sizeof(float));
                c->sg2.reserve(nb * nd * sizeof(unsigned));
                c->bt2.reserve(nb * nd * sizeof(unsigned long long));
                c->strip2.reserve((size_t)map_strip_floats(npos2) * sizeof(float));
                c->maperr.reserve(sizeof(int));
                mp.nd = nd;
                mp.cs = c->cs2.as<float>();
                mp.fb = c->fb2.as<float>();
                mp.sg = c->sg2.as<unsigned>();
                mp.bt = c->bt2.as<unsigned long long>();
                mp.strip = c->strip2.as<float>();
                mp.err = c->maperr.as<int>();
                CBP_CUDA(cudaMemsetAsync(c->maperr.p, 0, sizeof(int), c->stream));
                CBP_CUDA(cudaEventRecord(c->ev[6], c->stream));
                launch_map(mp, c->stream);
                CBP_CUDA(cudaEventRecord(c->ev[7], c->stream));
                c->last_map_np = np;
                c->last_map_nd = nd;
                c->last_map_Lq = Lq;
                c->last_map_p0 = s.p0;
                c->last_map_pass_idx = mp.pass_idx;
                c->last_map_pass_dst = mp.pass_dst;
                CBP_CUDA(cudaMemcpyAsync(&c->h_maperr, c->maperr.p, sizeof(int), cudaMemcpyDeviceToHost,
                                         c->stream));
                c->launches += 2;
                c->stage_launches[4] += 2;
            } else {
                // MAPALN=0: the phase-1 alignments themselves
                // (CuBatchDP::FinalizeALNDynProgDevice)
                CBP_CUDA(cudaEventRecord(c->ev[6], c->stream));
                launch_aln_final(mp, d[k].btck, d[k].maxsc, d[k].maxcoords, c->stream);
                CBP_CUDA(cudaEventRecord(c->ev[7], c->stream));
                c->launches += 1;
                c->stage_launches[4] += 1;
            }
            r.last_npos2 = npos2;
            // sort keys of this slab's records, for the hit order
            c->launches += launch_hit_keys(c->hitrecs.as<float>(), np, r.logE_thld, r.base_npass,
                                           c->hitkeys.as<uint64_t>() + k * keycap, c->hitcnt.as<int>() + k,
                                           c->stream);
            c->stage_launches[5] += 1;
            const size_t off = r.h_recs.size();
            r.h_recs.resize(off + (size_t)np * kRecFloats);
            CBP_CUDA(cudaMemcpyAsync(r.h_recs.data() + off, c->hitrecs.p, (size_t)np * kRecFloats * sizeof(float),
                                     cudaMemcpyDeviceToHost, c->stream));
            // this slab's alignment rows go to the running offset of
            // the whole result (slot of pair K at newDst + K*Lq)
            const long long shift = r.base_len + r.base_npass * (long long)Lq;
            const long long slablen = npos2 + (long long)np * Lq;
            for (int row = 0; row < 5; row++) {
                r.h_alns[row].resize((size_t)(shift + slablen), 0);
                CBP_CUDA(cudaMemcpyAsync(r.h_alns[row].data() + shift, c->alnbuf.as<char>() + (size_t)row * alnstride,
                                         (size_t)slablen, cudaMemcpyDeviceToHost, c->stream));
            }
            CBP_CUDA(cudaStreamSynchronize(c->stream));
            if (c->opt.mapaln && c->h_maperr)
                throw Error(CBP_ERR_CUDA, "MAP realignment: a wait between the warps of a pair timed out");
            CBP_CUDA(cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]));
            c->stage_ms[3] += ms;
            CBP_CUDA(cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]));
            c->stage_ms[4] += ms;
            // phase-2 offsets of this slab's pairs become offsets in the
            // whole result
            for (size_t i = off; i < r.h_recs.size(); i += kRecFloats) {
                uint32_t v;
                std::memcpy(&v, &r.h_recs[i + rProNewDst], 4);
                v += (uint32_t)r.base_len;
                std::memcpy(&r.h_recs[i + rProNewDst], &v, 4);
            }
            r.base_len += npos2;
            r.base_npass += np;
        }
    }
    // the reported hits of each query in the finalizer's order: one sort
    // over the keys of all its records; the reported ones come first
    for (size_t k = 0; k < nq; k++) {
        QueryResult& r = res[k];
        if (r.base_npass <= 0) continue;
        uint64_t* keys_d = c->hitkeys.as<uint64_t>() + k * keycap;
        CBP_CUDA(cudaEventRecord(c->ev[4], c->stream));
        const int nl = launch_hit_sort(keys_d, r.base_npass, c->stream);
        CBP_CUDA(cudaEventRecord(c->ev[5], c->stream));
        c->launches += nl;
        c->stage_launches[5] += nl;
        int nrep = 0;
        CBP_CUDA(cudaMemcpyAsync(&nrep, c->hitcnt.as<int>() + k, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        if (nrep < 0 || nrep > r.base_npass) throw Error(CBP_ERR_CUDA, "hit order: inconsistent count");
        std::vector<uint64_t> keys((size_t)nrep);
        if (nrep > 0)
            CBP_CUDA(cudaMemcpyAsync(keys.data(), keys_d, (size_t)nrep * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                     c->stream));
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        r.h_order.resize((size_t)nrep);
        for (int i = 0; i < nrep; i++) r.h_order[i] = (int32_t)(uint32_t)keys[i];
        float ms = 0.f;
        CBP_CUDA(cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]));
        c->stage_ms[5] += ms;
    }
    CBP_CUDA(cudaStreamSynchronize(c->stream));
    c->res = std::move(res);
    c->cur = 0;
}

}  // namespace

extern "C" {

void cbp_default_options(cbp_options* o)
{
    if (!o) return;
    o->ssswgt = 0.12f;
    o->cvswgt = 0.0f;
    o->ddmswgt = 0.2f;
    o->dstsegm = 6;
    o->mapaln = 1;
    o->minpp = 0.28f;
    o->ssemodel = 2;
    o->x_uninf = 1;
    o->eval = 10.0f;
    o->nohits = 700;
    o->noalns = 700;
    o->tc_form = CBP_TC_PLAIN;
    o->autotune = 1;
    o->all_codes = 0;
}

const char* cbp_last_error(void) { return g_last_error.c_str(); }

int cbp_create(int device, const cbp_options* opt, const float* ss_table, size_t dev_mem_bytes,
               cbp_context** out)
{
    return guarded([&] {
        if (!out) throw Error(CBP_ERR_ARG, "null output pointer");
        *out = nullptr;
        if (!opt || !ss_table) throw Error(CBP_ERR_ARG, "null options or SS table");
        if (!(opt->cvswgt >= 0.0f && opt->cvswgt < 1.0f))
            throw Error(CBP_ERR_ARG, "CVSWGT must be in [0, 1)");
        // value ranges of src/libpro/srcpro/MOptions.cpp:76-141
        if (!(opt->ssswgt >= 0.0f && opt->ssswgt < 1.0f))
            throw Error(CBP_ERR_ARG, "SSSWGT must be in [0,1)");
        if (!(opt->ddmswgt >= 0.0f && opt->ddmswgt < 1.0f))
            throw Error(CBP_ERR_ARG, "DDMSWGT must be in [0,1)");
        if (opt->dstsegm < 1 || opt->dstsegm > 20) throw Error(CBP_ERR_ARG, "DSTSEGM must be in [1,20]");
        if (opt->ssemodel < 0 || opt->ssemodel > 2) throw Error(CBP_ERR_ARG, "SSEMODEL must be 0, 1 or 2");
        if (!(opt->minpp >= 0.0f && opt->minpp < 1.0f)) throw Error(CBP_ERR_ARG, "MINPP must be in [0,1)");
        if (!(opt->eval >= 0.0f)) throw Error(CBP_ERR_ARG, "EVAL must be >= 0");
        if (opt->tc_form < CBP_TC_PLAIN || opt->tc_form > CBP_TC_TF32X3)
            throw Error(CBP_ERR_ARG, "tc_form must be CBP_TC_PLAIN, CBP_TC_BF16X3 or CBP_TC_TF32X3");
        int ndev = 0;
        CBP_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw Error(CBP_ERR_ARG, "invalid device");
        CBP_CUDA(cudaSetDevice(device));
        auto* c = new cbp_context();
        try {
            c->device = device;
            c->opt = *opt;
            CBP_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
            for (auto& e : c->ev) CBP_CUDA(cudaEventCreate(&e));
            dp1_set_attributes();
            tc_set_attributes();
            std::memcpy(c->sstab_h, ss_table, sizeof(c->sstab_h));
            build_dms_table(c->dmstab_h);
            c->nnweights.reserve(sizeof(kNNWeightsTable));
            CBP_CUDA(cudaMemcpy(c->nnweights.p, kNNWeightsTable, sizeof(kNNWeightsTable),
                                cudaMemcpyHostToDevice));
            c->sstab.reserve(sizeof(c->sstab_h));
            c->dmstab.reserve(sizeof(c->dmstab_h));
            CBP_CUDA(cudaMemcpy(c->sstab.p, c->sstab_h, sizeof(c->sstab_h), cudaMemcpyHostToDevice));
            CBP_CUDA(cudaMemcpy(c->dmstab.p, c->dmstab_h, sizeof(c->dmstab_h), cudaMemcpyHostToDevice));
            size_t fr = 0, tot = 0;
            CBP_CUDA(cudaMemGetInfo(&fr, &tot));
            c->mem_budget = dev_mem_bytes ? dev_mem_bytes : (size_t)(0.7 * (double)fr);
        } catch (...) {
            cbp_destroy(c);
            throw;
        }
        *out = c;
    });
}

int cbp_destroy(cbp_context* c)
{
    if (!c) return CBP_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->db.reset();
    c->query.release();
    if (c->phase1_exec) cudaGraphExecDestroy(c->phase1_exec);
    for (DevBuf* b : {&c->scores, &c->modscores, &c->btck, &c->bandbuf, &c->colorder, &c->dpmax, &c->dpcoords,
                      &c->dprecs, &c->passidx, &c->passdst, &c->passcnt, &c->hitrecs, &c->nnweights,
                      &c->cs2, &c->fb2, &c->sg2, &c->bt2, &c->strip2, &c->maperr, &c->alnbuf,
                      &c->cvsmap, &c->statrecs, &c->dp1err, &c->hitkeys, &c->hitcnt, &c->fits, &c->qtrn})
        b->release();
    c->sstab.release();
    c->dmstab.release();
    for (DevBuf* b : {&c->tcq, &c->tcerr}) b->release();
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return CBP_OK;
}

int cbp_set_db_details(cbp_context* c, uint64_t db_len, size_t n_seqs)
{
    return guarded([&] { check_ctx(c); c->db_len = db_len; c->n_seqs = n_seqs; });
}

int cbp_set_query_len(cbp_context* c, size_t qlen)
{
    return guarded([&] { check_ctx(c); c->query_len = qlen; });
}

int cbp_set_score_threshold(cbp_context* c, float t)
{
    return guarded([&] { check_ctx(c); c->score_thld = t; c->score_thld_set = true; });
}

int cbp_set_logE_threshold(cbp_context* c, float t)
{
    return guarded([&] { check_ctx(c); c->logE_thld = t; c->logE_thld_set = true; });
}

int cbp_set_max_slab_positions(cbp_context* c, size_t n)
{
    return guarded([&] { check_ctx(c); c->max_slab_positions = n; });
}

int cbp_transfer_chunk(cbp_context* c, char* const* beg, char* const* end, const size_t*)
{
    return guarded([&] {
        check_ctx(c);
        c->have_db = false;
        c->last_map_np = 0;   // the last search's phase-2 matrices refer to the old chunk
        // a fresh store: contexts sharing the previous one keep it
        auto st = std::make_shared<ProfilesStore>();
        upload_profiles(*st, beg, end, c->stream, c->opt.cvswgt > 0.0f);
        c->db = std::move(st);
        c->have_db = true;
    });
}

int cbp_device_memory(int device, size_t* free_bytes, size_t* total_bytes)
{
    return guarded([&] {
        if (!free_bytes || !total_bytes) throw Error(CBP_ERR_ARG, "null output pointer");
        int ndev = 0;
        CBP_CUDA(cudaGetDeviceCount(&ndev));
        if (device < 0 || device >= ndev) throw Error(CBP_ERR_ARG, "invalid device");
        CBP_CUDA(cudaSetDevice(device));
        CBP_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
    });
}

int cbp_slab_bytes(const cbp_options* opt, size_t query_len, size_t positions, size_t* bytes)
{
    return guarded([&] {
        if (!opt || !bytes) throw Error(CBP_ERR_ARG, "null options or output pointer");
        if (query_len < 1 || query_len > (size_t)INT32_MAX) throw Error(CBP_ERR_ARG, "invalid query length");
        const int Lq = (int)query_len;
        *bytes = slab_fixed_bytes(Lq) + slab_bytes_per_position(*opt, Lq) * positions;
    });
}

int cbp_share_database(cbp_context* c, cbp_context* owner)
{
    return guarded([&] {
        check_ctx(c);
        check_ctx(owner);
        if (c->device != owner->device)
            throw Error(CBP_ERR_ARG, "contexts on different devices cannot share a database");
        if (!owner->have_db) throw Error(CBP_ERR_STATE, "the owner has no database chunk");
        CBP_CUDA(cudaStreamSynchronize(owner->stream));   // its upload has completed
        c->last_map_np = 0;
        c->db = owner->db;
        c->have_db = true;
    });
}

int cbp_get_capacities(cbp_context* c, size_t query_len, size_t expected_profile_length,
                       size_t* max_db_pos, size_t* max_db_pros, size_t* max_pass2_pos,
                       size_t* max_pass2_pros)
{
    return guarded([&] {
        check_ctx(c);
        if (!max_db_pos || !max_db_pros || !max_pass2_pos || !max_pass2_pros)
            throw Error(CBP_ERR_ARG, "null output pointer");
        if (query_len < 1 || query_len > (size_t)INT32_MAX || expected_profile_length < 1)
            throw Error(CBP_ERR_ARG, "invalid query or profile length");
        *max_db_pos = *max_db_pros = *max_pass2_pos = *max_pass2_pros = 0;
        const int Lq = (int)query_len;
        const size_t slab = slab_fixed_bytes(Lq) + slab_bytes_per_position(c->opt, Lq) * expected_profile_length;
        if (slab > c->mem_budget) return;
        // resident bytes of a chunk, as upload_profiles stores it: per
        // position target frequencies, SS, transitions, packed distances,
        // list length, profile index, residue, SS state (and context
        // vectors); per profile its beginning transitions, background,
        // ENO, length and offset
        size_t per_pos = kNAA * 4 + kNSS * 4 + kNTrn * 4 + kDstStride + 1 + 4 + 1 + 1;
        if (c->opt.cvswgt > 0.0f) per_pos += (kNCV + 2) * 4;
        const size_t per_prof = kNTrn * 4 + kNAA * 4 + 4 + 4 + 8;
        CBP_CUDA(cudaSetDevice(c->device));
        size_t free_b = 0, total_b = 0;
        CBP_CUDA(cudaMemGetInfo(&free_b, &total_b));
        size_t held_working = 0;
        for (const DevBuf* b : {&c->scores, &c->modscores, &c->btck, &c->bandbuf, &c->dpmax,
                                &c->dpcoords, &c->dprecs, &c->passidx, &c->passdst, &c->passcnt,
                                &c->hitrecs, &c->statrecs, &c->cs2, &c->fb2, &c->sg2, &c->bt2,
                                &c->strip2, &c->maperr, &c->alnbuf})
            held_working += b->bytes;
        const size_t held_chunk = (c->db.use_count() == 1) ? c->db->bytes() : 0;
        const size_t still = c->mem_budget > held_working ? c->mem_budget - held_working : 0;
        const long long avail = (long long)free_b + (long long)held_chunk - (long long)still -
                                (long long)(total_b / 100);
        if (avail <= 0) return;
        const size_t pros = (size_t)avail / (per_prof + expected_profile_length * per_pos);
        *max_db_pros = *max_pass2_pros = pros;
        *max_db_pos = *max_pass2_pos = pros * expected_profile_length;
    });
}

int cbp_set_cvs2s_map(cbp_context* c, const float* keys, const float* scores, size_t card)
{
    return guarded([&] {
        check_ctx(c);
        if (!keys || !scores) throw Error(CBP_ERR_ARG, "null keys or scores");
        if (card < 1 || card > 100000) throw Error(CBP_ERR_ARG, "invalid map cardinality");
        // the lookup (SerializedCVS2Scores::GetScoreE1S1Step2Boundary) indexes
        // the scores by shift + rint(2 x score): keys must be the halves
        // (i - shift)/2, shift the number of negative keys
        int shift = 0;
        while ((size_t)shift < card && keys[shift] < 0.0f) shift++;
        for (size_t i = 0; i < card; i++)
            if (keys[i] != 0.5f * (float)((long long)i - shift))
                throw Error(CBP_ERR_ARG, "CVS map keys must be consecutive halves");
        for (size_t i = 0; i < card; i++)
            if (!std::isfinite(scores[i])) throw Error(CBP_ERR_ARG, "non-finite CVS map score");
        CBP_CUDA(cudaSetDevice(c->device));
        c->cvsmap.reserve(card * sizeof(float));
        CBP_CUDA(cudaMemcpy(c->cvsmap.p, scores, card * sizeof(float), cudaMemcpyHostToDevice));
        c->cvs_card = (int)card;
        c->cvs_shift = shift;
        c->cvs_key_first = keys[0];
        c->cvs_key_last = keys[card - 1];
        c->have_cvs = true;
    });
}

int cbp_process(cbp_context* c, int /*query_serial*/, size_t query_len, char* const* qbeg,
                char* const* qend)
{
    return guarded([&] { process_queries(c, 1, &query_len, &qbeg, &qend); });
}

int cbp_process_batch(cbp_context* c, size_t nqueries, const size_t* query_lens, char* const* const* qbeg,
                      char* const* const* qend)
{
    return guarded([&] {
        if (!query_lens || !qbeg || !qend) throw Error(CBP_ERR_ARG, "null query arrays");
        process_queries(c, nqueries, query_lens, qbeg, qend);
    });
}

int cbp_select_query(cbp_context* c, size_t k, size_t* nqueries)
{
    return guarded([&] {
        check_ctx(c);
        if (nqueries) *nqueries = c->res.size();
        if (k >= c->res.size()) throw Error(CBP_ERR_ARG, "query index beyond the last call's queries");
        c->cur = k;
    });
}

int cbp_wait_idle(cbp_context* c)
{
    return guarded([&] { check_ctx(c); CBP_CUDA(cudaStreamSynchronize(c->stream)); });
}

int cbp_read_score_matrix(cbp_context* c, float* scores, float* modscores, size_t ld, size_t* ncols,
                          size_t* first_profile)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_Lq) throw Error(CBP_ERR_STATE, "no processed query");
        if (ld < (size_t)c->last_ncols) throw Error(CBP_ERR_ARG, "ld smaller than the slab width");
        if (ncols) *ncols = (size_t)c->last_ncols;
        if (first_profile) *first_profile = (size_t)c->last_first_profile;
        const size_t w = (size_t)c->last_ncols * sizeof(float);
        const size_t r0 = (size_t)(c->last_row0 * c->last_ld);
        if (scores)
            CBP_CUDA(cudaMemcpy2D(scores, ld * sizeof(float), c->scores.as<float>() + r0, c->last_ld * sizeof(float),
                                  w, c->last_Lq, cudaMemcpyDeviceToHost));
        if (modscores)
            CBP_CUDA(cudaMemcpy2D(modscores, ld * sizeof(float), c->modscores.as<float>() + r0,
                                  c->last_ld * sizeof(float), w, c->last_Lq, cudaMemcpyDeviceToHost));
    });
}

int cbp_read_phase1(cbp_context* c, float* score, float* psts, uint32_t* beg, uint32_t* end,
                    int* passed, size_t nmax, size_t* nprof, int* pass_list, size_t* npass)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_Lq) throw Error(CBP_ERR_STATE, "no processed query");
        const size_t n = (size_t)c->last_nprof;
        if (nprof) *nprof = n;
        if (npass) *npass = (size_t)c->last_npass;
        if (nmax < n) throw Error(CBP_ERR_ARG, "output arrays too small");
        std::vector<Dp1Rec> r(n);
        CBP_CUDA(cudaMemcpy(r.data(), c->dprecs.as<Dp1Rec>() + c->last_dp_off, n * sizeof(Dp1Rec),
                            cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; i++) {
            if (score) score[i] = r[i].score;
            if (psts) psts[i] = r[i].psts;
            if (beg) beg[i] = r[i].beg;
            if (end) end[i] = r[i].end;
            if (passed) passed[i] = r[i].passed;
        }
        if (pass_list && c->last_npass > 0)
            CBP_CUDA(cudaMemcpy(pass_list, c->passidx.as<int>() + c->last_dp_off,
                                (size_t)c->last_npass * sizeof(int), cudaMemcpyDeviceToHost));
    });
}

int cbp_read_statistics(cbp_context* c, float* recs, size_t nmax, size_t* npass)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_Lq) throw Error(CBP_ERR_STATE, "no processed query");
        const size_t n = (size_t)c->last_npass;
        if (npass) *npass = n;
        if (!recs || n == 0) return;
        if (nmax < n) throw Error(CBP_ERR_ARG, "output array too small");
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        CBP_CUDA(cudaMemcpy(recs, c->statrecs.p, n * kRecFloats * sizeof(float),
                            cudaMemcpyDeviceToHost));
    });
}

int cbp_read_fits(cbp_context* c, double* fits, size_t nmax, size_t* npass)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_Lq) throw Error(CBP_ERR_STATE, "no processed query");
        if (c->opt.tc_form == CBP_TC_PLAIN) throw Error(CBP_ERR_STATE, "the plain form fits in FP32 only");
        const size_t n = (size_t)c->last_npass;
        if (npass) *npass = n;
        if (!fits || n == 0) return;
        if (nmax < n) throw Error(CBP_ERR_ARG, "output array too small");
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        CBP_CUDA(cudaMemcpy(fits, c->fits.p, n * kFitDoubles * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int cbp_read_btck(cbp_context* c, uint8_t* btck, size_t ld)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_Lq) throw Error(CBP_ERR_STATE, "no processed query");
        if (ld < (size_t)c->last_ncols) throw Error(CBP_ERR_ARG, "ld smaller than the slab width");
        CBP_CUDA(cudaMemcpy2D(btck, ld, c->btck.as<uint8_t>() + c->last_row0 * c->last_ld, c->last_ld,
                              (size_t)c->last_ncols, c->last_Lq,
                              cudaMemcpyDeviceToHost));
    });
}

int cbp_read_map_fb(cbp_context* c, size_t pair, float* fb, size_t ld, size_t* profile_len)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_map_np) throw Error(CBP_ERR_STATE, "no MAP realignment in the last slab");
        if (pair >= (size_t)c->last_map_np) throw Error(CBP_ERR_ARG, "pair index outside the last slab's pass list");
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        int pidx = 0;
        long long dst = 0;
        CBP_CUDA(cudaMemcpy(&pidx, c->last_map_pass_idx + pair, sizeof(int), cudaMemcpyDeviceToHost));
        CBP_CUDA(cudaMemcpy(&dst, c->last_map_pass_dst + pair, sizeof(long long), cudaMemcpyDeviceToHost));
        const int Ld = c->db->h_plen[(size_t)(c->last_map_p0 + pidx)];
        if (profile_len) *profile_len = (size_t)Ld;
        if (!fb) return;
        if (ld < (size_t)Ld) throw Error(CBP_ERR_ARG, "ld smaller than the profile length");
        // the pair's diagonal rows [dst, dst + Ld + 31) of each 32-row band;
        // cell (r, c) at local diagonal row c + r%32, lane r%32
        const int Lq = c->last_map_Lq;
        const size_t rows = (size_t)Ld + 31;
        std::vector<float> band(rows * 32);
        for (int b = 0; b * 32 < Lq; b++) {
            const float* src = c->fb2.as<float>() + ((size_t)b * c->last_map_nd + (size_t)dst) * 32;
            CBP_CUDA(cudaMemcpy(band.data(), src, band.size() * sizeof(float), cudaMemcpyDeviceToHost));
            for (int t = 0; t < 32 && b * 32 + t < Lq; t++)
                for (int col = 0; col < Ld; col++)
                    fb[(size_t)(b * 32 + t) * ld + col] = band[((size_t)col + t) * 32 + t];
        }
    });
}

int cbp_read_slab_columns(cbp_context* c, size_t first_col, size_t ncols, float* scores, float* modscores,
                          uint8_t* btck, size_t ld)
{
    return guarded([&] {
        check_ctx(c);
        if (!c->last_Lq) throw Error(CBP_ERR_STATE, "no processed query");
        if (first_col > (size_t)c->last_ncols || ncols > (size_t)c->last_ncols - first_col)
            throw Error(CBP_ERR_ARG, "column range outside the slab");
        if (ld < ncols) throw Error(CBP_ERR_ARG, "ld smaller than the column count");
        if (ncols == 0) return;
        CBP_CUDA(cudaStreamSynchronize(c->stream));
        const size_t w = ncols * sizeof(float);
        const size_t r0 = (size_t)(c->last_row0 * c->last_ld);
        if (scores)
            CBP_CUDA(cudaMemcpy2D(scores, ld * sizeof(float), (const float*)c->scores.p + r0 + first_col,
                                  c->last_ld * sizeof(float), w, c->last_Lq, cudaMemcpyDeviceToHost));
        if (modscores)
            CBP_CUDA(cudaMemcpy2D(modscores, ld * sizeof(float), (const float*)c->modscores.p + r0 + first_col,
                                  c->last_ld * sizeof(float), w, c->last_Lq, cudaMemcpyDeviceToHost));
        if (btck)
            CBP_CUDA(cudaMemcpy2D(btck, ld, (const uint8_t*)c->btck.p + r0 + first_col, c->last_ld, ncols,
                                  c->last_Lq, cudaMemcpyDeviceToHost));
    });
}

int cbp_get_hit_records(cbp_context* c, float* recs, size_t max_records, size_t* nrecords)
{
    return guarded([&] {
        check_ctx(c);
        const QueryResult& r = cur_result(c);
        const size_t n = r.h_recs.size() / kRecFloats;
        if (nrecords) *nrecords = n;
        if (recs) {
            if (max_records < n) throw Error(CBP_ERR_ARG, "record buffer too small");
            std::memcpy(recs, r.h_recs.data(), r.h_recs.size() * sizeof(float));
        }
    });
}

int cbp_get_hit_list(cbp_context* c, int32_t* order, size_t max_hits, size_t* nhits)
{
    return guarded([&] {
        check_ctx(c);
        // ordered on the device at the end of cbp_process; the first
        // max_hits entries are the top max_hits hits
        const QueryResult& r = cur_result(c);
        const size_t n = r.h_order.size();
        if (nhits) *nhits = n;
        if (order && n) std::memcpy(order, r.h_order.data(), std::min(n, max_hits) * sizeof(int32_t));
    });
}

int cbp_get_alignments(cbp_context* c, char* rows, size_t row_stride, size_t* length)
{
    return guarded([&] {
        check_ctx(c);
        const QueryResult& q = cur_result(c);
        const size_t n = q.h_alns[0].size();
        if (length) *length = n;
        if (rows) {
            if (row_stride < n) throw Error(CBP_ERR_ARG, "row stride smaller than the alignment rows");
            for (int r = 0; r < 5; r++) std::memcpy(rows + (size_t)r * row_stride, q.h_alns[r].data(), n);
        }
    });
}

int cbp_format_hits(cbp_context* c, const cbp_format_options* fo, const char* const* descs, char* buf,
                    size_t cap, size_t* used, size_t* nhits)
{
    int rc = CBP_OK;
    const int grc = guarded([&] {
        check_ctx(c);
        if (!c->have_db) throw Error(CBP_ERR_STATE, "no database chunk transferred");
        const ProfilesStore& db = *c->db;
        const QueryResult& q = cur_result(c);
        const size_t n = q.h_alns[0].size();
        std::vector<char> rows(5 * n);
        for (int r = 0; r < 5; r++)
            if (n) std::memcpy(rows.data() + (size_t)r * n, q.h_alns[r].data(), n);
        const int qss = c->query.h_ss.empty() ? 1 : c->query.h_ss[c->cur];
        rc = format_hits_from(q.h_recs.data(), q.h_recs.size() / kRecFloats, q.h_order.data(),
                              q.h_order.size(), rows.data(), n, n,
                              db.h_plen.data(), db.h_eno.data(), db.h_ss.empty() ? nullptr : db.h_ss.data(),
                              db.h_plen.size(), descs, q.Lq, q.eno, qss, c->opt.ssswgt,
                              q.logE_thld, (float)q.searchspace, fo, buf, cap, used, nhits);
    });
    return grc != CBP_OK ? grc : rc;
}

int cbp_get_search_space(cbp_context* c, uint64_t* search_space, size_t* delta_length)
{
    return guarded([&] {
        check_ctx(c);
        const QueryResult& r = cur_result(c);
        if (search_space) *search_space = r.searchspace;
        if (delta_length) *delta_length = r.delta_length;
    });
}

int cbp_set_karlin_altschul(cbp_context* c, float ungapped_lambda, float ungapped_k,
                            float gapped_lambda, float gapped_k, float gapped_alpha, float gapped_beta)
{
    return guarded([&] {
        check_ctx(c);
        if (!(ungapped_lambda > 0.f && ungapped_k > 0.f && gapped_lambda > 0.f && gapped_k > 0.f))
            throw Error(CBP_ERR_ARG, "lambda and K must be positive");
        c->ref_lambda = ungapped_lambda;
        c->ref_K = ungapped_k;
        c->gap_lambda = gapped_lambda;
        c->gap_K = gapped_k;
        c->gap_alpha = gapped_alpha;
        c->gap_beta = gapped_beta;
    });
}

void cbp_score_threshold(size_t query_len, uint64_t db_len, float evalue, float gapped_lambda,
                         float gapped_k, float* score_threshold, float* log_evalue_threshold)
{
    const size_t sspace = query_len * (size_t)db_len;
    float ev = evalue;
    float sthld = 999.0f, lthld = -99.0f;
    if (ev > 0.0f && sspace > 0 && gapped_lambda > 0.0f && gapped_k > 0.0f) {
        lthld = logf(ev);
        ev = ev < 1.0f ? ev * 10.0f : ev * 3.0f;
        ev /= gapped_k * (float)sspace;
        if (ev > 0.0f) {
            float sc = -logf(ev) / gapped_lambda;
            sthld = sc < 0.0f ? 0.0f : sc;
        }
    }
    if (score_threshold) *score_threshold = sthld;
    if (log_evalue_threshold) *log_evalue_threshold = lthld;
}

int cbp_get_tuning(cbp_context* c, size_t query_len, int* rows, int* window, int* dp_warps, float* ms, int n)
{
    return guarded([&] {
        check_ctx(c);
        const Tuning t = c->tuning.count((int)query_len / 64) ? c->tuning[(int)query_len / 64] : Tuning();
        if (rows) *rows = t.rows;
        if (window) *window = t.window;
        if (dp_warps) *dp_warps = t.dp_warps;
        for (int k = 0; ms && k < n && k < kScoreCandidates + kDpCandidates; k++)
            ms[k] = k < kScoreCandidates ? t.score_ms[k] : t.dp_ms[k - kScoreCandidates];
    });
}

int cbp_set_kernels(cbp_context* c, size_t query_len, int rows, int window, int dp_warps)
{
    return guarded([&] {
        check_ctx(c);
        if (rows != 8 && rows != 16 && rows != 32) throw Error(CBP_ERR_ARG, "rows per block must be 8, 16 or 32");
        if (window < 32 || window > kMaxOrderWindow || window % 32)
            throw Error(CBP_ERR_ARG, "ordering window must be a multiple of 32 in [32, 4096]");
        if (dp_warps != 1 && dp_warps != 2) throw Error(CBP_ERR_ARG, "DP warps per block must be 1 or 2");
        Tuning& t = c->tuning[(int)query_len / 64];
        t = Tuning();
        t.rows = rows;
        t.window = window;
        t.dp_warps = dp_warps;
        t.tuned = true;
    });
}

int cbp_stage_times(cbp_context* c, float* ms, int n)
{
    if (!c || !ms) return 0;
    int k = std::min(n, 6);
    for (int i = 0; i < k; i++) ms[i] = c->stage_ms[i];
    return k;
}

int cbp_stage_launches(cbp_context* c, uint64_t* launches, int n)
{
    if (!c || !launches) return 0;
    int k = std::min(n, 6);
    for (int i = 0; i < k; i++) launches[i] = c->stage_launches[i];
    return k;
}

int cbp_graph_launches(cbp_context* c, uint64_t* graphs)
{
    return guarded([&] {
        check_ctx(c);
        if (graphs) *graphs = c->graph_launches;
    });
}

int cbp_launch_count(cbp_context* c, uint64_t* launches)
{
    return guarded([&] {
        if (!c || !launches) throw Error(CBP_ERR_ARG, "null argument");
        *launches = c->launches;
    });
}

}  // extern "C"
