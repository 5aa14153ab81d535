// Phase-1 DP entry point that allocates no device memory.
//
// Some callers cannot allocate device memory at the time they run the
// search: a serving process whose device memory is handed out by its own
// pool allocator, or code enqueuing work where a cudaMalloc would
// synchronise the device or is not permitted. For them cbp_dp1_noalloc runs
// the phase-1 DP on buffers the caller already owns. Inputs and outputs come
// from the caller; the only scratch the DP needs -- the per-profile strip
// that carries the bottom row of one 32-row band to the next, 5 floats per
// slab column -- lives in the fixed-size device array below instead of a
// cudaMalloc'd buffer.
#include <cuda_runtime.h>

#include <string>

#include "cother_b200.h"
#include "common.cuh"
#include "dp1_kernel.cuh"

namespace cbp {
// defined in api.cu: records the message returned by cbp_last_error()
void set_last_error(const std::string& msg);
}

namespace {

// Largest slab width (score-matrix columns) the allocation-free DP accepts:
// the strip holds 5 states x this many columns, 1.25 MiB of device memory
// that every GPU which loads the library keeps until the process exits.
constexpr long long kNoAllocMaxColumns = CBP_NOALLOC_MAX_COLUMNS;

static __device__ __align__(256) float g_dp1_strip[5 * kNoAllocMaxColumns];

// Device address of g_dp1_strip on the current device. In host code the
// array's name only stands in for it. The address is looked up on every
// call, with the caller's device current, rather than cached: a device reset
// or a re-created primary context reloads the module at another address.
// The first lookup on a device loads the module there, which is why the
// first call should come before any stream capture; later lookups are cheap.
float* strip_address()
{
    float* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_dp1_strip);
    if (e != cudaSuccess)
        throw cbp::Error(CBP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    return ptr;
}

}  // namespace

extern "C" int cbp_dp1_noalloc(const float* scores, size_t ld, int query_len, const float* query_trn,
                               long long db_npos, int db_nprof, const float* db_trn,
                               const int* prof_len, const long long* prof_start,
                               int first_profile, int nprof, long long first_column,
                               uint8_t* btck, float* max_scores, uint32_t* max_coords,
                               void* stream)
{
    try {
        if (!scores || !query_trn || !db_trn || !prof_len || !prof_start || !btck || !max_scores ||
            !max_coords)
            throw cbp::Error(CBP_ERR_ARG, "cbp_dp1_noalloc: null pointer argument");
        if (ld == 0 || query_len <= 0 || nprof <= 0 || db_npos <= 0 || db_nprof <= 0 || first_profile < 0 ||
            first_profile + nprof > db_nprof || first_column < 0)
            throw cbp::Error(CBP_ERR_ARG, "cbp_dp1_noalloc: invalid sizes");
        if ((long long)ld > kNoAllocMaxColumns)
            throw cbp::Error(CBP_ERR_LIMIT, "cbp_dp1_noalloc: slab width " + std::to_string(ld) +
                                                " exceeds the fixed scratch of " +
                                                std::to_string(kNoAllocMaxColumns) + " columns");
        if (query_len >= 65536)
            throw cbp::Error(CBP_ERR_LIMIT, "cbp_dp1_noalloc: query length must be < 65536");
        cbp::Dp1Args a;
        a.scores = scores;
        a.ld = (long long)ld;
        a.Lq = query_len;
        a.qtrn = query_trn;
        a.db.N = db_npos;
        a.db.P = db_nprof;
        a.db.trn = db_trn;
        a.db.plen = prof_len;
        a.db.pstart = prof_start;
        a.col0 = first_column;
        a.p0 = first_profile;
        a.nprof = nprof;
        a.btck = btck;
        a.bandbuf = strip_address();
        a.maxsc = max_scores;
        a.maxcoords = max_coords;
        cbp::dp1_set_attributes();
        cbp::launch_dp1(a, static_cast<cudaStream_t>(stream));
        cbp::set_last_error("");
        return CBP_OK;
    } catch (const cbp::Error& e) {
        cbp::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        cbp::set_last_error(e.what());
        return CBP_ERR_ARG;
    }
}
