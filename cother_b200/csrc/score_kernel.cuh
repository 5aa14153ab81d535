// Score-matrix stage interface.
#pragma once

#include <cuda_runtime.h>
#include "layout.h"

namespace cbp {

struct ScoreArgs {
    ProfilesDev q;        // query profile
    ProfilesDev db;       // resident database chunk
    long long col0 = 0;   // first chunk position of the slab
    int ncols = 0;        // slab positions
    long long ld = 0;     // leading dimension of the outputs
    // slot -> slab column (ld entries, -1 = none): the columns of each
    // ordering window sorted by list length, so that the lanes of a warp run
    // DDMS loops of equal trip count; nullptr = identity
    const int* colorder = nullptr;
    int rows = 16;        // query positions per block: 8, 16 or 32
    int Lq = 0;
    float ssswgt = 0.f, ddmswgt = 0.f, initshift = 0.f;
    int dstsegm = 6;
    // context-vector term (CVSWGT > 0): the map's scores for keys
    // (i - cvs_shift)/2, its first and last keys, and the score's constants
    float cvswgt = 0.f;
    const float* cvs_scores = nullptr;
    int cvs_card = 0, cvs_shift = 0;
    float cvs_key_first = 0.f, cvs_key_last = 0.f;
    float cvs_lokappa0 = 0.f, cvs_pownu0 = 0.f, cvs_cterm = 0.f;
    bool cvs_int_priors = false;    // MAPALN=0: log priors truncated to integers
    const float* sstab = nullptr;   // [30][30]
    const float* dmstab = nullptr;  // [22][22]
    float* scores = nullptr;        // [Lq][ld]
    float* modscores = nullptr;     // [Lq][ld]
    // tensor-core form: the profile-profile sums, computed beforehand into
    // `scores` ([Lq][ld]), which the kernel then overwrites with the scores
    bool dots_in_scores = false;
    // set to 2 when a wait for the bulk-copied distance lists gave up (may
    // be null); the block then writes nothing
    int* err = nullptr;
};

// columns per ordering window of launch_column_order: default and largest
constexpr int kOrderWindow = 1024;
constexpr int kMaxOrderWindow = 4096;

void launch_score_matrix(const ScoreArgs& a, cudaStream_t stream);
// Fill order[0..ld) for the slab columns [col0, col0+ncols): within each
// window of `window` slots (a multiple of 32, at most kMaxOrderWindow), the
// window's columns by descending distance list length; slots past ncols
// get -1.
void launch_column_order(const uint8_t* dstlen, long long col0, int ncols, long long ld, int window, int* order,
                         cudaStream_t stream);
void build_dms_table(float* T);

}  // namespace cbp
