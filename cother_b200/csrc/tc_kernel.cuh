// Tensor-core form of the profile-profile term: interface.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include "layout.h"

namespace cbp {

struct TcArgs {
    ProfilesDev q;        // query profile
    ProfilesDev db;       // resident database chunk
    long long col0 = 0;   // first chunk position of the slab
    int ncols = 0;        // slab positions
    long long ld = 0;     // leading dimension of the score matrix
    int Lq = 0;           // rows of this query
    int qrow0 = 0;        // its first position in the (stacked) query profile set
    int qprof = 0;        // its profile index there (for its background)
};

// bytes of the query operand image for a query of Lq positions
size_t tc_query_image_bytes(int form, long long Lq);

// Per device, before the first tc_profile_sums (and outside any stream
// capture): the shared-memory opt-in of the tensor-core kernel.
void tc_set_attributes();

// The profile-profile sums of the slab into out ([Lq][ld]) on `stream`:
// the query operand image (qimg, tc_query_image_bytes) and the tcgen05
// contraction; *err is set to 1 when a wait gave up. Returns the launches.
int tc_profile_sums(const TcArgs& a, int form, void* qimg, float* out, int* err, cudaStream_t stream);

}  // namespace cbp
