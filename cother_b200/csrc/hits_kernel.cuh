// On-device ordering of the reported hits.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cbp {

// Keys of records base .. base+n-1 (`recs` holds the n records): the log
// E-value's order in the high word and the record index in the low word for
// a reported record (log E at most `logethld`, realigned), all ones
// otherwise; *nreported is increased by the reported count. Returns the
// launches made.
int launch_hit_keys(const float* recs, int n, float logethld, long long base, uint64_t* keys, int* nreported,
                    cudaStream_t stream);

// Keys the sort of n keys needs room for (a power of two, at least 4096).
long long hit_sort_capacity(long long n);

// Sort keys[0..n) ascending in place (keys needs hit_sort_capacity(n)
// entries; the tail is overwritten). Returns the launches made.
int launch_hit_sort(uint64_t* keys, long long n, cudaStream_t stream);

}  // namespace cbp
