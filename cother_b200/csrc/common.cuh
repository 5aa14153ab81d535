// Error handling and small helpers shared by the host driver and kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdexcept>
#include <string>

namespace cbp {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CBP_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t _e = (call);                                                    \
        if (_e != cudaSuccess)                                                      \
            throw ::cbp::Error(2, std::string(#call) + ": " + cudaGetErrorString(_e) + \
                                      " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
    } while (0)

#define CBP_CHECK_LAUNCH() CBP_CUDA(cudaGetLastError())

inline long long ceil_div(long long a, long long b) { return (a + b - 1) / b; }
inline long long align_up(long long a, long long b) { return ceil_div(a, b) * b; }

}  // namespace cbp
