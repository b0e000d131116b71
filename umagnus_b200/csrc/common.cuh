// common.cuh -- library context, error reporting and launch helpers.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "../../include/umagnus_b200.h"

namespace umag {

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

struct Context {
    int device = -1;
    bool initialised = false;
    cudaStream_t own_stream = nullptr;  // created by umag_init
    cudaStream_t stream = nullptr;      // stream all calls are queued on
    // reduction scratch: per-block partials + pinned host result
    void* red_dev = nullptr;            // device scratch for reductions
    size_t red_bytes = 0;
    double* red_host = nullptr;         // pinned, 8 doubles
    int sm_count = kNumSMs;
};

Context& ctx();
int set_error(int code, const char* fmt, ...);
int ensure_init();

#define UMAG_CUDA(call)                                                                   \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::umag::set_error(UMAG_E_CUDA, "%s: %s (%s:%d)", #call,                \
                                     cudaGetErrorString(e_), __FILE__, __LINE__);         \
    } while (0)

#define UMAG_LAUNCH_CHECK() UMAG_CUDA(cudaGetLastError())

#define UMAG_TRY(expr)            \
    do {                          \
        int s_ = (expr);          \
        if (s_ != UMAG_OK) return s_; \
    } while (0)

#define UMAG_REQUIRE(cond, ...)                                          \
    do {                                                                 \
        if (!(cond)) return ::umag::set_error(UMAG_E_ARG, __VA_ARGS__); \
    } while (0)

// Grid for a grid-stride loop over n elements: enough CTAs to fill the 148
// SMs several times over, never more than needed.
inline int grid_for(long long n, int block, int waves = 8) {
    long long need = (n + block - 1) / block;
    long long cap = (long long)ctx().sm_count * waves;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

}  // namespace umag
