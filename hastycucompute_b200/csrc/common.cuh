// Shared helpers of libhasty_b200: status handling, complex arithmetic, launch sizing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "hasty_b200.h"

namespace hb {

// Per-thread error message behind hb_last_error().
void set_error(const std::string& msg);
const char* get_error();

// Return-early helpers for functions returning an HB_* status.
#define HB_TRY(expr)                     \
    do {                                 \
        int hb_status_ = (expr);         \
        if (hb_status_ != HB_OK) return hb_status_; \
    } while (0)

#define HB_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t hb_e_ = (call);                                                     \
        if (hb_e_ != cudaSuccess) {                                                     \
            hb::set_error(std::string(#call) + " failed: " + cudaGetErrorString(hb_e_)); \
            return HB_ERR_CUDA;                                                         \
        }                                                                               \
    } while (0)

#define HB_REQUIRE(cond, code, msg)  \
    do {                             \
        if (!(cond)) {               \
            hb::set_error(msg);      \
            return (code);           \
        }                            \
    } while (0)

// Checks the launch just issued on the current thread.
inline int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string(what) + " launch failed: " + cudaGetErrorString(e));
        return HB_ERR_CUDA;
    }
    return HB_OK;
}

// ---- complex64 as float2 ------------------------------------------------------------------
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// The reference's ToeplitzMultType applied to a (fft/kernels/toeplitz_load_3D.cu:2-15):
// 1 -> a*b, 2 -> a*conj(b), anything else -> a.
__device__ __forceinline__ float2 mult_typed(float2 a, float2 b, int type) {
    if (type == HB_MULT_MULT) return cmul(a, b);
    if (type == HB_MULT_MULT_CONJ) return cmulc(a, b);
    return a;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

constexpr int kNumSMs = 148;  // B200

}  // namespace hb
