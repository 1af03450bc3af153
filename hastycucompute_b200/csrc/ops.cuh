// Pass operators shared by the NUFFT and Toeplitz paths (see fft.cuh for the Op contract).
#pragma once

#include "fft2.cuh"

namespace hb {

#ifdef __CUDACC__

// Plain strided transform: element (a, l, e) at base + a*s_a + l*s_l + e on both sides.
struct OpStrided {
    static constexpr bool kLoadLFast = false;
    static constexpr bool kStoreLFast = false;
    static constexpr bool kFusedK = false;
    static constexpr bool kChunkLoop = false;
    static constexpr bool kSenseReduce = false;
    const float2* src;
    float2* dst;
    int64_t s_a, s_l;
    int64_t d_a, d_l;
    float scale;
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const {
        return src[a * s_a + (int64_t)l * s_l + e];
    }
    __device__ __forceinline__ int64_t kcol(int64_t) const { return 0; }
    __device__ __forceinline__ const float2* kptr(int64_t) const { return nullptr; }
    __device__ __forceinline__ const float2* srow(int64_t, int64_t) const { return nullptr; }
    __device__ __forceinline__ float2 product_s(float2 v, float2) const { return v; }
    __device__ __forceinline__ int64_t group(int64_t) const { return 0; }
    __device__ __forceinline__ int ngroups() const { return 1; }
    __device__ __forceinline__ float2 kval(int64_t, int, int64_t) const { return make_float2(0.f, 0.f); }
    __device__ __forceinline__ void store(int64_t a, int o, int64_t e, float2 v) const {
        dst[a * d_a + (int64_t)o * d_l + e] = cscale(v, scale);
    }
    __device__ __forceinline__ float2 product(int64_t, int, int64_t, float2 v) const { return v; }
    __device__ __forceinline__ void write_row(int64_t, int, int, float2) const {}
    __device__ __forceinline__ void store_phase(const float2* res, const PassCfg& c, int64_t a0, int64_t e0, int, int,
                                                float2*) const {
        const float sc = scale;
        float2* d = dst;
        const int64_t da = d_a, dl = d_l;
        for_each_output<false>(res, c, a0, e0, [&](int64_t a, int o, int64_t e, float2 v) {
            d[a * da + (int64_t)o * dl + e] = cscale(v, sc);
        });
    }
    __device__ __forceinline__ void finish(const PassCfg&, int64_t, float2*) const {}
};

#endif

}  // namespace hb
