// Toeplitz-embedded normal operator on B200: kernel construction, kernel re-layout, the fused
// 2x-padded convolution with the reference's multiply flags, and the SENSE normal operator.
//
// The convolution never materialises a (2N)^d grid per batch. With B batches interleaved in
// one buffer ([..][B], B fastest), a 3-D apply is five pruned passes:
//   P1 axis 2: load in[b] * mults (N2 samples) -> FFT 2N2            -> W1[N0][N1][2N2][B]
//   P2 axis 1: N1 samples -> FFT 2N1                                 -> W2[N0][2N1][2N2][B]
//   P3 axis 0: N0 samples -> FFT 2N0, * K, IFFT 2N0, keep [0, N0)      -> W2 (in place)
//   P4 axis 1: IFFT 2N1, keep [0, N1)                                -> W1[N0][N1][2N2][B]
//   P5 axis 2: IFFT 2N2, keep [0, N2), * output mults (and for SENSE: sum over b of
//              conj(S_b) * v inside the CTA)                          -> out
// A 2-D apply is P1, the fused pass along axis 1, and P5. The straight convolution keeps
// [N-1, 2N-1) of each axis; the transformed kernel carries that shift as a phase ramp, so every
// pass pads and crops at offset 0 and runs the compile-time pass shapes of pass2_kernel.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include <cuda.h>

#include "nufft.cuh"
#include "ops.cuh"

namespace hb {

struct ToepGeom {
    int dim;
    int64_t N[3];  // internal 3-D (N0 == 1 in 2-D)
    int L[3];      // 2N on non-unit axes, 1 on unit axes
    int64_t n;     // N0*N1*N2
    int64_t B;
};

static int toep_geom(ToepGeom* t, int dim, const int64_t* shape, int64_t B) {
    HB_REQUIRE(dim == 2 || dim == 3, HB_ERR_INVALID_ARG, "Toeplitz operator supports dim 2 and 3");
    HB_REQUIRE(shape != nullptr, HB_ERR_INVALID_ARG, "shape is null");
    HB_REQUIRE(B >= 1, HB_ERR_INVALID_ARG, "batch count must be >= 1");
    t->dim = dim;
    t->B = B;
    t->n = 1;
    for (int ax = 0; ax < 3; ++ax) {
        t->N[ax] = 1;
        t->L[ax] = 1;
    }
    for (int i = 0; i < dim; ++i) {
        const int64_t v = shape[i];
        HB_REQUIRE(v > 1 && v <= (1 << 15), HB_ERR_INVALID_ARG, "image dimensions must be in (1, 32768]");
        t->N[3 - dim + i] = v;
        t->L[3 - dim + i] = (int)(2 * v);
        t->n *= v;
    }
    for (int ax = 3 - dim; ax < 3; ++ax) {
        int r = t->L[ax];
        for (int p : {2, 3, 5, 7, 11, 13})
            while (r % p == 0) r /= p;
        HB_REQUIRE(r == 1, HB_ERR_INVALID_ARG, "2N must have no prime factor above 13 on any axis");
    }
    return HB_OK;
}

static size_t toep_ws_elems(const ToepGeom& t) {
    size_t w1 = (size_t)t.N[0] * t.N[1] * t.L[2] * t.B;
    size_t w2 = t.dim == 3 ? (size_t)t.N[0] * t.L[1] * t.L[2] * t.B : 0;
    return w1 + w2;
}

// Per-thread cache of FFT length plans (twiddle tables) keyed by length and device. The first
// use of a length uploads its table with synchronous copies, so it must happen outside a stream
// capture; later uses only read the cache.
struct LenCache {
    int dev;
    FftLen f;
};
static thread_local std::vector<LenCache> g_len_cache;

static int get_len(int L, FftLen* out) {
    int dev = 0;
    HB_CUDA(cudaGetDevice(&dev));
    for (const auto& c : g_len_cache)
        if (c.dev == dev && c.f.L == L) {
            *out = c.f;
            return HB_OK;
        }
    LenCache c;
    c.dev = dev;
    HB_TRY(fftlen_make(&c.f, L));
    g_len_cache.push_back(c);
    *out = c.f;
    return HB_OK;
}

// ---- ops -------------------------------------------------------------------------------------
#ifdef __CUDACC__

struct OpToepIn {
    static constexpr int kHalfIO = 1;  // pass shape (pass2_kernel HM)
    static constexpr bool kLoadLFast = true;
    static constexpr bool kStoreLFast = false;
    static constexpr bool kFusedK = false;
    static constexpr bool kChunkLoop = false;
    static constexpr bool kSenseReduce = false;
    const float2* in;
    const float2* m1;
    const float2* m2;
    int in_m1, in_m2;
    float2* dst;
    int64_t N2, n, d_a, d_l;
    // frames: column e = f * cpf + c reads in[c] and m1[f] (cpf = 0: in[e], shared m1)
    int64_t cpf;
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const {
        const int64_t idx = a * N2 + l;
        const int64_t ei = cpf ? e % cpf : e;
        const int64_t m1o = cpf ? (e / cpf) * n : 0;
        float2 v = in[ei * n + idx];
        if (m1) v = mult_typed(v, m1[m1o + idx], in_m1);
        if (m2) v = mult_typed(v, m2[idx], in_m2);
        return v;
    }
    __device__ __forceinline__ int64_t kcol(int64_t) const { return 0; }
    __device__ __forceinline__ const float2* kptr(int64_t) const { return nullptr; }
    __device__ __forceinline__ const float2* srow(int64_t, int64_t) const { return nullptr; }
    __device__ __forceinline__ float2 product_s(float2 v, float2) const { return v; }
    __device__ __forceinline__ int64_t group(int64_t) const { return 0; }
    __device__ __forceinline__ int ngroups() const { return 1; }
    __device__ __forceinline__ float2 kval(int64_t, int, int64_t) const { return make_float2(0.f, 0.f); }
    __device__ __forceinline__ void store(int64_t a, int o, int64_t e, float2 v) const { dst[a * d_a + (int64_t)o * d_l + e] = v; }
    __device__ __forceinline__ float2 product(int64_t, int, int64_t, float2 v) const { return v; }
    __device__ __forceinline__ void write_row(int64_t, int, int, float2) const {}
    __device__ __forceinline__ void store_phase(const float2* res, const PassCfg& c, int64_t a0, int64_t e0, int, int,
                                                float2*) const {
        float2* d = dst;
        const int64_t da = d_a, dl = d_l;
        for_each_output<false>(res, c, a0, e0, [&](int64_t a, int o, int64_t e, float2 v) { d[a * da + (int64_t)o * dl + e] = v; });
    }
    __device__ __forceinline__ void finish(const PassCfg&, int64_t, float2*) const {}
};

// P1 of the SENSE normal operator: column e = f * cpf + c reads S_c[idx] * x_f[idx] (cpf = 0: one
// frame, x shared by all coils), times the diagonal m2[idx] when kDiag. The product is fixed at
// compile time.
template <bool kDiag>
struct OpToepInSenseT : OpToepIn {
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const {
        return cmul(load_col(a, l, e), row_at(a, l, e));
    }
    // the image factor x is the same for every coil column of a row within one frame: when a
    // CTA's columns e0 .. e0+eb-1 lie in one frame the pass stages that row once per CTA
    static constexpr bool kStageRow = true;
    __device__ __forceinline__ bool row_shared(int64_t e0, int eb) const {
        return cpf == 0 || e0 / cpf == (e0 + eb - 1) / cpf;
    }
    __device__ __forceinline__ const float2* row(int64_t a, int64_t e0) const {
        return m1 + (cpf ? (e0 / cpf) * n : 0) + a * N2;
    }
    __device__ __forceinline__ float2 row_at(int64_t a, int l, int64_t e) const {
        return m1[(cpf ? (e / cpf) * n : 0) + a * N2 + l];
    }
    __device__ __forceinline__ float2 load_col(int64_t a, int l, int64_t e) const {
        const int64_t idx = a * N2 + l;
        float2 v = in[(cpf ? e % cpf : e) * n + idx];
        if constexpr (kDiag) v = cmul(v, m2[idx]);
        return v;
    }
};
using OpToepInSense = OpToepInSenseT<false>;

// The Toeplitz passes along the middle axis: zero-padding N -> 2N (forward) and cropping
// 2N -> N (inverse), both at offset 0.
// (Prefetching measured slower for both at 160^3 x 32 coils: P2 1.48 vs 1.26 ms, P4 1.36 vs 1.16 ms,
// two or three CTAs per SM against four.)
struct OpStridedPad : OpStrided {
    static constexpr int kHalfIO = 1;
};
struct OpStridedCrop : OpStrided {
    static constexpr int kHalfIO = 2;
};

// In-place fused pass: FFT, * Kt[col][pos], IFFT, crop. buf[l][e] with row stride E.
struct OpToepMid {
    static constexpr int kHalfIO = 3;  // pass shape (pass2_kernel HM)
    static constexpr bool kPrefetch = true;  // persistent CTAs, next block's samples by cp.async
    static constexpr bool kLoadLFast = false;
    static constexpr bool kStoreLFast = false;
    static constexpr bool kFusedK = true;
    static constexpr bool kChunkLoop = false;
    static constexpr bool kSenseReduce = false;
    float2* buf;
    const float2* kt;
    int64_t E, B;
    int Lk;
    __device__ __forceinline__ float2 load(int64_t, int l, int64_t e) const { return buf[(int64_t)l * E + e]; }
    __device__ __forceinline__ const float2* sample_ptr(int64_t, int l, int64_t e) const { return buf + (int64_t)l * E + e; }
    // kernel column of column e: a 32-bit division whenever the operands fit (every workspace
    // this library sizes), the 64-bit one otherwise
    __device__ __forceinline__ int64_t kcol(int64_t e) const {
        return ((uint64_t)e | (uint64_t)B) <= 0xffffffffull ? (int64_t)((uint32_t)e / (uint32_t)B) : e / B;
    }
    __device__ __forceinline__ const float2* kptr(int64_t kc) const { return kt + kc * Lk; }
    __device__ __forceinline__ const float2* srow(int64_t, int64_t) const { return nullptr; }
    __device__ __forceinline__ float2 product_s(float2 v, float2) const { return v; }
    __device__ __forceinline__ int64_t group(int64_t) const { return 0; }
    __device__ __forceinline__ int ngroups() const { return 1; }
    __device__ __forceinline__ float2 kval(int64_t, int pos, int64_t e) const { return kt[kcol(e) * Lk + pos]; }
    __device__ __forceinline__ void store(int64_t, int o, int64_t e, float2 v) const { buf[(int64_t)o * E + e] = v; }
    __device__ __forceinline__ float2 product(int64_t, int, int64_t, float2 v) const { return v; }
    __device__ __forceinline__ void write_row(int64_t, int, int, float2) const {}
    __device__ __forceinline__ void store_phase(const float2* res, const PassCfg& c, int64_t a0, int64_t e0, int, int,
                                                float2*) const {
        float2* d = buf;
        const int64_t EE = E;
        for_each_output<false>(res, c, a0, e0, [&](int64_t, int o, int64_t e, float2 v) { d[(int64_t)o * EE + e] = v; });
    }
    __device__ __forceinline__ void finish(const PassCfg&, int64_t, float2*) const {}
};

struct OpToepOutFlat {
    static constexpr int kHalfIO = 2;  // pass shape (pass2_kernel HM)
    static constexpr bool kLoadLFast = false;
    static constexpr bool kStoreLFast = true;
    static constexpr bool kFusedK = false;
    static constexpr bool kChunkLoop = false;
    static constexpr bool kSenseReduce = false;
    const float2* src;  // [rows][L2][B]
    int64_t s_a, s_l;
    const float2* in;
    const float2* m1;
    const float2* m2;
    int io_mult, out_m1, out_m2, accumulate;
    float2* out;
    int64_t N2, n;
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const { return src[a * s_a + (int64_t)l * s_l + e]; }
    __device__ __forceinline__ int64_t kcol(int64_t) const { return 0; }
    __device__ __forceinline__ const float2* kptr(int64_t) const { return nullptr; }
    __device__ __forceinline__ const float2* srow(int64_t, int64_t) const { return nullptr; }
    __device__ __forceinline__ float2 product_s(float2 v, float2) const { return v; }
    __device__ __forceinline__ int64_t group(int64_t) const { return 0; }
    __device__ __forceinline__ int ngroups() const { return 1; }
    __device__ __forceinline__ float2 kval(int64_t, int, int64_t) const { return make_float2(0.f, 0.f); }
    __device__ __forceinline__ void store(int64_t a, int o, int64_t e, float2 v) const {
        const int64_t idx = a * N2 + o;
        if (m1) v = mult_typed(v, m1[idx], out_m1);
        if (m2) v = mult_typed(v, m2[idx], out_m2);
        if (io_mult) v = mult_typed(v, in[e * n + idx], io_mult);
        float2* dst = out + e * n + idx;
        if (accumulate) v = cadd(v, *dst);
        *dst = v;
    }
    __device__ __forceinline__ float2 product(int64_t, int, int64_t, float2 v) const { return v; }
    __device__ __forceinline__ void write_row(int64_t, int, int, float2) const {}
    __device__ __forceinline__ void store_phase(const float2* res, const PassCfg& c, int64_t a0, int64_t e0, int, int,
                                                float2*) const {
        for_each_output<true>(res, c, a0, e0, [&](int64_t a, int o, int64_t e, float2 v) { store(a, o, e, v); });
    }
    __device__ __forceinline__ void finish(const PassCfg&, int64_t, float2*) const {}
};

// Last pass of the SENSE normal operator: out[f][a][o] = sum_c conj(S_c[a][o]) * v_{f,c}[a][o],
// columns e = f * cpf + c (one frame when cpf = B). The CTA walks every batch chunk of its rows and
// keeps one running sum per (row, frame) in shared memory (extra).
struct OpToepOutSense {
    static constexpr int kHalfIO = 2;  // pass shape (pass2_kernel HM)
    static constexpr bool kPrefetch = true;  // persistent rows, next chunk's samples by cp.async
    static constexpr bool kLoadLFast = false;
    static constexpr bool kStoreLFast = false;
    static constexpr bool kFusedK = false;
    static constexpr bool kChunkLoop = true;
    static constexpr bool kSenseReduce = true;
    const float2* src;
    int64_t s_a, s_l;
    const float2* smaps;
    float2* out;
    int64_t N2, n;
    int64_t cpf;  // coils per frame
    int nfr;      // frames
    const float2* odiag;  // optional: the coil sum is multiplied by conj(odiag[idx])
    int accumulate;       // add into out instead of overwriting it
    __device__ __forceinline__ void emit(int64_t oi, int64_t ii, float2 v) const {
        if (odiag) v = cmulc(v, odiag[ii]);
        if (accumulate) v = cadd(v, out[oi]);
        out[oi] = v;
    }
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const { return src[a * s_a + (int64_t)l * s_l + e]; }
    __device__ __forceinline__ const float2* sample_ptr(int64_t a, int l, int64_t e) const { return src + a * s_a + (int64_t)l * s_l + e; }
    __device__ __forceinline__ int64_t kcol(int64_t) const { return 0; }
    __device__ __forceinline__ const float2* kptr(int64_t) const { return nullptr; }
    __device__ __forceinline__ const float2* srow(int64_t a, int64_t e) const { return smaps + (e % cpf) * n + a * N2; }
    __device__ __forceinline__ float2 product_s(float2 v, float2 sv) const { return cmulc(v, sv); }
    __device__ __forceinline__ int64_t group(int64_t e) const { return e / cpf; }
    __device__ __forceinline__ int ngroups() const { return nfr; }
    __device__ __forceinline__ float2 kval(int64_t, int, int64_t) const { return make_float2(0.f, 0.f); }
    __device__ __forceinline__ void store(int64_t, int, int64_t, float2) const {}
    __device__ __forceinline__ float2 product(int64_t a, int o, int64_t e, float2 v) const {
        return cmulc(v, smaps[(e % cpf) * n + a * N2 + o]);
    }
    __device__ __forceinline__ void write_row(int64_t a, int o, int g, float2 v) const {
        emit(g * n + a * N2 + o, a * N2 + o, v);
    }
    // generic-kernel path: acc is [A_blk][nfr][Lout], zeroed on the first chunk
    __device__ __forceinline__ void store_phase(const float2* res, const PassCfg& c, int64_t a0, int64_t e0, int Ab, int Eb,
                                                float2* acc) const {
        const int ng = nfr;
        if (e0 == 0) {
            for (int i = threadIdx.x; i < Ab * ng * c.Lout; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
            __syncthreads();
        }
        const int tot = Ab * c.Lout;
        for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
            const int o = idx % c.Lout, al = idx / c.Lout;
            const int64_t a = a0 + al;
            if (a >= c.A) continue;
            int pos = (o + c.out_shift) % c.L;
            if (pos < 0) pos += c.L;
            const int64_t idx_img = a * N2 + o;
            float2 run = make_float2(0.f, 0.f);
            int64_t gcur = group(e0);
            for (int el = 0; el < Eb; ++el) {
                const int64_t e = e0 + el;
                if (e >= c.E) break;
                const int64_t gg = group(e);
                if (gg != gcur) {
                    float2* dst = acc + ((int64_t)al * ng + gcur) * c.Lout + o;
                    *dst = cadd(*dst, run);
                    run = make_float2(0.f, 0.f);
                    gcur = gg;
                }
                const float2 v = res[pos * c.Wp + al * Eb + el];
                run = cadd(run, cmulc(v, smaps[(e % cpf) * n + idx_img]));
            }
            float2* dst = acc + ((int64_t)al * ng + gcur) * c.Lout + o;
            *dst = cadd(*dst, run);
        }
    }
    __device__ __forceinline__ void finish(const PassCfg& c, int64_t a0, float2* acc) const {
        const int ng = nfr;
        const int tot = c.A_blk * ng * c.Lout;
        for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
            const int o = idx % c.Lout, rest = idx / c.Lout, gg = rest % ng, al = rest / ng;
            const int64_t a = a0 + al;
            if (a >= c.A) continue;
            emit(gg * n + a * N2 + o, a * N2 + o, acc[idx]);
        }
    }
};

// The crop of the straight convolution keeps positions [N-1, 2N-1) of each axis. A circular shift
// of the inverse transform's output by s = N - 1 is a phase ramp on its input,
//     y[i + s] = sum_k (K[k] exp(+2 pi i k s / L)) X[k] exp(+2 pi i k i / L),
// so the transformed kernel carries the ramp of every axis and all passes crop at offset 0.
// (kr, kc) index the kernel as [R][Cc] with Cc = Lb * Lc (3-D) or Lb (2-D, Lc = 1).
__device__ __forceinline__ float2 crop_ramp(float2 v, int64_t kr, int64_t kc, int64_t R, int64_t Lb, int64_t Lc) {
    const int64_t kb = kc / Lc, kk = kc % Lc;
    double ph = 2.0 * ((double)((kr * (R / 2 - 1)) % R) / (double)R + (double)((kb * (Lb / 2 - 1)) % Lb) / (double)Lb);
    if (Lc > 1) ph += 2.0 * (double)((kk * (Lc / 2 - 1)) % Lc) / (double)Lc;
    ph -= 2.0 * floor(ph * 0.5);  // radians / pi in [0, 2)
    double sn, cs;
    sincospi(ph, &sn, &cs);
    return make_float2((float)((double)v.x * cs - (double)v.y * sn), (float)((double)v.x * sn + (double)v.y * cs));
}

// Kt[c * R + z] = K[z][c] * scale * ramp : transpose [R][Cc] -> [Cc][R]
__global__ void k_transpose_scale(const float2* __restrict__ in, float2* __restrict__ out, int64_t R, int64_t Cc,
                                  int64_t Lb, int64_t Lc, float scale) {
    __shared__ float2 tile[32][33];
    const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t r = r0 + j, c = c0 + threadIdx.x;
        if (r < R && c < Cc) tile[j][threadIdx.x] = in[r * Cc + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t c = c0 + j, r = r0 + threadIdx.x;
        if (r < R && c < Cc) out[c * R + r] = crop_ramp(cscale(tile[threadIdx.x][j], scale), r, c, R, Lb, Lc);
    }
}

#endif

// ---- the convolution --------------------------------------------------------------------------
struct ToepArgs {
    const float2* in;
    float2* out;
    const float2* kt;
    const float2* m1;
    const float2* m2;
    int io_mult, in_m1, out_m1, in_m2, out_m2, accumulate;
    bool sense;
    int64_t frames = 1;  // SENSE over frames: t.B = frames * coils, kernels per frame
    const float2* smaps_out = nullptr;  // SENSE: coil maps of the reduction (default: the input maps)
    const float2* odiag = nullptr;      // SENSE: conj(odiag) multiplies the coil sum
};

static int toep_run(const ToepGeom& t, const ToepArgs& a, float2* ws, cudaStream_t s) {
    const int64_t B = t.B;
    const int64_t N0 = t.N[0], N1 = t.N[1], N2 = t.N[2];
    const int L0 = t.L[0], L1 = t.L[1], L2 = t.L[2];
    float2* W1 = ws;                                   // [N0][N1][L2][B]
    float2* W2 = ws + (size_t)N0 * N1 * L2 * B;        // [N0][L1][L2][B] (3-D only)
    FftLen f0, f1, f2;
    HB_TRY(get_len(L2, &f2));
    HB_TRY(get_len(L1, &f1));
    if (t.dim == 3) HB_TRY(get_len(L0, &f0));

    const int64_t cpf = a.sense ? B / a.frames : 0;  // coils per frame (SENSE)
    // P1: axis 2, pad N2 -> L2, forward
    {
        if (a.sense && a.m2) {
            OpToepInSenseT<true> op{{a.in, a.m1, a.m2, HB_MULT_MULT, HB_MULT_MULT, W1, N2, t.n, (int64_t)L2 * B, B,
                                     a.frames > 1 ? cpf : 0}};
            HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, (int)N2, 0, L2, 0, 0, 0, s, "toeplitz P1"));
        } else if (a.sense) {
            OpToepInSense op{{a.in, a.m1, nullptr, HB_MULT_MULT, HB_MULT_NONE, W1, N2, t.n, (int64_t)L2 * B, B,
                              a.frames > 1 ? cpf : 0}};
            HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, (int)N2, 0, L2, 0, 0, 0, s, "toeplitz P1"));
        } else {
            OpToepIn op{a.in, a.m1, a.m2, a.in_m1, a.in_m2, W1, N2, t.n, (int64_t)L2 * B, B, a.frames > 1 ? cpf : 0};
            HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, (int)N2, 0, L2, 0, 0, 0, s, "toeplitz P1"));
        }
    }
    const int64_t E2 = (int64_t)L2 * B;
    if (t.dim == 3) {
        // P2: axis 1, pad N1 -> L1, forward
        {
            OpStridedPad op{{W1, W2, N1 * E2, E2, (int64_t)L1 * E2, E2, 1.0f}};
            HB_TRY(launch_fft_pass(op, f1, N0, E2, (int)N1, 0, L1, 0, 0, 0, s, "toeplitz P2"));
        }
        // P3: axis 0 fused, in place on W2
        {
            const int64_t E = (int64_t)L1 * E2;
            OpToepMid op{W2, a.kt, E, a.frames > 1 ? cpf : B, L0};
            HB_TRY(launch_fft_pass(op, f0, 1, E, (int)N0, 0, (int)N0, 0, 0, 0, s, "toeplitz P3"));
        }
        // P4: axis 1 inverse, crop -> W1
        {
            OpStridedCrop op{{W2, W1, (int64_t)L1 * E2, E2, N1 * E2, E2, 1.0f}};
            HB_TRY(launch_fft_pass(op, f1, N0, E2, L1, 0, (int)N1, 0, 1, 0, s, "toeplitz P4"));
        }
    } else {
        // fused pass along axis 1, in place on W1 ([1][N1][L2][B])
        OpToepMid op{W1, a.kt, E2, a.frames > 1 ? cpf : B, L1};
        HB_TRY(launch_fft_pass(op, f1, 1, E2, (int)N1, 0, (int)N1, 0, 0, 0, s, "toeplitz P3"));
    }
    // P5: axis 2 inverse, crop, output ops
    {
        if (a.sense && a.frames > 1) {
            // frames: one launch per frame over that frame's coil columns, so a CTA sums one frame's
            // coils of a row (one running sum in shared memory) instead of walking every frame's
            // columns with a running sum per frame (measured at 24 frames x 16 coils x 128^3:
            // 7.4 ms against 10.3 ms per apply)
            for (int64_t f = 0; f < a.frames; ++f) {
                OpToepOutSense op{W1 + f * cpf, (int64_t)L2 * B, B, a.smaps_out ? a.smaps_out : a.in, a.out + f * t.n,
                                  N2, t.n, cpf, 1, a.odiag, a.accumulate};
                HB_TRY(launch_fft_pass(op, f2, N0 * N1, cpf, L2, 0, (int)N2, 0, 1, sizeof(float2) * (size_t)N2, s,
                                       "toeplitz P5 sense"));
            }
        } else if (a.sense) {
            OpToepOutSense op{W1,   (int64_t)L2 * B,   B,       a.smaps_out ? a.smaps_out : a.in, a.out, N2, t.n, cpf,
                              (int)a.frames, a.odiag, a.accumulate};
            HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, L2, 0, (int)N2, 0, 1,
                                   sizeof(float2) * (size_t)N2 * a.frames, s, "toeplitz P5 sense"));
        } else {
            OpToepOutFlat op{W1, (int64_t)L2 * B, B, a.in, a.m1, a.m2, a.io_mult, a.out_m1, a.out_m2, a.accumulate,
                             a.out, N2, t.n};
            HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, L2, 0, (int)N2, 0, 1, 0, s, "toeplitz P5"));
        }
    }
    return HB_OK;
}

static bool valid_mult(int m) { return m == HB_MULT_NONE || m == HB_MULT_MULT || m == HB_MULT_MULT_CONJ; }

struct WsGuard {
    float2* ptr = nullptr;
    bool owned = false;
    cudaStream_t s = nullptr;
    ~WsGuard() {
        if (owned && ptr) cudaFreeAsync(ptr, s);
    }
};

static int get_workspace(const ToepGeom& t, void* ws, size_t ws_bytes, cudaStream_t s, WsGuard* g) {
    const size_t need = toep_ws_elems(t) * sizeof(float2);
    if (ws) {
        if (ws_bytes < need) {
            set_error("workspace too small: need " + std::to_string(need) + " bytes, got " + std::to_string(ws_bytes));
            return HB_ERR_WORKSPACE;
        }
        g->ptr = (float2*)ws;
        return HB_OK;
    }
    g->s = s;
    cudaError_t e = cudaMallocAsync((void**)&g->ptr, need, s);
    if (e != cudaSuccess) {
        set_error(std::string("cudaMallocAsync(workspace) failed: ") + cudaGetErrorString(e));
        g->ptr = nullptr;
        return HB_ERR_ALLOC;
    }
    g->owned = true;
    return HB_OK;
}

int toeplitz_workspace_size(int dim, const int64_t* shape, int64_t nbatch, size_t* bytes) {
    ToepGeom t;
    HB_TRY(toep_geom(&t, dim, shape, nbatch));
    HB_REQUIRE(bytes != nullptr, HB_ERR_INVALID_ARG, "bytes is null");
    *bytes = toep_ws_elems(t) * sizeof(float2);
    return HB_OK;
}

int toeplitz_multiplication(int dim, const int64_t* shape, int64_t nbatch, const void* input, void* output,
                            const void* kernel, void* workspace, size_t workspace_bytes, const void* mult1,
                            const void* mult2, int io_mult, int in_m1, int out_m1, int in_m2, int out_m2, int accumulate,
                            cudaStream_t s) {
    ToepGeom t;
    HB_TRY(toep_geom(&t, dim, shape, nbatch));
    HB_REQUIRE(input && output && kernel, HB_ERR_INVALID_ARG, "input, output and kernel must be non-null");
    HB_REQUIRE(valid_mult(io_mult), HB_ERR_INVALID_ARG, "Invalid input_output_mult_type");
    HB_REQUIRE(valid_mult(in_m1), HB_ERR_INVALID_ARG, "Invalid input_mult_type");
    HB_REQUIRE(valid_mult(out_m1), HB_ERR_INVALID_ARG, "Invalid output_mult_type");
    HB_REQUIRE(valid_mult(in_m2), HB_ERR_INVALID_ARG, "Invalid input_mult2_type");
    HB_REQUIRE(valid_mult(out_m2), HB_ERR_INVALID_ARG, "Invalid output_mult2_type");
    HB_REQUIRE(accumulate == HB_ACC_NONE || accumulate == HB_ACC_ACCUMULATE, HB_ERR_INVALID_ARG, "Invalid accumulate_type");
    WsGuard g;
    HB_TRY(get_workspace(t, workspace, workspace_bytes, s, &g));
    ToepArgs a{};
    a.in = (const float2*)input;
    a.out = (float2*)output;
    a.kt = (const float2*)kernel;
    a.m1 = (const float2*)mult1;
    a.m2 = (const float2*)mult2;
    a.io_mult = io_mult;
    a.in_m1 = in_m1;
    a.out_m1 = out_m1;
    a.in_m2 = in_m2;
    a.out_m2 = out_m2;
    a.accumulate = accumulate;
    a.sense = false;
    return toep_run(t, a, g.ptr, s);
}

int sense_normal(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps, const void* kernel,
                 void* out, void* workspace, size_t workspace_bytes, cudaStream_t s) {
    ToepGeom t;
    HB_TRY(toep_geom(&t, dim, shape, ncoils));
    HB_REQUIRE(x && smaps && kernel && out, HB_ERR_INVALID_ARG, "x, smaps, kernel and out must be non-null");
    HB_REQUIRE(out != x, HB_ERR_INVALID_ARG, "out must not alias x");
    WsGuard g;
    HB_TRY(get_workspace(t, workspace, workspace_bytes, s, &g));
    ToepArgs a{};
    a.in = (const float2*)smaps;
    a.out = (float2*)out;
    a.kt = (const float2*)kernel;
    a.m1 = (const float2*)x;
    a.m2 = nullptr;
    a.in_m1 = HB_MULT_MULT;
    a.in_m2 = HB_MULT_NONE;
    a.sense = true;
    return toep_run(t, a, g.ptr, s);
}

int sense_normal_ex(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps_in,
                    const void* smaps_out, const void* diag, int accumulate, const void* kernel, void* out,
                    void* workspace, size_t workspace_bytes, cudaStream_t s) {
    ToepGeom t;
    HB_TRY(toep_geom(&t, dim, shape, ncoils));
    HB_REQUIRE(x && smaps_in && kernel && out, HB_ERR_INVALID_ARG, "x, smaps_in, kernel and out must be non-null");
    HB_REQUIRE(out != x && out != smaps_in && out != smaps_out && out != diag, HB_ERR_INVALID_ARG,
               "out must not alias an input");
    HB_REQUIRE(accumulate == HB_ACC_NONE || accumulate == HB_ACC_ACCUMULATE, HB_ERR_INVALID_ARG, "Invalid accumulate_type");
    WsGuard g;
    HB_TRY(get_workspace(t, workspace, workspace_bytes, s, &g));
    ToepArgs a{};
    a.in = (const float2*)smaps_in;
    a.out = (float2*)out;
    a.kt = (const float2*)kernel;
    a.m1 = (const float2*)x;
    a.m2 = (const float2*)diag;
    a.in_m1 = HB_MULT_MULT;
    a.in_m2 = diag ? HB_MULT_MULT : HB_MULT_NONE;
    a.accumulate = accumulate;
    a.sense = true;
    a.smaps_out = (const float2*)smaps_out;
    a.odiag = (const float2*)diag;
    return toep_run(t, a, g.ptr, s);
}

int sense_normal_batched(int dim, const int64_t* shape, int64_t nframes, int64_t ncoils, const void* x,
                         const void* smaps, const void* kernels, void* out, void* workspace, size_t workspace_bytes,
                         cudaStream_t s) {
    HB_REQUIRE(nframes >= 1 && ncoils >= 1, HB_ERR_INVALID_ARG, "nframes and ncoils must be >= 1");
    ToepGeom t;
    HB_TRY(toep_geom(&t, dim, shape, nframes * ncoils));
    HB_REQUIRE(x && smaps && kernels && out, HB_ERR_INVALID_ARG, "x, smaps, kernels and out must be non-null");
    HB_REQUIRE(out != x, HB_ERR_INVALID_ARG, "out must not alias x");
    WsGuard g;
    HB_TRY(get_workspace(t, workspace, workspace_bytes, s, &g));
    ToepArgs a{};
    a.in = (const float2*)smaps;
    a.out = (float2*)out;
    a.kt = (const float2*)kernels;
    a.m1 = (const float2*)x;
    a.m2 = nullptr;
    a.in_m1 = HB_MULT_MULT;
    a.in_m2 = HB_MULT_NONE;
    a.sense = true;
    a.frames = nframes;
    return toep_run(t, a, g.ptr, s);
}

// Kt[(c * F + f) * R + r] = K_f[r][c] * scale : per-frame transpose [F][R][Cc] -> [Cc][F][R]
__global__ void k_transpose_scale_frames(const float2* __restrict__ in, float2* __restrict__ out, int64_t R, int64_t Cc,
                                         int64_t Lb, int64_t Lc, int64_t F, float scale) {
    __shared__ float2 tile[32][33];
    const int64_t f = blockIdx.z;
    const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
    const float2* src = in + f * R * Cc;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t r = r0 + j, c = c0 + threadIdx.x;
        if (r < R && c < Cc) tile[j][threadIdx.x] = src[r * Cc + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t c = c0 + j, r = r0 + threadIdx.x;
        if (r < R && c < Cc) out[(c * F + f) * R + r] = crop_ramp(cscale(tile[threadIdx.x][j], scale), r, c, R, Lb, Lc);
    }
}

int transform_toeplitz_kernels(int dim, const int64_t* kshape, int64_t nframes, const void* kin, void* kout,
                               cudaStream_t s) {
    HB_REQUIRE(dim == 2 || dim == 3, HB_ERR_INVALID_ARG, "Toeplitz kernel must be 2-D or 3-D");
    HB_REQUIRE(kshape && kin && kout && nframes >= 1 && nframes <= 65535, HB_ERR_INVALID_ARG, "bad argument");
    HB_REQUIRE(kin != kout, HB_ERR_INVALID_ARG, "kernel_in and kernel_out must not alias");
    int64_t R = kshape[0], Cc = 1, tot = 1;
    for (int i = 0; i < dim; ++i) {
        HB_REQUIRE(kshape[i] >= 2 && kshape[i] % 2 == 0, HB_ERR_SHAPE, "kernel dimensions must be even (2N)");
        tot *= kshape[i];
        if (i > 0) Cc *= kshape[i];
    }
    const float scale = (float)(1.0 / (double)tot);
    dim3 grid((unsigned)ceil_div(Cc, 32), (unsigned)ceil_div(R, 32), (unsigned)nframes);
    const int64_t Lb = kshape[1], Lc = dim == 3 ? kshape[2] : 1;
    k_transpose_scale_frames<<<grid, dim3(32, 8), 0, s>>>((const float2*)kin, (float2*)kout, R, Cc, Lb, Lc, nframes, scale);
    return check_launch("transform_toeplitz_kernels");
}

int transform_toeplitz_kernel(int dim, const int64_t* kshape, const void* kin, void* kout, cudaStream_t s) {
    HB_REQUIRE(dim == 2 || dim == 3, HB_ERR_INVALID_ARG, "Toeplitz kernel must be 2-D or 3-D");
    HB_REQUIRE(kshape && kin && kout, HB_ERR_INVALID_ARG, "null argument");
    HB_REQUIRE(kin != kout, HB_ERR_INVALID_ARG, "kernel_in and kernel_out must not alias");
    int64_t R = kshape[0], Cc = 1, tot = 1;
    for (int i = 0; i < dim; ++i) {
        HB_REQUIRE(kshape[i] >= 2 && kshape[i] % 2 == 0, HB_ERR_SHAPE, "kernel dimensions must be even (2N)");
        tot *= kshape[i];
        if (i > 0) Cc *= kshape[i];
    }
    const float scale = (float)(1.0 / (double)tot);
    dim3 grid((unsigned)ceil_div(Cc, 32), (unsigned)ceil_div(R, 32));
    const int64_t Lb = kshape[1], Lc = dim == 3 ? kshape[2] : 1;
    k_transpose_scale<<<grid, dim3(32, 8), 0, s>>>((const float2*)kin, (float2*)kout, R, Cc, Lb, Lc, scale);
    return check_launch("transform_toeplitz_kernel");
}

int toeplitz_kernel_frames(int dim, const int64_t* kshape, int nframes, const int64_t* npts, const float* c0,
                           const float* c1, const float* c2, const void* nudata, void* kout, int width, cudaStream_t s);

int toeplitz_kernel(int dim, const int64_t* kshape, int64_t M, const float* c0, const float* c1, const float* c2,
                    const void* nudata, void* kout, int width, cudaStream_t s) {
    return toeplitz_kernel_frames(dim, kshape, 1, &M, c0, c1, c2, nudata, kout, width, s);
}

// The kernels of nframes frames: one frame-batched type-1 NUFFT over every frame's points, then
// the zero-padding FFT passes over all frames' rows at once. kout is [nframes][2N..].
int toeplitz_kernel_frames(int dim, const int64_t* kshape, int nframes, const int64_t* npts, const float* c0,
                           const float* c1, const float* c2, const void* nudata, void* kout, int width, cudaStream_t s) {
    HB_REQUIRE(dim >= 2 && dim <= 3, HB_ERR_INVALID_ARG, "Toeplitz kernel must be 2-D or 3-D");
    HB_REQUIRE(kshape && npts && kout, HB_ERR_INVALID_ARG, "null argument");
    HB_REQUIRE(nframes >= 1, HB_ERR_INVALID_ARG, "nframes must be >= 1");
    int64_t Mtot = 0;
    for (int f = 0; f < nframes; ++f) Mtot += npts[f] > 0 ? npts[f] : 0;
    HB_REQUIRE(nudata || Mtot == 0, HB_ERR_INVALID_ARG, "null argument");
    const int64_t F = nframes;
    int64_t nm[3], L[3] = {1, 1, 1}, Nimg = 1;
    for (int i = 0; i < dim; ++i) {
        HB_REQUIRE(kshape[i] >= 4 && kshape[i] % 2 == 0, HB_ERR_SHAPE, "kernel dimensions must be even (2N)");
        nm[i] = kshape[i] - 1;
        L[3 - dim + i] = kshape[i];
        Nimg *= kshape[i] / 2;
    }
    NufftPlan plan;
    int st = plan_make(&plan, 1, dim, nm, 1, 1, 1e-5f, width, 2.0, HB_METHOD_DEFAULT);
    float2 *red = nullptr, *b1 = nullptr, *b2 = nullptr;
    auto cleanup = [&]() {
        plan_free(&plan);
        if (red) cudaFree(red);
        if (b1) cudaFree(b1);
        if (b2) cudaFree(b2);
    };
    if (st != HB_OK) {
        cleanup();
        return st;
    }
    const int64_t r0 = L[0] > 1 ? L[0] - 1 : 1, r1 = L[1] - 1, r2 = L[2] - 1;
    const size_t nred = (size_t)F * r0 * r1 * r2;
    cudaError_t e = cudaMalloc(&red, sizeof(float2) * nred);
    if (e == cudaSuccess) e = cudaMalloc(&b1, sizeof(float2) * (size_t)F * r0 * r1 * L[2]);
    if (e == cudaSuccess) e = cudaMalloc(&b2, sizeof(float2) * (size_t)F * r0 * L[1] * L[2]);
    if (e != cudaSuccess) {
        cleanup();
        set_error(std::string("toeplitz_kernel temporaries: ") + cudaGetErrorString(e));
        return HB_ERR_ALLOC;
    }
    do {
        if ((st = plan_setpts_frames(&plan, nframes, npts, c0, c1, c2, s)) != HB_OK) break;
        if ((st = plan_execute(&plan, (const float2*)nudata, red, s)) != HB_OK) break;
        FftLen f0, f1, f2;
        if ((st = get_len((int)L[2], &f2)) != HB_OK) break;
        if ((st = get_len((int)L[1], &f1)) != HB_OK) break;
        if (dim == 3 && (st = get_len((int)L[0], &f0)) != HB_OK) break;
        const float scale = (float)(1.0 / (double)Nimg);
        float2* K = (float2*)kout;
        // axis 2: [F r0 r1][r2] -> b1 [F r0 r1][L2]
        {
            OpStrided op{red, b1, r2, 1, L[2], 1, 1.0f};
            if ((st = launch_fft_pass(op, f2, F * r0 * r1, 1, (int)r2, 0, (int)L[2], 0, 0, 0, s, "toeplitz_kernel axis2")) !=
                HB_OK)
                break;
        }
        // axis 1: [F r0][r1][L2] -> [F r0][L1][L2]
        {
            float2* dst = dim == 3 ? b2 : K;
            OpStrided op{b1, dst, r1 * L[2], L[2], L[1] * L[2], L[2], dim == 3 ? 1.0f : scale};
            if ((st = launch_fft_pass(op, f1, F * r0, L[2], (int)r1, 0, (int)L[1], 0, 0, 0, s, "toeplitz_kernel axis1")) !=
                HB_OK)
                break;
        }
        // axis 0: [F][r0][L1 L2] -> [F][L0][L1 L2]
        if (dim == 3) {
            const int64_t E = L[1] * L[2];
            OpStrided op{b2, K, r0 * E, E, L[0] * E, E, scale};
            if ((st = launch_fft_pass(op, f0, F, E, (int)r0, 0, (int)L[0], 0, 0, 0, s, "toeplitz_kernel axis0")) != HB_OK)
                break;
        }
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
            set_error(std::string("toeplitz_kernel sync: ") + cudaGetErrorString(e));
            st = HB_ERR_CUDA;
        }
    } while (0);
    cleanup();
    return st;
}

}  // namespace hb

// ---- allocation-free SENSE normal operator ------------------------------------------------------
// For callers that cannot allocate device memory: an allocator-less runtime embedded in another
// framework, a driver layer that hands out only fixed buffers, or code running where
// cudaMalloc is off limits. The workspace and the FFT twiddle tables live in file-scope device
// arrays of fixed size that every GPU loading this library keeps until the process exits.
namespace hb {

constexpr size_t kNoAllocWsBytes = size_t(32) << 20;  // 32 MiB of workspace
constexpr int kNoAllocMaxLen = 4096;                  // longest 2N per axis
static __device__ __align__(256) float2 g_noalloc_ws[kNoAllocWsBytes / sizeof(float2)];
static __device__ __align__(256) float2 g_noalloc_tw[3 * kNoAllocMaxLen];

struct NoAllocDevice {
    int dev = -1;
    unsigned long long ctx_id = 0;  // driver context id the addresses belong to
    float2* ws = nullptr;
    float2* tw = nullptr;
};
static std::mutex g_noalloc_mu;
static std::vector<NoAllocDevice> g_noalloc_dev;

// Unique id of the current driver context (cuCtxGetId, reached through the runtime's driver
// entry-point query so the library does not link libcuda). A device reset destroys the primary
// context and the next runtime call creates a new one with a new id, at which point the module
// holding the arrays is loaded again at new addresses.
static int current_context_id(unsigned long long* id) {
    using PfnGetCurrent = CUresult (*)(CUcontext*);
    using PfnGetId = CUresult (*)(CUcontext, unsigned long long*);
    static PfnGetCurrent get_current = nullptr;
    static PfnGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (PfnGetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (PfnGetId)f;
    });
    HB_REQUIRE(get_current && get_id, HB_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
    CUcontext ctx = nullptr;
    HB_REQUIRE(get_current(&ctx) == CUDA_SUCCESS && ctx != nullptr, HB_ERR_CUDA, "no current CUDA context");
    HB_REQUIRE(get_id(ctx, id) == CUDA_SUCCESS, HB_ERR_CUDA, "cuCtxGetId failed");
    return HB_OK;
}

// Device addresses of the two arrays for the current device, looked up once per device and
// context with that device current.
static int noalloc_addresses(NoAllocDevice* out) {
    int dev = 0;
    HB_CUDA(cudaGetDevice(&dev));
    HB_CUDA(cudaSetDevice(dev));  // initialises the device's primary context and makes it current
    unsigned long long ctx_id = 0;
    HB_TRY(current_context_id(&ctx_id));
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if ((int)g_noalloc_dev.size() <= dev) g_noalloc_dev.resize(dev + 1);
    NoAllocDevice& d = g_noalloc_dev[dev];
    if (d.ws == nullptr || d.tw == nullptr || d.dev != dev || d.ctx_id != ctx_id) {
        void* ws = nullptr;
        void* tw = nullptr;
        HB_CUDA(cudaGetSymbolAddress(&ws, g_noalloc_ws));
        HB_CUDA(cudaGetSymbolAddress(&tw, g_noalloc_tw));
        d.dev = dev;
        d.ctx_id = ctx_id;
        d.ws = (float2*)ws;
        d.tw = (float2*)tw;
    }
    *out = d;
    return HB_OK;
}

__global__ void k_fill_twiddles(float2* tw, int L) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= L) return;
    double sn, cs;
    sincospi(-2.0 * (double)m / (double)L, &sn, &cs);
    tw[m] = make_float2((float)cs, (float)sn);
}

// Radix plan of L (same factor order as fftlen_make) with the twiddles at `tw`.
static int noalloc_len(int L, float2* tw, cudaStream_t s, FftLen* f) {
    f->L = L;
    f->nrad = 0;
    f->tw = tw;
    int rest = L;
    for (int r : {8, 4, 2, 5, 3, 7, 11, 13}) {
        while (rest % r == 0 && rest > 1) {
            HB_REQUIRE(f->nrad < kMaxRadices, HB_ERR_INVALID_ARG, "FFT length has too many factors");
            f->rad[f->nrad++] = r;
            rest /= r;
        }
    }
    HB_REQUIRE(rest == 1, HB_ERR_INVALID_ARG, "2N must have no prime factor above 13 on any axis");
    k_fill_twiddles<<<(unsigned)ceil_div(L, 256), 256, 0, s>>>(tw, L);
    return check_launch("k_fill_twiddles");
}

int sense_normal_noalloc(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps,
                         const void* kernel, void* out, cudaStream_t s) {
    ToepGeom t;
    HB_TRY(toep_geom(&t, dim, shape, ncoils));
    HB_REQUIRE(x && smaps && kernel && out, HB_ERR_INVALID_ARG, "x, smaps, kernel and out must be non-null");
    HB_REQUIRE(out != x, HB_ERR_INVALID_ARG, "out must not alias x");
    const size_t need = toep_ws_elems(t) * sizeof(float2);
    if (need > kNoAllocWsBytes) {
        set_error("hb_sense_normal_noalloc: problem needs " + std::to_string(need) +
                  " bytes of workspace, the fixed array holds " + std::to_string(kNoAllocWsBytes) +
                  (t.dim == 3 ? " (3-D: 6 * prod(N) * ncoils * 8 bytes must fit)"
                              : " (2-D: 2 * prod(N) * ncoils * 8 bytes must fit)"));
        return HB_ERR_WORKSPACE;
    }
    for (int ax = 0; ax < 3; ++ax)
        HB_REQUIRE(t.L[ax] <= kNoAllocMaxLen, HB_ERR_INVALID_ARG, "hb_sense_normal_noalloc: 2N must be <= 4096");
    NoAllocDevice d;
    HB_TRY(noalloc_addresses(&d));
    FftLen f0, f1, f2;
    HB_TRY(noalloc_len(t.L[2], d.tw + 2 * kNoAllocMaxLen, s, &f2));
    HB_TRY(noalloc_len(t.L[1], d.tw + 1 * kNoAllocMaxLen, s, &f1));
    if (t.dim == 3) HB_TRY(noalloc_len(t.L[0], d.tw, s, &f0));

    const int64_t B = t.B, N0 = t.N[0], N1 = t.N[1], N2 = t.N[2];
    const int L0 = t.L[0], L1 = t.L[1], L2 = t.L[2];
    const float2* S = (const float2*)smaps;
    float2* W1 = d.ws;
    float2* W2 = d.ws + (size_t)N0 * N1 * L2 * B;
    const int64_t E2 = (int64_t)L2 * B;
    {
        OpToepInSense op{{S, (const float2*)x, nullptr, HB_MULT_MULT, HB_MULT_NONE, W1, N2, t.n, E2, B, 0}};
        HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, (int)N2, 0, L2, 0, 0, 0, s, "noalloc P1"));
    }
    if (t.dim == 3) {
        {
            OpStridedPad op{{W1, W2, N1 * E2, E2, (int64_t)L1 * E2, E2, 1.0f}};
            HB_TRY(launch_fft_pass(op, f1, N0, E2, (int)N1, 0, L1, 0, 0, 0, s, "noalloc P2"));
        }
        {
            const int64_t E = (int64_t)L1 * E2;
            OpToepMid op{W2, (const float2*)kernel, E, B, L0};
            HB_TRY(launch_fft_pass(op, f0, 1, E, (int)N0, 0, (int)N0, 0, 0, 0, s, "noalloc P3"));
        }
        {
            OpStridedCrop op{{W2, W1, (int64_t)L1 * E2, E2, N1 * E2, E2, 1.0f}};
            HB_TRY(launch_fft_pass(op, f1, N0, E2, L1, 0, (int)N1, 0, 1, 0, s, "noalloc P4"));
        }
    } else {
        OpToepMid op{W1, (const float2*)kernel, E2, B, L1};
        HB_TRY(launch_fft_pass(op, f1, 1, E2, (int)N1, 0, (int)N1, 0, 0, 0, s, "noalloc P3"));
    }
    {
        OpToepOutSense op{W1, E2, B, S, (float2*)out, N2, t.n, B, 1, nullptr, 0};
        HB_TRY(launch_fft_pass(op, f2, N0 * N1, B, L2, 0, (int)N2, 0, 1, sizeof(float2) * (size_t)N2, s,
                               "noalloc P5 sense"));
    }
    return HB_OK;
}

}  // namespace hb
