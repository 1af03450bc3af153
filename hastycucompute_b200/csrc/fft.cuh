// Shared-memory mixed-radix FFT passes over strided columns.
//
// One "pass" transforms a 3-level array  X[a][l][e]  (a = outer batch, l = the transformed
// axis, e = inner columns, contiguous) along l. A CTA takes A_blk outer x E_blk inner columns,
// stages the L samples of each column in shared memory, runs Stockham radix-{2,3,4,5,7,8,11,13}
// stages between two shared buffers, and writes back. Pruning is built into the pass:
//   - only Lin input samples are read; sample l lands at FFT position (l + in_shift) mod L and
//     every other position is zero (zero padding / centred modes without a padding pass);
//   - only Lout outputs are kept; output o comes from position (o + out_shift) mod L (crop /
//     centred modes without a crop pass).
// An Op object supplies the element loads and stores, so pre-multiplies (coil maps, the
// deapodisation), post-multiplies and the coil reduction run inside the pass.
#pragma once

#include <stdint.h>

#include <type_traits>
#include <utility>

#include "common.cuh"
#include "timing.cuh"

namespace hb {

constexpr int kMaxRadices = 12;
constexpr int kPassThreads = 256;

// Radix plan and twiddle table of one FFT length (owned by whoever builds it).
struct FftLen {
    int L = 1;
    int nrad = 0;
    int rad[kMaxRadices] = {0};
    float2* tw = nullptr;  // device, L entries, tw[m] = exp(-2 pi i m / L)
};

// Factorises L into radices 8,4,2,5,3,7,11,13 (an error if L has another prime factor) and
// uploads its twiddle table (synchronous cudaMalloc + cudaMemcpy).
int fftlen_make(FftLen* f, int L);
void fftlen_free(FftLen* f);

struct PassCfg {
    int L;
    int nrad;
    int rad[kMaxRadices];
    const float2* tw;
    int Lin, in_shift;    // sample l in [0, Lin) -> position (l + in_shift) mod L
    int Lout, out_shift;  // output o in [0, Lout) <- position (o + out_shift) mod L
    int64_t A, E;         // outer and inner extents
    int A_blk, E_blk;     // per CTA
    int W, Wp;            // W = A_blk*E_blk columns; Wp = shared row stride (odd)
    int64_t n_eb;         // inner blocks per outer block
    int inverse;          // 0: exp(-...), 1: exp(+...)
};

// Chooses the columns per CTA for length L so that two CTAs fit on an SM.
int pass_columns_for(int L);

// Fills the block decomposition of cfg for extents (A, E) and length information. max_cols > 0
// fixes the columns per CTA (the register kernel); otherwise they follow the shared budget.
void pass_setup(PassCfg* c, const FftLen& f, int64_t A, int64_t E, int Lin, int in_shift,
                int Lout, int out_shift, int inverse, int max_cols = 0);

// Shared bytes a pass kernel needs (two buffers + twiddles + op extra).
inline size_t pass_smem_bytes(const PassCfg& c, size_t extra_bytes) {
    return (size_t)(2 * c.L * c.Wp + c.L) * sizeof(float2) + extra_bytes;
}

#ifdef __CUDACC__

// ---- compile-time twiddles -----------------------------------------------------------------
// W_R^m = exp(-2 pi i m / R) evaluated while compiling: the angle is reduced to [-pi, pi] and
// sine / cosine are summed from their Taylor series in double (terms to x^31, error far below
// float rounding), then rounded once to float. Exact quarter turns become swaps.
constexpr double kTwoPi = 6.283185307179586476925286766559;

constexpr double ct_sin(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 16; ++k) {
        term *= -x * x / (double)((2 * k) * (2 * k + 1));
        sum += term;
    }
    return sum;
}
constexpr double ct_cos(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 16; ++k) {
        term *= -x * x / (double)((2 * k - 1) * (2 * k));
        sum += term;
    }
    return sum;
}
template <int R, int M>
constexpr double ct_angle() {
    constexpr int m = ((M % R) + R) % R;
    return kTwoPi * (double)(2 * m > R ? m - R : m) / (double)R;  // in [-pi, pi]
}

// Calls f(std::integral_constant<int, I>) for I = 0 .. N-1 (indices usable as constants).
template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- DFT codelets ----------------------------------------------------------------------
// forward: y_s = sum_r x_r exp(-2 pi i r s / R); INV flips the sign of the exponent.
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }   // a * (-i)
__device__ __forceinline__ float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }   // a * (+i)

template <bool INV>
__device__ __forceinline__ void dft2(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
    float2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = csub(x1, x3);
    float2 r3 = INV ? mul_pi(t3) : mul_mi(t3);
    x0 = cadd(t0, t2);
    x2 = csub(t0, t2);
    x1 = cadd(t1, r3);
    x3 = csub(t1, r3);
}

template <bool INV>
__device__ __forceinline__ void dft3(float2* v) {
    const float s = 0.86602540378443864676f;  // sin(2 pi / 3)
    float2 t = cadd(v[1], v[2]);
    float2 u = csub(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    float2 su = cscale(u, s);
    float2 isu = INV ? mul_pi(su) : mul_mi(su);  // -/+ i s u
    v[0] = cadd(v[0], t);
    v[1] = cadd(m, isu);
    v[2] = csub(m, isu);
}

template <bool INV>
__device__ __forceinline__ void dft5(float2* v) {
    const float c1 = 0.30901699437494742410f;   // cos(2 pi/5)
    const float c2 = -0.80901699437494742410f;  // cos(4 pi/5)
    const float s1 = 0.95105651629515357212f;   // sin(2 pi/5)
    const float s2 = 0.58778525229247312917f;   // sin(4 pi/5)
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 u1 = csub(v[1], v[4]), u2 = csub(v[2], v[3]);
    float2 a1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 a2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 b1 = make_float2(s1 * u1.x + s2 * u2.x, s1 * u1.y + s2 * u2.y);
    float2 b2 = make_float2(s2 * u1.x - s1 * u2.x, s2 * u1.y - s1 * u2.y);
    float2 ib1 = INV ? mul_pi(b1) : mul_mi(b1);  // -/+ i b1
    float2 ib2 = INV ? mul_pi(b2) : mul_mi(b2);
    v[0] = make_float2(v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y);
    v[1] = cadd(a1, ib1);
    v[4] = csub(a1, ib1);
    v[2] = cadd(a2, ib2);
    v[3] = csub(a2, ib2);
}

template <bool INV>
__device__ __forceinline__ void dft7(float2* v) {
    const float c1 = 0.62348980185873353053f;   // cos(2 pi/7)
    const float c2 = -0.22252093395631440429f;  // cos(4 pi/7)
    const float c3 = -0.90096886790241912624f;  // cos(6 pi/7)
    const float s1 = 0.78183148246802980871f;   // sin(2 pi/7)
    const float s2 = 0.97492791218182360702f;   // sin(4 pi/7)
    const float s3 = 0.43388373911755812048f;   // sin(6 pi/7)
    const float2 t1 = cadd(v[1], v[6]), t2 = cadd(v[2], v[5]), t3 = cadd(v[3], v[4]);
    const float2 u1 = csub(v[1], v[6]), u2 = csub(v[2], v[5]), u3 = csub(v[3], v[4]);
    const float2 x0 = v[0];
    auto lin3 = [](float a, float2 p, float b, float2 q, float c, float2 r) {
        return make_float2(a * p.x + b * q.x + c * r.x, a * p.y + b * q.y + c * r.y);
    };
    const float2 a1 = cadd(x0, lin3(c1, t1, c2, t2, c3, t3));
    const float2 a2 = cadd(x0, lin3(c2, t1, c3, t2, c1, t3));
    const float2 a3 = cadd(x0, lin3(c3, t1, c1, t2, c2, t3));
    const float2 b1 = lin3(s1, u1, s2, u2, s3, u3);
    const float2 b2 = lin3(s2, u1, -s3, u2, -s1, u3);
    const float2 b3 = lin3(s3, u1, -s1, u2, s2, u3);
    const float2 ib1 = INV ? mul_pi(b1) : mul_mi(b1);
    const float2 ib2 = INV ? mul_pi(b2) : mul_mi(b2);
    const float2 ib3 = INV ? mul_pi(b3) : mul_mi(b3);
    v[0] = cadd(x0, cadd(t1, cadd(t2, t3)));
    v[1] = cadd(a1, ib1);
    v[6] = csub(a1, ib1);
    v[2] = cadd(a2, ib2);
    v[5] = csub(a2, ib2);
    v[3] = cadd(a3, ib3);
    v[4] = csub(a3, ib3);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2* v) {
    const float h = 0.70710678118654752440f;
    // even / odd radix-4 halves
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // o_s *= W8^s, W8 = exp(-/+ 2 pi i / 8)
    float2 w1o, w2o, w3o;
    if (!INV) {
        w1o = make_float2(h * (o1.x + o1.y), h * (o1.y - o1.x));   // (1 - i)/sqrt2
        w2o = mul_mi(o2);
        w3o = make_float2(h * (-o3.x + o3.y), h * (-o3.y - o3.x)); // (-1 - i)/sqrt2
    } else {
        w1o = make_float2(h * (o1.x - o1.y), h * (o1.y + o1.x));   // (1 + i)/sqrt2
        w2o = mul_pi(o2);
        w3o = make_float2(h * (-o3.x - o3.y), h * (-o3.y + o3.x)); // (-1 + i)/sqrt2
    }
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, w1o);
    v[5] = csub(e1, w1o);
    v[2] = cadd(e2, w2o);
    v[6] = csub(e2, w2o);
    v[3] = cadd(e3, w3o);
    v[7] = csub(e3, w3o);
}

// Odd-prime DFT (11, 13) by the symmetric pairs t_j = x_j + x_{R-j}, u_j = x_j - x_{R-j}:
//   y_k = x_0 + sum_j cos(2 pi jk/R) t_j -/+ i sum_j sin(2 pi jk/R) u_j, y_{R-k} with the other
// sign (forward / inverse); every cosine and sine is a compile-time constant.
template <int R, bool INV>
__device__ __forceinline__ void dft_odd(float2* v) {
    constexpr int H = (R - 1) / 2;
    float2 t[H], u[H];
#pragma unroll
    for (int j = 1; j <= H; ++j) {
        t[j - 1] = cadd(v[j], v[R - j]);
        u[j - 1] = csub(v[j], v[R - j]);
    }
    const float2 x0 = v[0];
    float2 sum = x0;
#pragma unroll
    for (int j = 0; j < H; ++j) sum = cadd(sum, t[j]);
    static_for<H>([&](auto kk) {
        constexpr int k = decltype(kk)::value + 1;
        float2 a = x0, b = make_float2(0.f, 0.f);
        static_for<H>([&](auto jj) {
            constexpr int j = decltype(jj)::value + 1;
            constexpr float c = (float)ct_cos(ct_angle<R, j * k>());
            constexpr float sn = (float)ct_sin(ct_angle<R, j * k>());
            a.x = fmaf(c, t[j - 1].x, a.x);
            a.y = fmaf(c, t[j - 1].y, a.y);
            b.x = fmaf(sn, u[j - 1].x, b.x);
            b.y = fmaf(sn, u[j - 1].y, b.y);
        });
        const float2 ib = INV ? mul_pi(b) : mul_mi(b);
        v[k] = cadd(a, ib);
        v[R - k] = csub(a, ib);
    });
    v[0] = sum;
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 11 || R == 13) dft_odd<R, INV>(v);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) dft5<INV>(v);
    else if constexpr (R == 7) dft7<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
}

// One Stockham stage: src -> dst, p = product of the radices already applied.
//   butterfly i in [0, L/R): k = i mod p; inputs src[i + r L/R]; twiddle exp(-/+2 pi i k r/(pR));
//   outputs dst[(i - k) R + k + s p].
template <int R, bool INV>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ src, float2* __restrict__ dst,
                                          const float2* __restrict__ tw, int L, int p, int W, int Wp) {
    const int m = L / R;
    const int total = m * W;
    const int twstep = L / (p * R);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int col = idx % W;
        const int i = idx / W;
        const int k = i % p;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[(i + r * m) * Wp + col];
        if (p > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 t = tw[r * k * twstep];
                if (INV) t.y = -t.y;
                v[r] = cmul(v[r], t);
            }
        }
        dft<R, INV>(v);
        const int j = (i - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(j + r * p) * Wp + col] = v[r];
    }
}

// Runs all stages; a holds the input, b is scratch. Returns the buffer with the result.
// Must be entered after a __syncthreads that published a.
template <bool INV>
__device__ float2* fft_run(float2* a, float2* b, const float2* tw, const PassCfg& c, int W) {
    int p = 1;
    for (int s = 0; s < c.nrad; ++s) {
        const int R = c.rad[s];
        switch (R) {
            case 8: fft_stage<8, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 4: fft_stage<4, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 2: fft_stage<2, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 5: fft_stage<5, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 3: fft_stage<3, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 7: fft_stage<7, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 11: fft_stage<11, INV>(a, b, tw, c.L, p, W, c.Wp); break;
            case 13: fft_stage<13, INV>(a, b, tw, c.L, p, W, c.Wp); break;
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        p *= R;
    }
    return a;
}

__device__ __forceinline__ float2* fft_run_dir(float2* a, float2* b, const float2* tw, const PassCfg& c,
                                               int W, bool inverse) {
    return inverse ? fft_run<true>(a, b, tw, c, W) : fft_run<false>(a, b, tw, c, W);
}

// ---- generic pass kernel -----------------------------------------------------------------
// Op contract:
//   static constexpr bool kLoadLFast      // true: the source is contiguous along l
//   static constexpr bool kFusedK         // multiply by a kernel, then transform back
//   static constexpr bool kChunkLoop      // CTA walks all inner blocks of its outer block
//   float2 load(int64_t a, int l, int64_t e) const
//   float2 kval(int64_t a, int p, int64_t e) const                  (kFusedK)
//   void store_phase(const float2* res, const PassCfg&, int64_t a0, int64_t e0, int Ab, int Eb,
//                    float2* extra) const                          (all outputs of this chunk)
//   void finish(const PassCfg&, int64_t a0, float2* extra) const    (kChunkLoop)
template <class Op>
__global__ void __launch_bounds__(kPassThreads) pass_kernel(const Op op, const PassCfg c) {
    extern __shared__ float2 smem[];
    float2* bufA = smem;
    float2* bufB = smem + (size_t)c.L * c.Wp;
    float2* tw = bufB + (size_t)c.L * c.Wp;
    float2* extra = tw + c.L;

    for (int i = threadIdx.x; i < c.L; i += blockDim.x) tw[i] = c.tw[i];

    int64_t ab, eb_begin, eb_end;
    if (Op::kChunkLoop) {
        ab = blockIdx.x;
        eb_begin = 0;
        eb_end = c.n_eb;
    } else {
        const unsigned neb = (unsigned)c.n_eb;  // grid < 2^31 blocks: a 32-bit split
        const unsigned q = blockIdx.x / neb;
        ab = q;
        eb_begin = blockIdx.x - q * neb;
        eb_end = eb_begin + 1;
    }
    const int64_t a0 = ab * c.A_blk;
    const int W = c.W;

    for (int64_t eb = eb_begin; eb < eb_end; ++eb) {
        const int64_t e0 = eb * c.E_blk;
        // load all L positions of every column (zero where no sample lands)
        const int total = c.A_blk * c.L * c.E_blk;
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            int pos, el, al;
            if (Op::kLoadLFast) {
                pos = idx % c.L;
                int rest = idx / c.L;
                el = rest % c.E_blk;
                al = rest / c.E_blk;
            } else {
                el = idx % c.E_blk;
                int rest = idx / c.E_blk;
                pos = rest % c.L;
                al = rest / c.L;
            }
            int l = pos - c.in_shift;
            l %= c.L;
            if (l < 0) l += c.L;
            const int64_t a = a0 + al, e = e0 + el;
            float2 v = make_float2(0.f, 0.f);
            if (l < c.Lin && a < c.A && e < c.E) v = op.load(a, l, e);
            bufA[pos * c.Wp + al * c.E_blk + el] = v;
        }
        __syncthreads();
        float2* res = fft_run_dir(bufA, bufB, tw, c, W, c.inverse != 0);
        if constexpr (Op::kFusedK) {
            const int tot2 = c.L * W;
            for (int idx = threadIdx.x; idx < tot2; idx += blockDim.x) {
                const int col = idx % W, pos = idx / W;
                const int al = col / c.E_blk, el = col % c.E_blk;
                const int64_t a = a0 + al, e = e0 + el;
                if (a < c.A && e < c.E) res[pos * c.Wp + col] = cmul(res[pos * c.Wp + col], op.kval(a, pos, e));
            }
            __syncthreads();
            float2* other = (res == bufA) ? bufB : bufA;
            res = fft_run_dir(res, other, tw, c, W, c.inverse == 0);
        }
        op.store_phase(res, c, a0, e0, c.A_blk, c.E_blk, extra);
        __syncthreads();
    }
    if constexpr (Op::kChunkLoop) op.finish(c, a0, extra);
}

// Helper for store phases: visits every kept (a, o, e) of the chunk with the value res[...].
// LFAST: consecutive threads take consecutive o (destination contiguous along o).
template <bool LFAST, class F>
__device__ __forceinline__ void for_each_output(const float2* res, const PassCfg& c, int64_t a0, int64_t e0,
                                                F&& f) {
    const int total = c.A_blk * c.Lout * c.E_blk;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        int o, el, al;
        if (LFAST) {
            o = idx % c.Lout;
            int rest = idx / c.Lout;
            el = rest % c.E_blk;
            al = rest / c.E_blk;
        } else {
            el = idx % c.E_blk;
            int rest = idx / c.E_blk;
            o = rest % c.Lout;
            al = rest / c.Lout;
        }
        const int64_t a = a0 + al, e = e0 + el;
        if (a >= c.A || e >= c.E) continue;
        int pos = (o + c.out_shift) % c.L;
        if (pos < 0) pos += c.L;
        f(a, o, e, res[pos * c.Wp + al * c.E_blk + el]);
    }
}

// Launches pass_kernel<Op> with the needed dynamic shared memory.
template <class Op>
int launch_pass(const Op& op, const PassCfg& c, size_t extra_bytes, cudaStream_t s, const char* name) {
    const size_t smem = pass_smem_bytes(c, extra_bytes);
    static_assert(kPassThreads == 256, "");
    cudaError_t e = cudaFuncSetAttribute(pass_kernel<Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);

    if (e != cudaSuccess) {
        set_error(std::string(name) + ": cudaFuncSetAttribute failed: " + cudaGetErrorString(e));
        return HB_ERR_CUDA;
    }
    const int64_t n_ab = ceil_div(c.A, c.A_blk);
    const int64_t blocks = Op::kChunkLoop ? n_ab : n_ab * c.n_eb;
    if (blocks <= 0) return HB_OK;
    if (blocks > 0x7fffffffLL) {
        set_error(std::string(name) + ": grid too large");
        return HB_ERR_INVALID_ARG;
    }
    TimedSection ts(name, s);
    pass_kernel<Op><<<(unsigned)blocks, kPassThreads, smem, s>>>(op, c);
    return check_launch(name);
}

#endif  // __CUDACC__

}  // namespace hb
