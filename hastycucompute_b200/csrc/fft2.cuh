// Two-level register FFT pass (L = P * Q) for the lengths the hot path uses.
//
// For one column x[0..L), with n = t + Q j and k = k1 + P k2 (t, k2 < Q; j, k1 < P):
//     X[k1 + P k2] = sum_t W_Q^{t k2} [ W_L^{t k1} sum_j x[t + Q j] W_P^{j k1} ]
// Step 1: thread t loads its P samples straight from global memory into registers, runs the
// P-point DFT, applies the twiddles W_L^{t k1} and writes one row of the shared transpose.
// Step 2: thread k1 reads its Q values, runs the Q-point DFT and stores X[k1 + P k2] directly.
// One shared-memory round trip per transform, P (or Q) independent global accesses per thread.
// A CTA handles CW columns; the pruned load / store position maps are those of fft.cuh.
//
// Fused kernel passes (forward, multiply, inverse) continue from step 2 without a transpose:
// thread k1 multiplies by the kernel, runs the inverse Q-point DFT over k2, twiddles by
// W_L^{-n2 k1}, and after one more transpose thread n2 runs the inverse P-point DFT giving
// x[n2 + Q n1].
#pragma once

#include <type_traits>
#include <utility>

#include "fft.cuh"

namespace hb {

#ifdef __CUDACC__

template <int R>
struct IsBaseRadix {
    static constexpr bool value = R == 1 || R == 2 || R == 3 || R == 4 || R == 5 || R == 7 || R == 8;
};

// first factor used to split a composite register DFT
template <int R>
constexpr int split_factor() {
    return (R % 4 == 0) ? 4 : (R % 2 == 0) ? 2 : (R % 3 == 0) ? 3 : (R % 5 == 0) ? 5 : 7;
}

// W_L^m from the shared table (exp(-2 pi i m / L)), conjugated for the inverse
template <bool INV>
__device__ __forceinline__ float2 tw_get(const float2* tw, int m) {
    float2 w = tw[m];
    if (INV) w.y = -w.y;
    return w;
}

// a * W_R^M (INV: conjugate twiddle)
template <int R, int M, bool INV>
__device__ __forceinline__ float2 cmul_tw(float2 a) {
    constexpr int m = ((M % R) + R) % R;
    if constexpr (m == 0) {
        return a;
    } else if constexpr (4 * m == R) {
        return INV ? mul_pi(a) : mul_mi(a);  // -i (forward) / +i (inverse)
    } else if constexpr (2 * m == R) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * m == 3 * R) {
        return INV ? mul_mi(a) : mul_pi(a);
    } else {
        constexpr float c = (float)ct_cos(ct_angle<R, M>());
        constexpr float sn = (float)(INV ? ct_sin(ct_angle<R, M>()) : -ct_sin(ct_angle<R, M>()));
        return make_float2(fmaf(a.x, c, -a.y * sn), fmaf(a.x, sn, a.y * c));
    }
}

// In-register DFT of size R (composite sizes split as A x B with constant twiddles).
template <int R, bool INV>
__device__ __forceinline__ void dft_reg(float2* v, const float2* = nullptr, int = 0) {
    if constexpr (R == 1) {
        return;
    } else if constexpr (IsBaseRadix<R>::value) {
        dft<R, INV>(v);
    } else {
        constexpr int A = split_factor<R>();
        constexpr int B = R / A;
        float2 y[R];
        static_for<B>([&](auto tc) {
            constexpr int t = decltype(tc)::value;
            float2 a[A];
#pragma unroll
            for (int j = 0; j < A; ++j) a[j] = v[t + B * j];
            dft<A, INV>(a);
            static_for<A>([&](auto kc) {
                constexpr int k1 = decltype(kc)::value;
                y[t * A + k1] = cmul_tw<R, t * k1, INV>(a[k1]);
            });
        });
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 b[B];
#pragma unroll
            for (int t = 0; t < B; ++t) b[t] = y[t * A + k1];
            dft_reg<B, INV>(b);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = b[k2];
        }
    }
}

// DFT of size R whose inputs v[R/2..R) are zero: X[2m] = DFT_{R/2}(v)[m],
// X[2m+1] = DFT_{R/2}(v_j W_R^j)[m].
template <int R, bool INV>
__device__ __forceinline__ void dft_reg_halfzero(float2* v, const float2* = nullptr, int = 0) {
    if constexpr (R % 2 != 0 || R < 4) {
        dft_reg<R, INV>(v);
    } else {
        constexpr int H = R / 2;
        float2 a[H], b[H];
        static_for<H>([&](auto jc) {
            constexpr int j = decltype(jc)::value;
            a[j] = v[j];
            b[j] = cmul_tw<R, j, INV>(v[j]);
        });
        dft_reg<H, INV>(a);
        dft_reg<H, INV>(b);
#pragma unroll
        for (int m = 0; m < H; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
}

constexpr int kCW = 16;  // columns per CTA
constexpr int kMaxKCols = 4;  // distinct kernel columns a fused CTA stages in shared memory

// 8-byte asynchronous global -> shared copy (sm_80+ LDGSTS); completes at cp_async_wait_all.
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// 16-byte variant (both addresses 16-byte aligned); bypasses L1.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// waits until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Op::kStageRow (optional, default false): on zero-padded inputs each sample is
// load_col(a, l, e) * row(a, e0)[l] when row_shared(e0, E_blk) (one row factor for all columns
// e0 .. e0+E_blk-1 of a row), else load_col(a, l, e) * row_at(a, l, e).
template <class Op, class = void>
struct StageRow {
    static constexpr bool value = false;
};
template <class Op>
struct StageRow<Op, std::void_t<decltype(Op::kStageRow)>> {
    static constexpr bool value = Op::kStageRow;
};

// Op::kPrefetch (optional, default false; inputs at fixed positions: zero-padded Lin == L/2 or the
// full L, shift 0): where a CTA holds one outer row (A_blk == 1) the CTAs are persistent and walk
// the (row, column block) jobs with a stride of the grid (a chunk-looping operator keeps all blocks
// of a row on one CTA); each job's samples arrive in shared memory by cp.async issued while the
// previous job is transformed, and Op::sample_ptr(a, l, e) gives the sample's address (columns contiguous
// along e). Other block shapes run the same operator without prefetching.
template <class Op, class = void>
struct Prefetch {
    static constexpr bool value = false;
};
template <class Op>
struct Prefetch<Op, std::void_t<decltype(Op::kPrefetch)>> {
    static constexpr bool value = Op::kPrefetch;
};

// kernel columns a fused CTA stages: two for the prefetching passes (which also hold a block of
// samples in shared memory), kMaxKCols otherwise
template <bool PF>
constexpr int max_kcols() {
    return PF ? 2 : kMaxKCols;
}

// Op contract (in addition to fft.cuh's):
//   static constexpr bool kStoreLFast    // destination contiguous along the output index
//   static constexpr bool kSenseReduce   // sum over inner columns into one output row
//   void store(int64_t a, int o, int64_t e, float2 v) const
//   float2 product(int64_t a, int o, int64_t e, float2 v) const        (kSenseReduce)
//   void write_row(int64_t a, int o, float2 v) const                   (kSenseReduce)
//   int64_t kcol(int64_t e) const; const float2* kptr(int64_t kc) const (kFusedK: column e
//       multiplies by kptr(kcol(e))[pos]; the CTA stages its distinct columns in shared memory)
//   const float2* srow(int64_t a, int64_t e) const                      (kSenseReduce: the
//       factor row of (a, e), staged per chunk; product_s(v, s) combines a value with it)
//
// HM (compile-time pass shape): bit 0 = the input is zero-padded to twice its length at offset 0
// (Lin == L/2, in_shift == 0), so only samples j < P/2 of step 1 are loaded and the P-point DFT
// skips the zero half; bit 1 = the output is the first half (Lout == L/2, out_shift == 0), so
// step 2 stores k2 < Q/2 (fused passes: step 3 stores n1 < P/2) with no position checks. A
// halved operator also fixes the side its bits leave out at the full length L with shift 0, so
// those loads and stores go to compile-time positions as well. Bits 2 / 3 declare the same for
// the input / output of an operator without a fixed shape (kHalfIO 0): the launcher picks them
// from the pass's lengths and shifts.
//
// CTAs per SM (320-thread blocks): the coil-reduce pass keeps 2 (96 registers; prefetching the
// next chunk, 160^3 x 32 coils: 0.756 ms; at 3 CTAs it spills 32 bytes per thread and takes
// 0.805 ms), the fused-kernel passes 3 (64 registers; the prefetching instance at L = 320 spills
// 12 bytes and takes 3.31 ms against 3.41 ms at 2 CTAs and 96 registers), every other pass 4 (48
// registers, a few spilled words): they move bytes, and the fourth CTA hides more of the load
// latency than the spills cost (prefetching them at 2 or 3 CTAs measured slower).
template <class Op, int L, int HM, bool PF>
constexpr int pass2_min_blocks() {
    return Op::kSenseReduce ? 2 : Op::kFusedK ? 3 : (PF ? ((HM & 1) ? 3 : 2) : 4);
}
template <int P, int Q, class Op, int HM = 0, bool PF = false>
__global__ void __launch_bounds__(Q* kCW, (Q * kCW > 320) ? 1 : pass2_min_blocks<Op, P * Q, HM, PF>())
    pass2_kernel(const Op op, const PassCfg c) {
    constexpr int L = P * Q;
    constexpr int CWp = kCW + 1;
    constexpr bool kHalfIn = (HM & 1) != 0;
    constexpr bool kHalfOut = (HM & 2) != 0;
    // all L positions, unshifted: the side a halved operator leaves out, or bits 2 / 3
    constexpr bool kFullIn = !kHalfIn && ((HM & 2) != 0 || (HM & 4) != 0);
    constexpr bool kFullOut = !kHalfOut && ((HM & 1) != 0 || (HM & 8) != 0);
    static_assert(!((HM & 1) && (HM & 4)) && !((HM & 2) && (HM & 8)), "a side is either half or full");
    static_assert(!kHalfIn || P % 2 == 0, "half input needs an even P");
    static_assert(!kHalfOut || (P % 2 == 0 && Q % 2 == 0), "half output needs even P and Q");
    extern __shared__ float2 smem2[];
    // Outer twiddles from a [Q][P] table: one base address per thread and constant offsets.
    // Step 1 uses it when a warp spans few rows t (column-fast loads); with row-fast loads the
    // lanes' rows are P entries apart and would collide in the shared banks, so those passes
    // index tw[t * k1]. Fused passes also read it in step 2, by column.
    constexpr bool kT2 = Op::kFusedK || !Op::kLoadLFast;
    float2* tw = smem2;                // L: tw[m] = W_L^m
    float2* T2 = tw + L;               // kT2: [Q][P], T2[t * P + k1] = W_L^(t k1)
    float2* Y = T2 + (kT2 ? L : 0);    // [L][CWp] transpose buffer
    float2* acc = Y + L * CWp;  // kSenseReduce: [A_blk][groups][Lout] running sums
    constexpr bool kPf = PF;
    static_assert(!kPf || (Prefetch<Op>::value && (kHalfIn || kFullIn) && !StageRow<Op>::value && !Op::kLoadLFast),
                  "prefetch: operators with fixed input positions and column-fast loads");
    constexpr int kPfRows = kHalfIn ? L / 2 : L;
    float2* Ks = acc + (Op::kSenseReduce ? c.A_blk * op.ngroups() * c.Lout : 0);  // kFusedK: [max_kcols][L]
    float2* Ss = Ks + (Op::kFusedK ? max_kcols<PF>() * L : 0);    // kSenseReduce: [W][Lout]
    float2* Rs = Ss + (Op::kSenseReduce ? c.W * c.Lout : 0);      // StageRow: [A_blk][L/2]
    float2* Pf = Rs + (StageRow<Op>::value ? c.A_blk * (L / 2) : 0);  // kPf: [kPfRows][kCW] samples

    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        tw[i] = c.tw[i];
        if constexpr (kT2) T2[i] = c.tw[(i / P) * (i % P)];  // (Q-1)(P-1) < L
    }
    const int tid = threadIdx.x;
    const int in_shift = ((c.in_shift % L) + L) % L;
    const int out_shift = ((c.out_shift % L) + L) % L;
    __syncthreads();

    // jobs (outer row block ab, inner column block eb) of this CTA: the first, then advance() to
    // the next. A prefetching operator without a chunk loop has one outer row (A == 1, checked by
    // the launcher) and strides over its column blocks; with a chunk loop it strides over rows and
    // takes every block of a row.
    // (no 64-bit division here: a row block ab exists while ab * A_blk < A, and the grid index
    // splits with a 32-bit division -- the launcher keeps the grid below 2^31 blocks)
    int64_t ab = 0, eb = 0;
    if constexpr (kPf && !Op::kChunkLoop) {
        ab = 0;
        eb = blockIdx.x;
    } else if constexpr (Op::kChunkLoop) {
        ab = blockIdx.x;  // kPf: rows blockIdx.x, +gridDim.x, ..., every block of a row here
        eb = 0;
    } else {
        const unsigned neb = (unsigned)c.n_eb;
        const unsigned q = blockIdx.x / neb;
        ab = q;
        eb = blockIdx.x - q * neb;
    }
    bool have = (kPf && !Op::kChunkLoop) ? eb < c.n_eb : ab * c.A_blk < c.A;
    auto advance = [&](int64_t& abj, int64_t& ebj) -> bool {
        if constexpr (kPf && !Op::kChunkLoop) {
            ebj += gridDim.x;
            return ebj < c.n_eb;
        } else if constexpr (Op::kChunkLoop) {
            if (++ebj < c.n_eb) return true;
            if (!kPf) return false;
            ebj = 0;
            abj += gridDim.x;
            return abj * c.A_blk < c.A;
        } else {
            return false;
        }
    };
    // kPf: the samples l < kPfRows of job (row a, block eb)'s kCW columns into Pf[l][col] (16-byte
    // copies of two columns where both exist and are aligned, else one column at a time; missing
    // columns are 0)
    auto prefetch = [&](int64_t a, int64_t eb) {
        if constexpr (kPf) {
            const int64_t e0p = eb * c.E_blk;
            constexpr int PC = kCW / 2;
            // a whole block of columns, rows at a fixed 16-byte multiple apart from a 16-byte
            // aligned first sample (every large pass): unconditional 16-byte copies at offsets
            // that only depend on the thread
            const float2* b0 = op.sample_ptr(a, 0, e0p);
            const int64_t rs = op.sample_ptr(a, 1, e0p) - b0;
            const bool lin = op.sample_ptr(a, 2, e0p) - b0 == 2 * rs;
            if (lin && e0p + kCW <= c.E && (((uintptr_t)b0 | (uintptr_t)(rs * (int64_t)sizeof(float2))) & 15) == 0) {
                constexpr int kThreads = Q * kCW;
#pragma unroll
                for (int i0 = 0; i0 < kPfRows * PC; i0 += kThreads) {
                    const int i = i0 + tid;
                    if (kPfRows * PC % kThreads == 0 || i < kPfRows * PC) {
                        const int l = i / PC, pc = i - l * PC;
                        cp_async16(Pf + l * kCW + 2 * pc, b0 + l * rs + 2 * pc);
                    }
                }
                cp_async_commit();
                return;
            }
#pragma unroll 1
            for (int i = tid; i < kPfRows * PC; i += blockDim.x) {
                const int l = i / PC, pc = i - l * PC;
                const int64_t e = e0p + 2 * pc;
                float2* dst = Pf + l * kCW + 2 * pc;
                const float2* src = op.sample_ptr(a, l, e);
                if (e + 1 < c.E && ((uintptr_t)src & 15) == 0) {
                    cp_async16(dst, src);
                } else {
                    if (e < c.E) cp_async8(dst, src); else dst[0] = make_float2(0.f, 0.f);
                    if (e + 1 < c.E) cp_async8(dst + 1, src + 1); else dst[1] = make_float2(0.f, 0.f);
                }
            }
            cp_async_commit();
        }
    };
    if (kPf && have) prefetch(ab * c.A_blk, eb);
    // column -> (row in the block, inner index); with one row per CTA (every large problem) the
    // runtime division by E_blk is skipped
    auto split_col = [&](int col, int& al, int& el) {
        if (c.A_blk == 1) {
            al = 0;
            el = col;
        } else {
            al = col / c.E_blk;
            el = col - al * c.E_blk;
        }
    };
    if constexpr (Op::kSenseReduce) {
        for (int i = tid; i < c.A_blk * op.ngroups() * c.Lout; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
        __syncthreads();
    }

    while (have) {
        const int64_t a0 = ab * c.A_blk;
        const int64_t e0 = eb * c.E_blk;
        int64_t ab_n = ab, eb_n = eb;
        const bool next = advance(ab_n, eb_n);
        if constexpr (kPf && !Op::kFusedK) {
            // this job's samples (the only copies in flight)
            cp_async_wait_all();
            __syncthreads();
        }
        // ---- stage the kernel columns / factor rows this chunk needs (asynchronous) -----------
        int64_t kc0 = 0;
        bool k_staged = false;
        int nk = 1;
        if constexpr (Op::kFusedK) {
            const int64_t elast = min(e0 + c.E_blk, c.E) - 1;
            kc0 = op.kcol(e0);
            nk = (int)(op.kcol(elast) - kc0 + 1);
            k_staged = (c.A_blk == 1) && nk <= max_kcols<PF>();
            if (k_staged) {
                for (int i = tid; i < nk * L; i += blockDim.x) cp_async8(Ks + i, op.kptr(kc0 + i / L) + (i % L));
                cp_async_commit();
            }
            if constexpr (kPf) {
                // this job's samples: the group before the kernel columns just issued
                if (k_staged) cp_async_wait_group<1>(); else cp_async_wait_all();
                __syncthreads();
            }
        }
        if constexpr (Op::kSenseReduce) {
            // one warp per column row: the row pointer once, then contiguous copies
            const int lane = tid & 31, nw = blockDim.x >> 5;
            for (int col = tid >> 5; col < c.W; col += nw) {
                const int al = col / c.E_blk, el = col - al * c.E_blk;
                const int64_t a = a0 + al, e = e0 + el;
                if (a >= c.A || e >= c.E) continue;
                const float2* src = op.srow(a, e);
                float2* dst = Ss + col * c.Lout;
                if ((((uintptr_t)src | (uintptr_t)dst) & 15) == 0 && (c.Lout & 1) == 0) {
                    for (int o = 2 * lane; o < c.Lout; o += 64) cp_async16(dst + o, src + o);
                } else {
                    for (int o = lane; o < c.Lout; o += 32) cp_async8(dst + o, src + o);
                }
            }
            cp_async_commit();
        }
        // ---- step 1: thread (col, t) loads x[t + Q j], j < P --------------------------------
        {
            int col, t;
            if (Op::kLoadLFast) {
                t = tid % Q;
                col = tid / Q;
            } else {
                col = tid % kCW;
                t = tid / kCW;
            }
            int al, el;
            split_col(col, al, el);
            const int64_t a = a0 + al, e = e0 + el;
            const bool colok = col < c.W && a < c.A && e < c.E;
            float2 v[P];
            bool halfzero;
            if constexpr (kHalfIn && StageRow<Op>::value) {
                // sample = column factor (own load) x row factor shared by the CTA's columns of
                // the same row: the rows go through shared memory once instead of one global load
                // per column
                constexpr int H = L / 2;
                const bool staged = op.row_shared(e0, c.E_blk);
                if (staged) {
                    for (int i = tid; i < c.A_blk * H; i += blockDim.x) {
                        const int ar = i / H, lr = i - ar * H;
                        if (a0 + ar < c.A) cp_async8(Rs + i, op.row(a0 + ar, e0) + lr);
                    }
                    cp_async_commit();
                }
#pragma unroll
                for (int j = 0; j < P; ++j)
                    v[j] = (j < P / 2 && colok) ? op.load_col(a, t + Q * j, e) : make_float2(0.f, 0.f);
                if (staged) {
                    cp_async_wait_all();
                    __syncthreads();
                    // only real columns: a padding column's al can be A_blk, past the staged rows
                    if (colok) {
#pragma unroll
                        for (int j = 0; j < P / 2; ++j) v[j] = cmul(v[j], Rs[al * H + t + Q * j]);
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < P / 2; ++j)
                        if (colok) v[j] = cmul(v[j], op.row_at(a, t + Q * j, e));
                }
                halfzero = true;
            } else if constexpr (kHalfIn && kPf) {
#pragma unroll
                for (int j = 0; j < P; ++j) v[j] = (j < P / 2) ? Pf[(t + Q * j) * kCW + col] : make_float2(0.f, 0.f);
                halfzero = true;
            } else if constexpr (kHalfIn) {
#pragma unroll
                for (int j = 0; j < P; ++j)
                    v[j] = (j < P / 2 && colok) ? op.load(a, t + Q * j, e) : make_float2(0.f, 0.f);
                halfzero = true;
            } else if constexpr (kFullIn && kPf) {
#pragma unroll
                for (int j = 0; j < P; ++j) v[j] = Pf[(t + Q * j) * kCW + col];
                halfzero = false;
            } else if constexpr (kFullIn) {
#pragma unroll
                for (int j = 0; j < P; ++j) v[j] = colok ? op.load(a, t + Q * j, e) : make_float2(0.f, 0.f);
                halfzero = false;
            } else {
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    const int pos = t + Q * j;
                    int l = pos - in_shift;
                    if (l < 0) l += L;
                    v[j] = (colok && l < c.Lin) ? op.load(a, l, e) : make_float2(0.f, 0.f);
                }
                // zero padding to 2x (Lin == L/2 at shift 0): only v[0..P/2) can be non-zero
                halfzero = (2 * c.Lin == L) && in_shift == 0;
            }
            // W_L^(t k1) = trow[k1 * tstep]
            const float2* trow = (kT2 && !Op::kLoadLFast) ? T2 + t * P : tw;
            const int tstep = (kT2 && !Op::kLoadLFast) ? 1 : t;
            if (c.inverse) {
                if (halfzero)
                    dft_reg_halfzero<P, true>(v, tw, Q);
                else
                    dft_reg<P, true>(v, tw, Q);
#pragma unroll
                for (int k1 = 1; k1 < P; ++k1) v[k1] = cmul(v[k1], tw_get<true>(trow, k1 * tstep));
            } else {
                if (halfzero)
                    dft_reg_halfzero<P, false>(v, tw, Q);
                else
                    dft_reg<P, false>(v, tw, Q);
#pragma unroll
                for (int k1 = 1; k1 < P; ++k1) v[k1] = cmul(v[k1], tw_get<false>(trow, k1 * tstep));
            }
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) Y[(k1 * Q + t) * CWp + col] = v[k1];
        }
        if (Op::kFusedK || Op::kSenseReduce) cp_async_wait_all();
        __syncthreads();
        // every thread has read Pf: the next job's samples load while this one is transformed
        if (kPf && next) prefetch(ab_n * c.A_blk, eb_n);
        // ---- step 2: thread (col, k1) runs the Q-point DFT ----------------------------------------
        const bool s2active = tid < P * kCW;
        int col2 = 0, k1 = 0;
        if (Op::kStoreLFast && !Op::kFusedK) {
            k1 = tid % P;
            col2 = tid / P;
        } else {
            col2 = tid % kCW;
            k1 = tid / kCW;
        }
        int al2, el2;
        split_col(col2, al2, el2);
        const int64_t a2 = a0 + al2, e2 = e0 + el2;
        const bool colok2 = s2active && col2 < c.W && a2 < c.A && e2 < c.E;
        float2 u[Q];
        if (s2active) {
#pragma unroll
            for (int t = 0; t < Q; ++t) u[t] = Y[(k1 * Q + t) * CWp + col2];
            if (c.inverse)
                dft_reg<Q, true>(u, tw, P);
            else
                dft_reg<Q, false>(u, tw, P);
        }
        if constexpr (Op::kFusedK) {
            // multiply by the kernel at position k1 + P k2, inverse Q-point DFT over k2. The thread
            // writes back into the transpose slots it read, so no barrier is needed here; the
            // one-CTA-per-block instances keep one as a scheduling fence (without it the compiler
            // interleaves the two halves and spills). The prefetching instances run without it
            // (3.39 against 3.51 ms for P3 at 160^3 x 32 coils, measured at 2 CTAs per SM).
            if (!PF) __syncthreads();
            if (s2active) {
                if (k_staged) {
                    // one kernel column for the whole block (the common case) needs no division
                    const float2* kc = Ks + (nk == 1 ? 0 : (int)(op.kcol(e2) - kc0)) * L;
#pragma unroll
                    for (int k2 = 0; k2 < Q; ++k2) u[k2] = colok2 ? cmul(u[k2], kc[k1 + P * k2]) : make_float2(0.f, 0.f);
                } else {
#pragma unroll
                    for (int k2 = 0; k2 < Q; ++k2) u[k2] = colok2 ? cmul(u[k2], op.kval(a2, k1 + P * k2, e2)) : make_float2(0.f, 0.f);
                }
                const float2* tcol = T2 + k1;  // W_L^(n2 k1) = tcol[n2 * P]
                if (c.inverse) {
                    dft_reg<Q, false>(u, tw, P);
#pragma unroll
                    for (int n2 = 1; n2 < Q; ++n2) u[n2] = cmul(u[n2], tw_get<false>(tcol, n2 * P));
                } else {
                    dft_reg<Q, true>(u, tw, P);
#pragma unroll
                    for (int n2 = 1; n2 < Q; ++n2) u[n2] = cmul(u[n2], tw_get<true>(tcol, n2 * P));
                }
#pragma unroll
                for (int n2 = 0; n2 < Q; ++n2) Y[(k1 * Q + n2) * CWp + col2] = u[n2];
            }
            __syncthreads();
            // thread (col, n2): inverse P-point DFT over k1 -> x[n2 + Q n1]
            {
                const int col3 = tid % kCW, n2 = tid / kCW;
                int al3, el3;
                split_col(col3, al3, el3);
                const int64_t a3 = a0 + al3, e3 = e0 + el3;
                const bool colok3 = col3 < c.W && a3 < c.A && e3 < c.E;
                float2 z[P];
#pragma unroll
                for (int q = 0; q < P; ++q) z[q] = Y[(q * Q + n2) * CWp + col3];
                if (c.inverse)
                    dft_reg<P, false>(z, tw, Q);
                else
                    dft_reg<P, true>(z, tw, Q);
                if (colok3) {
                    if constexpr (kHalfOut) {
#pragma unroll
                        for (int n1 = 0; n1 < P / 2; ++n1) op.store(a3, n2 + Q * n1, e3, z[n1]);
                    } else if constexpr (kFullOut) {
#pragma unroll
                        for (int n1 = 0; n1 < P; ++n1) op.store(a3, n2 + Q * n1, e3, z[n1]);
                    } else {
#pragma unroll
                        for (int n1 = 0; n1 < P; ++n1) {
                            const int pos = n2 + Q * n1;
                            int o = pos - out_shift;
                            if (o < 0) o += L;
                            if (o < c.Lout) op.store(a3, o, e3, z[n1]);
                        }
                    }
                }
            }
        } else if constexpr (Op::kSenseReduce) {
            // spectra into Y[o][col]; then thread o forms sum_col product(v) for its row
            __syncthreads();  // everyone has read Y
            if (s2active) {
                if constexpr (kHalfOut) {
#pragma unroll
                    for (int k2 = 0; k2 < Q / 2; ++k2) Y[(k1 + P * k2) * CWp + col2] = u[k2];
                } else if constexpr (kFullOut) {
#pragma unroll
                    for (int k2 = 0; k2 < Q; ++k2) Y[(k1 + P * k2) * CWp + col2] = u[k2];
                } else {
#pragma unroll
                    for (int k2 = 0; k2 < Q; ++k2) {
                        const int pos = k1 + P * k2;
                        int o = pos - out_shift;
                        if (o < 0) o += L;
                        if (o < c.Lout) Y[o * CWp + col2] = u[k2];
                    }
                }
            }
            __syncthreads();
            const int Lo = kHalfOut ? L / 2 : c.Lout;
            const int tot = c.A_blk * Lo;
            const int ng = op.ngroups();
            if (ng == 1) {
                // one frame: every column of the chunk adds into the row's single sum
                const int ecount = (int)min((int64_t)c.E_blk, c.E - e0);
                for (int idx = tid; idx < tot; idx += blockDim.x) {
                    const int o = idx % Lo, al = idx / Lo;
                    if (a0 + al >= c.A) continue;
                    float2 run = acc[idx];
                    const float2* yr = Y + o * CWp + al * c.E_blk;
                    const float2* sr = Ss + (al * c.E_blk) * Lo + o;
                    for (int el = 0; el < ecount; ++el) run = cadd(run, op.product_s(yr[el], sr[el * Lo]));
                    acc[idx] = run;
                }
            } else
            for (int idx = tid; idx < tot; idx += blockDim.x) {
                const int o = idx % c.Lout, al = idx / c.Lout;
                const int64_t a = a0 + al;
                if (a >= c.A) continue;
                float2 run = make_float2(0.f, 0.f);
                int64_t gcur = op.group(e0);
                for (int el = 0; el < c.E_blk; ++el) {
                    const int64_t e = e0 + el;
                    if (e >= c.E) break;
                    const int64_t gg = op.group(e);
                    if (gg != gcur) {
                        float2* dst = acc + ((int64_t)al * ng + gcur) * c.Lout + o;
                        *dst = cadd(*dst, run);
                        run = make_float2(0.f, 0.f);
                        gcur = gg;
                    }
                    const int col = al * c.E_blk + el;
                    run = cadd(run, op.product_s(Y[o * CWp + col], Ss[col * c.Lout + o]));
                }
                float2* dst = acc + ((int64_t)al * ng + gcur) * c.Lout + o;
                *dst = cadd(*dst, run);
            }
        } else {
            if (colok2) {
                if constexpr (kHalfOut) {
#pragma unroll
                    for (int k2 = 0; k2 < Q / 2; ++k2) op.store(a2, k1 + P * k2, e2, u[k2]);
                } else if constexpr (kFullOut) {
#pragma unroll
                    for (int k2 = 0; k2 < Q; ++k2) op.store(a2, k1 + P * k2, e2, u[k2]);
                } else {
#pragma unroll
                    for (int k2 = 0; k2 < Q; ++k2) {
                        const int pos = k1 + P * k2;
                        int o = pos - out_shift;
                        if (o < 0) o += L;
                        if (o < c.Lout) op.store(a2, o, e2, u[k2]);
                    }
                }
            }
        }
        if constexpr (Op::kSenseReduce) {
            // the row block's last chunk: write its sums and clear them for the next row block
            if (!next || ab_n != ab) {
                __syncthreads();
                const int ng = op.ngroups();
                const int tot = c.A_blk * ng * c.Lout;
                for (int idx = tid; idx < tot; idx += blockDim.x) {
                    const int o = idx % c.Lout, rest = idx / c.Lout, gg = rest % ng, al = rest / ng;
                    const int64_t a = a0 + al;
                    if (a < c.A) op.write_row(a, o, gg, acc[idx]);
                    acc[idx] = make_float2(0.f, 0.f);
                }
            }
        }
        if (next) __syncthreads();  // the next job rewrites Y, the staged rows and the sums
        ab = ab_n;
        eb = eb_n;
        have = next;
    }
}

// (P, Q) for the lengths with a register kernel; {0, 0} for the generic kernel.
inline void reg_split(int L, int* P, int* Q) {
    switch (L) {
        case 64: *P = 8; *Q = 8; return;
        case 128: *P = 8; *Q = 16; return;
        case 256: *P = 16; *Q = 16; return;
        case 320: *P = 16; *Q = 20; return;
        case 512: *P = 16; *Q = 32; return;
        case 640: *P = 20; *Q = 32; return;
        default: *P = 0; *Q = 0; return;
    }
}

// Op::kHalfIO (optional, default 0): the HM shape every pass of this operator has.
template <class Op, class = void>
struct HalfIO {
    static constexpr int value = 0;
};
template <class Op>
struct HalfIO<Op, std::void_t<decltype(Op::kHalfIO)>> {
    static constexpr int value = Op::kHalfIO;
};

template <int P, int Q, class Op, int HM, bool PF>
int launch_pass2_inst(const Op& op, const PassCfg& c, size_t smem, int64_t blocks, cudaStream_t s, const char* name) {
    auto kern = pass2_kernel<P, Q, Op, HM, PF>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // the staging passes want every CTA they can fit; plain passes keep the default L1 split
    if (e == cudaSuccess && (Op::kFusedK || Op::kSenseReduce || PF))
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) {
        set_error(std::string(name) + ": cudaFuncSetAttribute failed: " + cudaGetErrorString(e));
        return HB_ERR_CUDA;
    }
    int64_t grid = blocks;
    if constexpr (PF) {
        // persistent CTAs: as many as are resident at once (the shared bytes of a prefetching
        // instance depend only on its template arguments)
        static int per_sm = 0, sms = 0;
        if (per_sm == 0) {
            int dev = 0, n = 0, m = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, Q * kCW, smem) != cudaSuccess) {
                set_error(std::string(name) + ": occupancy query failed");
                return HB_ERR_CUDA;
            }
            sms = m;
            per_sm = n > 0 ? n : 1;
        }
        grid = std::min<int64_t>(blocks, (int64_t)per_sm * sms);
    }
    TimedSection ts(name, s);
    kern<<<(unsigned)grid, Q * kCW, smem, s>>>(op, c);
    return check_launch(name);
}

template <int P, int Q, class Op>
int launch_pass2_pq(const Op& op, PassCfg c, size_t extra_bytes, cudaStream_t s, const char* name) {
    constexpr int L = P * Q;
    constexpr int HM = HalfIO<Op>::value;
    const int in_sh = ((c.in_shift % L) + L) % L, out_sh = ((c.out_shift % L) + L) % L;
    const bool full_in = c.Lin == L && in_sh == 0, full_out = c.Lout == L && out_sh == 0;
    if constexpr (HM != 0) {
        const bool ok_in = (HM & 1) ? (2 * c.Lin == L && in_sh == 0) : full_in;
        const bool ok_out = (HM & 2) ? (2 * c.Lout == L && out_sh == 0) : full_out;
        if (!ok_in || !ok_out) {
            set_error(std::string(name) + ": pass shape does not match the operator's padding / crop");
            return HB_ERR_INVALID_ARG;
        }
    }
    // prefetching where the operator asks for it and a CTA holds one outer row of kCW-column blocks
    // (or the whole row); the other shapes run the plain instance
    constexpr bool kPfOp = Prefetch<Op>::value && HM != 0;
    const bool pf = kPfOp && c.A_blk == 1 && (c.E_blk == kCW || c.n_eb == 1) && (Op::kChunkLoop || c.A == 1);
    size_t smem = (size_t)((Op::kFusedK || !Op::kLoadLFast ? 2 : 1) * L + L * (kCW + 1)) * sizeof(float2) + extra_bytes;
    if (Op::kFusedK) smem += (size_t)(pf ? max_kcols<true>() : max_kcols<false>()) * L * sizeof(float2);
    if (pf) smem += (size_t)((HM & 1) ? L / 2 : L) * kCW * sizeof(float2);
    if (Op::kSenseReduce) smem += (size_t)c.W * c.Lout * sizeof(float2);
    if (StageRow<Op>::value) smem += (size_t)c.A_blk * (L / 2) * sizeof(float2);
    const int64_t n_ab = ceil_div(c.A, c.A_blk);
    const int64_t blocks = Op::kChunkLoop ? n_ab : n_ab * c.n_eb;
    if (blocks <= 0) return HB_OK;
    if (blocks > 0x7fffffffLL) {
        set_error(std::string(name) + ": grid too large");
        return HB_ERR_INVALID_ARG;
    }
    if constexpr (HM != 0) {
        if constexpr (kPfOp) {
            if (pf) return launch_pass2_inst<P, Q, Op, HM, true>(op, c, smem, blocks, s, name);
        }
        return launch_pass2_inst<P, Q, Op, HM, false>(op, c, smem, blocks, s, name);
    } else {
        // no fixed shape: a side that spans all L positions unshifted gets compile-time positions
        if (full_in && full_out) return launch_pass2_inst<P, Q, Op, 12, false>(op, c, smem, blocks, s, name);
        if (full_in) return launch_pass2_inst<P, Q, Op, 4, false>(op, c, smem, blocks, s, name);
        if (full_out) return launch_pass2_inst<P, Q, Op, 8, false>(op, c, smem, blocks, s, name);
        return launch_pass2_inst<P, Q, Op, 0, false>(op, c, smem, blocks, s, name);
    }
}

// Runs the register kernel when L has one, otherwise the generic shared-memory kernel.
// `extra_per_row` is the kSenseReduce accumulator size per outer row (bytes).
template <class Op>
int launch_fft_pass(const Op& op, const FftLen& f, int64_t A, int64_t E, int Lin, int in_shift, int Lout,
                    int out_shift, int inverse, size_t extra_per_row, cudaStream_t s, const char* name) {
    int P, Q;
    reg_split(f.L, &P, &Q);
    PassCfg c;
    if (P > 0) {
        pass_setup(&c, f, A, E, Lin, in_shift, Lout, out_shift, inverse, kCW);
        const size_t extra = extra_per_row * c.A_blk;
        switch (f.L) {
            case 64: return launch_pass2_pq<8, 8>(op, c, extra, s, name);
            case 128: return launch_pass2_pq<8, 16>(op, c, extra, s, name);
            case 256: return launch_pass2_pq<16, 16>(op, c, extra, s, name);
            case 320: return launch_pass2_pq<16, 20>(op, c, extra, s, name);
            case 512: return launch_pass2_pq<16, 32>(op, c, extra, s, name);
            case 640: return launch_pass2_pq<20, 32>(op, c, extra, s, name);
        }
    }
    pass_setup(&c, f, A, E, Lin, in_shift, Lout, out_shift, inverse);
    return launch_pass(op, c, extra_per_row * c.A_blk, s, name);
}

#endif  // __CUDACC__

}  // namespace hb
