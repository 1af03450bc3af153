// NUFFT type 1 / type 2 on B200: bin sort, tile-owned spreading, point-gather interpolation,
// and the pruned FFT passes with the deapodisation fused into the first / last pass.
//
// Algorithm (the restated cufinufft pipeline, cpp/corelib/lib/fft/nufft.cppm:205-250 calls):
//   type 1: g = spread(c)  ->  G = FFT_sign(g) over the fine grid  ->  f[k] = G[k mod nf]/phihat(k)
//   type 2: G[k mod nf] = f[k]/phihat(k)  ->  g = FFT_sign(G)  ->  c_j = interp(g, x_j)
// with phi the Kaiser-Bessel kernel and phihat its Fourier transform.
#include <algorithm>
#include <cmath>
#include <vector>

#include "nufft.cuh"
#include "ops.cuh"

namespace hb {

// ---------------------------------------------------------------------------------------------
// small helpers

static bool smooth235(int n) {
    for (int r : {2, 3, 5})
        while (n % r == 0 && n > 1) n /= r;
    return n == 1;
}

static int fine_size(int64_t N, double sigma, int w, int T) {
    if (N <= 1) return 1;
    int64_t lo = (int64_t)std::ceil(sigma * (double)N - 1e-9);
    lo = std::max<int64_t>(lo, 2 * w);
    lo = std::max<int64_t>(lo, T);
    for (int64_t n = lo;; ++n)
        if (n % T == 0 && smooth235((int)n)) return (int)n;
}

static int pow2ceil(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Coil chunk (power of two, <= 32) a spread CTA accumulates at once.
static int spread_cc(const GridGeom& g) {
    const int cells = g.T[0] * g.T[1] * g.T[2];
    int cmax = 32;
    while (cmax > 1 && (size_t)cells * cmax * 8 > 131072) cmax >>= 1;
    return std::min(pow2ceil(g.C), cmax);
}

// ---------------------------------------------------------------------------------------------
// setpts kernels

struct FoldArgs {
    const float* c[3];  // caller coordinate per internal axis (nullptr on unit axes)
    float* u[3];        // unsorted fine coordinates
    int* binid;
    int* rank;
    int* count;
    int* err;
    int nf[3], T[3], nb[3];
    float scale[3];
    float hw;
    int64_t M;
    const int* foff;  // frame point offsets (nullptr: one frame)
    int nfr;
    int ntf;          // bins per frame
};

__device__ __forceinline__ float fold_fine(float x, float scale, int nf) {
    float u = __fmul_rn(x, scale);
    const float fnf = (float)nf;
    const float q = floorf(__fdiv_rn(u, fnf));
    u = __fsub_rn(u, __fmul_rn(q, fnf));
    if (u < 0.f) u = __fadd_rn(u, fnf);
    if (u >= fnf) u = __fsub_rn(u, fnf);
    return u;
}

__device__ __forceinline__ int first_cell(float u, float hw, int nf) {
    int i0 = (int)ceilf(__fsub_rn(u, hw));
    if (i0 < 0) i0 += nf;
    if (i0 >= nf) i0 -= nf;
    return i0;
}

__global__ void k_fold_bin(const FoldArgs a) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= a.M) return;
    int b[3];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        if (a.c[ax] == nullptr) {
            b[ax] = 0;
            continue;
        }
        float x = a.c[ax][j];
        if (!isfinite(x)) {
            atomicExch(a.err, 1);
            x = 0.f;
        }
        const float u = fold_fine(x, a.scale[ax], a.nf[ax]);
        a.u[ax][j] = u;
        b[ax] = first_cell(u, a.hw, a.nf[ax]) / a.T[ax];
    }
    const int bin = (b[0] * a.nb[1] + b[1]) * a.nb[2] + b[2] + frame_of_point(a.foff, a.nfr, j) * a.ntf;
    a.binid[j] = bin;
    a.rank[j] = atomicAdd(&a.count[bin], 1);
}

__global__ void k_scatter_sorted(const float* u0, const float* u1, const float* u2, const int* binid,
                                 const int* rank, const int* bin_start, float* s0, float* s1, float* s2,
                                 int* perm, int64_t M) {
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= M) return;
    const int s = bin_start[binid[j]] + rank[j];
    perm[s] = (int)j;
    if (s0) s0[s] = u0[j];
    if (s1) s1[s] = u1[j];
    if (s2) s2[s] = u2[j];
}

// ---- exclusive scan of ints (n + 1 outputs, out[n] = total) -------------------------------------
constexpr int kScanBlock = 1024;

__device__ __forceinline__ int block_excl_scan(int v, int* warp_sums, int& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int ws = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, ws, o);
            if (lane >= o) ws += y;
        }
        warp_sums[lane] = ws;  // inclusive over warps
    }
    __syncthreads();
    const int warp_off = wid > 0 ? warp_sums[wid - 1] : 0;
    total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warp_off + x - v;
}

__global__ void k_scan_blocks(const int* in, int* out, int* sums, int64_t n) {
    __shared__ int ws[32];
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int total;
    const int ex = block_excl_scan(v, ws, total);
    if (i < n) out[i] = ex;
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(int* sums, int64_t nblocks, int* total_out) {
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nblocks; base += kScanBlock) {
        const int64_t i = base + threadIdx.x;
        const int v = i < nblocks ? sums[i] : 0;
        int total;
        const int ex = block_excl_scan(v, ws, total);
        if (i < nblocks) sums[i] = ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

__global__ void k_scan_add(int* out, const int* sums, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) out[i] += sums[blockIdx.x];
}

int exclusive_scan_int(const int* in, int* out, int64_t n, cudaStream_t s, int* sums) {
    const int64_t nb = ceil_div(std::max<int64_t>(n, 1), kScanBlock);
    const bool own = sums == nullptr;
    if (own) HB_CUDA(cudaMallocAsync(&sums, sizeof(int) * nb, s));
    k_scan_blocks<<<(unsigned)nb, kScanBlock, 0, s>>>(in, out, sums, n);
    k_scan_sums<<<1, kScanBlock, 0, s>>>(sums, nb, out + n);
    k_scan_add<<<(unsigned)nb, kScanBlock, 0, s>>>(out, sums, n);
    int st = check_launch("exclusive_scan_int");
    if (own) HB_CUDA(cudaFreeAsync(sums, s));
    return st;
}

// ---- spread work list --------------------------------------------------------------------------
struct TileNbr {
    int nb[3];
    int nfr;  // frames
    int ntf;  // tiles per frame
};

// Visits the (up to 8) bins whose points can reach tile (tz, ty, tx): along each axis with more
// than one bin, the tile's own bin and the one before it (a footprint spans at most 2 tiles).
template <class F>
__device__ __forceinline__ void for_each_nbr_bin(const int* nb, int tz, int ty, int tx, F&& f) {
    const int nz = nb[0] > 1 ? 2 : 1, ny = nb[1] > 1 ? 2 : 1, nx = nb[2] > 1 ? 2 : 1;
    for (int dz = 0; dz < nz; ++dz) {
        const int bz = (tz - dz + nb[0]) % nb[0];
        for (int dy = 0; dy < ny; ++dy) {
            const int by = (ty - dy + nb[1]) % nb[1];
            for (int dx = 0; dx < nx; ++dx) {
                const int bx = (tx - dx + nb[2]) % nb[2];
                f((bz * nb[1] + by) * nb[2] + bx);
            }
        }
    }
}

__global__ void k_tile_extra_count(const int* bin_start, TileNbr t, int64_t ntiles, int maxp, int* extra_cnt) {
    const int64_t tile = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    const int64_t fr = t.nfr > 1 ? tile / t.ntf : 0, lt = tile - fr * t.ntf, fb = fr * t.ntf;
    const int tx = (int)(lt % t.nb[2]), ty = (int)((lt / t.nb[2]) % t.nb[1]), tz = (int)(lt / ((int64_t)t.nb[2] * t.nb[1]));
    int64_t total = 0;
    for_each_nbr_bin(t.nb, tz, ty, tx, [&](int bin) { total += bin_start[fb + bin + 1] - bin_start[fb + bin]; });
    const int64_t nsub = total > 0 ? (total + maxp - 1) / maxp : 1;
    extra_cnt[tile] = (int)(nsub - 1);
}

__global__ void k_tile_extra_fill(const int* extra_cnt, const int* extra_off, int64_t ntiles, int4* extra) {
    const int64_t tile = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    const int n = extra_cnt[tile], off = extra_off[tile];
    for (int c = 0; c < n; ++c) extra[off + c] = make_int4((int)tile, c + 1, n, off);
}

// Adds the extra subproblems' partial tiles into the grid: CTA blockIdx.x takes entry e = extra[b]
// and, for its share (chunk e.y - 1 of e.z) of the tile's cells x transforms, adds the tile's e.z
// scratch slots e.w .. e.w + e.z - 1 in slot order to the grid value chunk 0 stored. Deterministic:
// no atomics, a fixed sum order.
__global__ void __launch_bounds__(256) k_spread_extra_reduce(const GridArgs a) {
    const GridGeom& g = a.g;
    const int4 e = a.extra[blockIdx.x];
    int tile = e.x;
    const int fr = split_frame_tile(g, tile);
    float2* const gridf = a.grid + fr * g.fgrid;
    const int T0 = g.T[0], T1 = g.T[1], T2 = g.T[2];
    const int tx = tile % g.nb[2], ty = (tile / g.nb[2]) % g.nb[1], tz = tile / (g.nb[2] * g.nb[1]);
    const int org0 = tz * T0, org1 = ty * T1, org2 = tx * T2;
    const int64_t E = (int64_t)T0 * T1 * T2 * g.C;
    const int q = e.y - 1, n = e.z;
    const int64_t i0 = q * E / n, i1 = (q + 1) * E / n;
    const float2* src = a.extra_scratch + (int64_t)e.w * E;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        float2 sum = src[i];
        for (int s = 1; s < n; ++s) {
            const float2 v = src[(int64_t)s * E + i];
            sum.x += v.x;
            sum.y += v.y;
        }
        const int64_t cell = i / g.C;
        const int c = (int)(i - cell * g.C);
        const int x = (int)(cell % T2), y = (int)((cell / T2) % T1), z = (int)(cell / ((int64_t)T2 * T1));
        float2* dst = gridf + (((int64_t)(org0 + z) * g.nf[1] + (org1 + y)) * g.nf[2] + org2 + x) * g.C + c;
        const float2 v0 = *dst;
        *dst = make_float2(v0.x + sum.x, v0.y + sum.y);
    }
}

// Dense tiles (more candidates than a subproblem holds) for the lanes-on-transforms kernel: a
// tile of `total` candidates is spread in nsub = ceil(total / maxp) parts, each into its own
// scratch slot. cnt[tile] = nsub for dense tiles, 0 otherwise; the fill writes one work entry
// {tile, part, nsub, first slot} per part at the scanned offsets (slots are numbered like entries).
__global__ void k_tile_parts_count(const int* bin_start, TileNbr t, int64_t ntiles, int maxp, int* cnt) {
    const int64_t tile = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    const int64_t fr = t.nfr > 1 ? tile / t.ntf : 0, lt = tile - fr * t.ntf, fb = fr * t.ntf;
    const int tx = (int)(lt % t.nb[2]), ty = (int)((lt / t.nb[2]) % t.nb[1]), tz = (int)(lt / ((int64_t)t.nb[2] * t.nb[1]));
    int64_t total = 0;
    for_each_nbr_bin(t.nb, tz, ty, tx, [&](int bin) { total += bin_start[fb + bin + 1] - bin_start[fb + bin]; });
    cnt[tile] = total > maxp ? (int)((total + maxp - 1) / maxp) : 0;
}

__global__ void k_tile_parts_fill(const int* cnt, const int* off, int64_t ntiles, int4* parts) {
    const int64_t tile = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (tile >= ntiles) return;
    const int n = cnt[tile], o = off[tile];
    for (int q = 0; q < n; ++q) parts[o + q] = make_int4((int)tile, q, n, o);
}

// ---------------------------------------------------------------------------------------------
// execute kernels

// xin[j][c] = in[c][j]: the caller's [C][M] values with the transforms interleaved, in the
// caller's point order (a tiled transpose, coalesced on both sides). Spreading reads the values of
// sorted point s as the contiguous row xin[perm[s]].
__global__ void k_interleave_in(const float2* __restrict__ in, float2* __restrict__ xin, int64_t M, int C) {
    __shared__ float2 tile[32][33];
    const int64_t j0 = (int64_t)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r;
        const int64_t j = j0 + threadIdx.x;
        if (c < C && j < M) tile[r][threadIdx.x] = in[(int64_t)c * M + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int64_t j = j0 + r;
        const int c = c0 + threadIdx.x;
        if (c < C && j < M) xin[j * C + c] = tile[threadIdx.x][r];
    }
}

constexpr int kGridThreads = 256;
constexpr int kGridWarps = kGridThreads / 32;
constexpr int kSlotFloats = 3 * kMaxWidth;

// Per point: fine coordinate -> first cell (wrapped) and the tap weights of each axis. The
// lanes of a slot share the weight evaluation; weights land in wts[axis*kMaxWidth + d].
__device__ __forceinline__ void point_setup(const GridArgs& a, const float* coef, int64_t s, bool valid, int lane_in_slot,
                                            int slot_lanes, float* wts, int* i0) {
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int w = a.g.wa[ax];
        if (w == 1) {
            i0[ax] = 0;
            if (lane_in_slot == 0) wts[ax * kMaxWidth] = 1.f;
            continue;
        }
        const float u = valid ? a.su[ax][s] : 0.f;
        const float hw = a.kb.hw;
        const float v = __fsub_rn(u, hw);
        const int ic = (int)ceilf(v);
        const float t = __fsub_rn((float)ic, v);
        const float sarg = fmaf(2.f, t, -1.f);
        int iw = ic;
        const int nf = a.g.nf[ax];
        if (iw < 0) iw += nf;
        if (iw >= nf) iw -= nf;
        i0[ax] = iw;
        for (int d = lane_in_slot; d < w; d += slot_lanes) wts[ax * kMaxWidth + d] = kb_tap(coef, a.kb.deg, d, sarg);
    }
}

// Type-1 spreading. One CTA owns one tile of the fine grid and produces its cells exactly once
// (plain stores for chunk 0 of every tile, atomic adds for the extra chunks of dense tiles): no
// halo, no zero fill, no global atomics outside dense tiles. Candidate points come from the
// tile's bin and its lower neighbours; each point is clipped to the tile. Lanes of a warp map
// to (point slot, transform) so one point's weights serve CC transforms at once; accumulation is
// in shared memory.
template <int CC>
__global__ void __launch_bounds__(kGridThreads) k_spread(const GridArgs a, int extra_mode) {
    extern __shared__ float sm[];
    const GridGeom& g = a.g;
    const int T0 = g.T[0], T1 = g.T[1], T2 = g.T[2];
    const int cells = T0 * T1 * T2;
    float* acc_re = sm;
    float* acc_im = acc_re + cells * CC;
    float* coef = acc_im + cells * CC;
    float* wts_all = coef + kCoefFloats;
    constexpr int NS = 32 / CC;
    __shared__ int s_start[8], s_pref[9], s_nbin;

    int tile, chunk;
    if (extra_mode) {
        const int4 e = a.extra[blockIdx.x];
        tile = e.x;
        chunk = e.y;
    } else {
        tile = blockIdx.x;
        chunk = 0;
    }
    const int fr = split_frame_tile(g, tile);
    const int fbin = fr * (int)g.ntf;
    float2* const gridf = a.grid + fr * g.fgrid;
    // an extra subproblem writes its partial tile [cell][C] to its scratch slot
    float2* const xslot = extra_mode ? a.extra_scratch + (int64_t)blockIdx.x * cells * g.C : nullptr;
    const int tx = tile % g.nb[2], ty = (tile / g.nb[2]) % g.nb[1], tz = tile / (g.nb[2] * g.nb[1]);
    const int o0 = tz * T0, o1 = ty * T1, o2 = tx * T2;

    for (int i = threadIdx.x; i < kCoefFloats; i += blockDim.x) coef[i] = (&a.kb.coef[0][0])[i];
    if (threadIdx.x == 0) {
        int n = 0, acc = 0;
        for_each_nbr_bin(g.nb, tz, ty, tx, [&](int bin) {
            const int st = a.bin_start[fbin + bin];
            s_start[n] = st;
            s_pref[n] = acc;
            acc += a.bin_start[fbin + bin + 1] - st;
            ++n;
        });
        s_pref[n] = acc;
        s_nbin = n;
    }
    __syncthreads();
    const int total = s_pref[s_nbin];
    const int k_begin = chunk * a.maxp;
    const int k_end = min(total, k_begin + a.maxp);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / CC, coil = lane % CC;
    float* wts = wts_all + (warp * NS + slot) * kSlotFloats;

    for (int cc0 = 0; cc0 < g.C; cc0 += CC) {
        for (int i = threadIdx.x; i < cells * CC; i += blockDim.x) {
            acc_re[i] = 0.f;
            acc_im[i] = 0.f;
        }
        __syncthreads();
        const bool coil_ok = (cc0 + coil) < g.C;
        for (int base = k_begin + warp * NS; base < k_end; base += kGridWarps * NS) {
            const int k = base + slot;
            const bool valid = k < k_end;
            int64_t s = 0;
            if (valid) {
                int b = 0;
                while (b + 1 < s_nbin && s_pref[b + 1] <= k) ++b;
                s = s_start[b] + (k - s_pref[b]);
            }
            int i0[3];
            point_setup(a, coef, s, valid, coil, CC, wts, i0);
            __syncwarp();
            if (valid && coil_ok) {
                const float2 v = a.inT[(int64_t)a.perm[s] * g.C + cc0 + coil];
                int r0 = i0[0] - o0, r1 = i0[1] - o1, r2 = i0[2] - o2;
                if (r0 < 0) r0 += g.nf[0];
                if (r1 < 0) r1 += g.nf[1];
                if (r2 < 0) r2 += g.nf[2];
                for (int dz = 0; dz < g.wa[0]; ++dz) {
                    int cz = r0 + dz;
                    if (cz >= g.nf[0]) cz -= g.nf[0];
                    if (cz >= T0) continue;
                    const float wz = wts[dz];
                    for (int dy = 0; dy < g.wa[1]; ++dy) {
                        int cy = r1 + dy;
                        if (cy >= g.nf[1]) cy -= g.nf[1];
                        if (cy >= T1) continue;
                        const float wzy = wz * wts[kMaxWidth + dy];
                        const int rowc = (cz * T1 + cy) * T2;
                        for (int dx = 0; dx < g.wa[2]; ++dx) {
                            int cx = r2 + dx;
                            if (cx >= g.nf[2]) cx -= g.nf[2];
                            if (cx >= T2) continue;
                            const float wgt = wzy * wts[2 * kMaxWidth + dx];
                            const int ci = (rowc + cx) * CC + coil;
                            atomicAdd(&acc_re[ci], wgt * v.x);
                            atomicAdd(&acc_im[ci], wgt * v.y);
                        }
                    }
                }
            }
            __syncwarp();
        }
        __syncthreads();
        for (int i = threadIdx.x; i < cells * CC; i += blockDim.x) {
            const int c = i % CC, cell = i / CC;
            if (cc0 + c >= g.C) continue;
            const int cx = cell % T2, cy = (cell / T2) % T1, cz = cell / (T1 * T2);
            const int64_t gi = ((int64_t)(o0 + cz) * g.nf[1] + (o1 + cy)) * g.nf[2] + (o2 + cx);
            float2* dst = extra_mode ? xslot + (int64_t)cell * g.C + cc0 + c : gridf + gi * g.C + cc0 + c;
            *dst = make_float2(acc_re[i], acc_im[i]);
        }
        __syncthreads();
    }
}

// ---- output-stationary spreading ------------------------------------------------------------
// One CTA owns one tile (one thread per cell) and keeps CC transforms of its cell in registers.
// Candidate points pass through shared memory in chunks of kSpreadChunk, double-buffered: while
// the CTA accumulates chunk i, its threads stage chunk i+1 -- one thread per (point, axis)
// evaluates the w tap weights, the point's first cell relative to the tile and the warp blocks
// its footprint meets along that axis, and the CC values arrive by cp.async. One barrier per
// chunk. A warp owns a compact block of 32 cells (2x4x4 in 3-D, 4x8 in 2-D by default) and
// skips a point with one vote when the footprint misses the block. The finished tile leaves
// through shared memory, so each warp store covers whole runs of coils of the interleaved grid.
// No atomics except for the extra chunks of dense tiles, which add their partial tile.
constexpr int kSpreadChunk = 128;
constexpr int kSpreadThreads = 512;

struct SpreadTileShape {
    int bz, by, bx;  // warp block
};

// Shared-memory plan (in floats) after the kernel-polynomial copy: two staging buffers
// {values float2[chunk][CC], taps float[chunk][3][kMaxWidth], first cells int[chunk] (3 bytes,
// +16 biased), block masks uint2[chunk] (3 x 16 bits)}, reused at the end as per-warp output
// tiles float2[32 cells][H + 1].
template <int CC>
struct SpreadSmem {
    static constexpr int kVal = kSpreadChunk * CC * 2;
    static constexpr int kW = kSpreadChunk * 3 * kMaxWidth;
    static constexpr int kBuf = kVal + kW + 3 * kSpreadChunk;
    static constexpr int kHalf = CC < 16 ? CC : 16;  // coils per output round
    static constexpr int kOut = (kSpreadThreads / 32) * 32 * (kHalf + 1) * 2;
    static constexpr int kFloats = kCoefFloats + (2 * kBuf > kOut ? 2 * kBuf : kOut);
};

// Bits lo/bs .. hi/bs (inclusive) of a block mask; bs = 1 << lbs.
__device__ __forceinline__ unsigned block_bits(int lo, int hi, int lbs) {
    return (2u << (hi >> lbs)) - (1u << (lo >> lbs));
}

template <int CC>
__global__ void __launch_bounds__(kSpreadThreads, (CC <= 8) ? 2 : 1)
    k_spread_reg(const GridArgs a, int extra_mode, SpreadTileShape wb) {
    using SM = SpreadSmem<CC>;
    extern __shared__ float4 sm_f4[];
    float* coef = reinterpret_cast<float*>(sm_f4);
    float* region = coef + kCoefFloats;
    __shared__ int s_start[8], s_pref[9], s_nbin;
    const GridGeom& g = a.g;
    const int T0 = g.T[0], T1 = g.T[1], T2 = g.T[2];

    int tile, chunk;
    if (extra_mode) {
        const int4 e = a.extra[blockIdx.x];
        tile = e.x;
        chunk = e.y;
    } else {
        tile = blockIdx.x;
        chunk = 0;
    }
    const int fr = split_frame_tile(g, tile);
    const int fbin = fr * (int)g.ntf;
    float2* const gridf = a.grid + fr * g.fgrid;
    // an extra subproblem writes its partial tile [cell][C] to its scratch slot
    float2* const slot = extra_mode ? a.extra_scratch + (int64_t)blockIdx.x * (T0 * T1 * T2) * g.C : nullptr;
    const int tx = tile % g.nb[2], ty = (tile / g.nb[2]) % g.nb[1], tz = tile / (g.nb[2] * g.nb[1]);
    const int org0 = tz * T0, org1 = ty * T1, org2 = tx * T2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // this thread's cell and its warp's block
    // the block edges divide the power-of-two tile edges, so they are powers of two: shifts
    const int lbz = __ffs(wb.bz) - 1, lby = __ffs(wb.by) - 1, lbx = __ffs(wb.bx) - 1;
    const int nbx = T2 >> lbx, nby = T1 >> lby;
    const int bxi = warp % nbx, byi = (warp / nbx) % nby, bzi = warp / (nbx * nby);
    const int cz = (bzi << lbz) + (lane >> (lby + lbx));
    const int cy = (byi << lby) + ((lane >> lbx) & (wb.by - 1));
    const int cx = (bxi << lbx) + (lane & (wb.bx - 1));
    const int czb = cz + 16, cyb = cy + 16, cxb = cx + 16;
    const unsigned mz = 1u << bzi, my = 1u << (16 + byi), mx = 1u << bxi;
    const int w0 = g.wa[0], w1 = g.wa[1], w2 = g.wa[2];
    const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];

    for (int i = tid; i < kCoefFloats; i += kSpreadThreads) coef[i] = (&a.kb.coef[0][0])[i];
    // the (up to 8) bins whose points reach the tile, in for_each_nbr_bin order: one lane each,
    // offsets by a shuffle scan
    if (warp == 0) {
        const int nz = g.nb[0] > 1 ? 2 : 1, ny = g.nb[1] > 1 ? 2 : 1, nx = g.nb[2] > 1 ? 2 : 1;
        const int nbn = nz * ny * nx;
        int st = 0, cnt = 0;
        if (lane < nbn) {
            const int dx = lane % nx, dy = (lane / nx) % ny, dz = lane / (nx * ny);
            const int bz = (tz - dz + g.nb[0]) % g.nb[0], by = (ty - dy + g.nb[1]) % g.nb[1];
            const int bx = (tx - dx + g.nb[2]) % g.nb[2];
            const int bin = (bz * g.nb[1] + by) * g.nb[2] + bx;
            st = a.bin_start[fbin + bin];
            cnt = a.bin_start[fbin + bin + 1] - st;
        }
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < nbn) {
            s_start[lane] = st;
            s_pref[lane] = incl - cnt;
        }
        if (lane == nbn - 1) {
            s_pref[nbn] = incl;
            s_nbin = nbn;
        }
    }
    __syncthreads();
    const int nbin = s_nbin;
    const int total = s_pref[nbin];
    if (total == 0) {
        // no point reaches the tile: zero its cells with 16-byte stores (rows of T2 cells x C
        // transforms are contiguous and 16-byte aligned: T2 and the tile origin are multiples of 8)
        if (!extra_mode) {
            const int rowf4 = (T2 * g.C) >> 1;
            const int nrow = T0 * T1;
            for (int i = tid; i < nrow * rowf4; i += kSpreadThreads) {
                const int r = i / rowf4, c4 = i - r * rowf4;
                const int zz = r / T1, yy = r - zz * T1;
                float4* dst = reinterpret_cast<float4*>(
                    gridf + (((int64_t)(org0 + zz) * nf1 + (org1 + yy)) * nf2 + org2) * g.C);
                dst[c4] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        return;
    }
    const int k_begin = chunk * a.maxp;
    const int k_end = min(total, k_begin + a.maxp);
    const float hw = a.kb.hw;
    const bool vec = (g.C % 2) == 0;

    // Candidate k of this tile -> sorted point index. The candidates are visited interleaved:
    // the list (bins concatenated) is cut into 8 near-equal segments and k takes segment k % 8,
    // position k / 8, so every chunk samples all of the tile's bins and the warps' shares of a
    // chunk stay even (a chunk drawn from one lower-neighbour bin would only reach the warps at
    // the tile's low faces).
    const int seg_len = total >> 3, seg_rem = total & 7;
    auto sorted_index = [&](int k0) -> int {
        const int sg = k0 & 7;
        const int k = sg * seg_len + min(sg, seg_rem) + (k0 >> 3);
        int b = 0;
#pragma unroll
        for (int j = 1; j < 8; ++j) b += (j < nbin && s_pref[j] <= k) ? 1 : 0;
        return s_start[b] + (k - s_pref[b]);
    };

    auto stage = [&](int base, int cc0, float* buf) {
        const int n = min(kSpreadChunk, k_end - base);
        float2* bval = reinterpret_cast<float2*>(buf);
        float* bwt = buf + SM::kVal;
        unsigned char* brel = reinterpret_cast<unsigned char*>(bwt + SM::kW);
        unsigned short* bam = reinterpret_cast<unsigned short*>(brel + 4 * kSpreadChunk);
        // the CC values of each point (asynchronous)
        if constexpr (CC == 1) {
            for (int q = tid; q < n; q += kSpreadThreads) {
                if (cc0 < g.C) cp_async8(bval + q, a.inT + (int64_t)a.perm[sorted_index(base + q)] * g.C + cc0);
            }
        } else {
            constexpr int CP = CC / 2;
            for (int i = tid; i < n * CP; i += kSpreadThreads) {
                const int q = i / CP, c = 2 * (i % CP);
                float2* dst = bval + q * CC + c;
                const int cg = cc0 + c;
                const float2* src = a.inT + (int64_t)a.perm[sorted_index(base + q)] * g.C + cg;
                if (vec && cg < g.C) {
                    cp_async16(dst, src);
                } else {
                    if (cg < g.C) cp_async8(dst, src); else dst[0] = make_float2(0.f, 0.f);
                    if (cg + 1 < g.C) cp_async8(dst + 1, src + 1); else dst[1] = make_float2(0.f, 0.f);
                }
            }
        }
        // per (point, axis): tap weights, first cell relative to the tile, warp blocks met
        for (int i = tid; i < 3 * n; i += kSpreadThreads) {
            const int q = i / 3, ax = i - 3 * q;
            const int w = g.wa[ax];
            float* wt = bwt + (q * 3 + ax) * kMaxWidth;
            int relb = 16;
            unsigned am = 1u;
            if (w > 1) {
                const float u = a.su[ax][sorted_index(base + q)];
                const float v = __fsub_rn(u, hw);
                const int ic = (int)ceilf(v);
                const float sarg = fmaf(2.f, __fsub_rn((float)ic, v), -1.f);
                const int nf = g.nf[ax], T = g.T[ax];
                const int lbs = ax == 0 ? lbz : (ax == 1 ? lby : lbx);
                int iw = ic;
                if (iw < 0) iw += nf;
                if (iw >= nf) iw -= nf;
                int rel = iw - (ax == 0 ? org0 : (ax == 1 ? org1 : org2));
                if (rel < 0) rel += nf;
                for (int d = 0; d < w; ++d) wt[d] = kb_tap(coef, a.kb.deg, d, sarg);
                // footprint cells rel .. rel+w-1 (mod nf) inside [0, T)
                am = 0u;
                if (rel < T) {
                    am |= block_bits(rel, min(rel + w - 1, T - 1), lbs);
                    relb = rel + 16;
                } else {
                    relb = max(rel - nf + 16, 0);  // a footprint reaching the tile starts >= -(w-1)
                }
                if (rel + w - 1 >= nf) am |= block_bits(0, min(rel + w - 1 - nf, T - 1), lbs);
            } else {
                wt[0] = 1.f;
            }
            brel[q * 4 + ax] = (unsigned char)relb;
            bam[q * 4 + ax] = (unsigned short)am;
        }
    };

    for (int cc0 = 0; cc0 < g.C; cc0 += CC) {
        float ar[CC], ai[CC];
#pragma unroll
        for (int c = 0; c < CC; ++c) ar[c] = ai[c] = 0.f;
        const int nch = (k_end - k_begin + kSpreadChunk - 1) / kSpreadChunk;
        if (nch > 0) stage(k_begin, cc0, region);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        for (int it = 0; it < nch; ++it) {
            const int base = k_begin + it * kSpreadChunk;
            if (it + 1 < nch) stage(base + kSpreadChunk, cc0, region + ((it + 1) & 1) * SM::kBuf);
            cp_async_commit();
            // accumulate chunk it: each warp visits the points whose footprint meets its block
            {
                const int n = min(kSpreadChunk, k_end - base);
                const float* buf = region + (it & 1) * SM::kBuf;
                const float2* bval = reinterpret_cast<const float2*>(buf);
                const float* bwt = buf + SM::kVal;
                const int* brel = reinterpret_cast<const int*>(bwt + SM::kW);
                const uint2* bam = reinterpret_cast<const uint2*>(brel + kSpreadChunk);
                for (int q0 = 0; q0 < n; q0 += 32) {
                    const int qq = q0 + lane;
                    bool hit = false;
                    if (qq < n) {
                        const uint2 m = bam[qq];
                        hit = (m.x & mz) && (m.x & my) && (m.y & mx);
                    }
                    unsigned bits = __ballot_sync(0xffffffffu, hit);
                    while (bits) {
                        const int q = q0 + __ffs(bits) - 1;
                        bits &= bits - 1;
                        const int pk = brel[q];
                        int dz = czb - (pk & 0xff);
                        int dy = cyb - ((pk >> 8) & 0xff);
                        int dx = cxb - ((pk >> 16) & 0xff);
                        if (dz < 0) dz += nf0;
                        if (dy < 0) dy += nf1;
                        if (dx < 0) dx += nf2;
                        // branch-free: outside the footprint read tap 0 and select weight 0
                        const bool in = dz < w0 && dy < w1 && dx < w2;
                        const float* wq = bwt + q * 3 * kMaxWidth;
                        const float wp = wq[in ? dz : 0] * wq[kMaxWidth + (in ? dy : 0)] * wq[2 * kMaxWidth + (in ? dx : 0)];
                        const float wgt = in ? wp : 0.f;
                        const float2* vq = bval + q * CC;
                        if constexpr (CC == 1) {
                            const float2 v = vq[0];
                            ar[0] = fmaf(wgt, v.x, ar[0]);
                            ai[0] = fmaf(wgt, v.y, ai[0]);
                        } else {
#pragma unroll
                            for (int c = 0; c < CC; c += 2) {
                                const float4 v = *reinterpret_cast<const float4*>(vq + c);
                                ar[c] = fmaf(wgt, v.x, ar[c]);
                                ai[c] = fmaf(wgt, v.y, ai[c]);
                                ar[c + 1] = fmaf(wgt, v.z, ar[c + 1]);
                                ai[c + 1] = fmaf(wgt, v.w, ai[c + 1]);
                            }
                        }
                    }
                }
            }
            cp_async_wait_all();
            __syncthreads();
        }
        // write the tile: each warp transposes its 32 cells x H coils through shared memory
        {
            constexpr int H = SM::kHalf;
            constexpr int CPR = 32 / H;  // cells per store round
            float2* ow = reinterpret_cast<float2*>(region) + warp * 32 * (H + 1);
#pragma unroll
            for (int h0 = 0; h0 < CC; h0 += H) {
#pragma unroll
                for (int c = 0; c < H; ++c) ow[lane * (H + 1) + c] = make_float2(ar[h0 + c], ai[h0 + c]);
                __syncwarp();
                const int c = lane % H;
                const int cg = cc0 + h0 + c;
                for (int j0 = 0; j0 < 32; j0 += CPR) {
                    const int j = j0 + lane / H;
                    const int jz = (bzi << lbz) + (j >> (lby + lbx));
                    const int jy = (byi << lby) + ((j >> lbx) & (wb.by - 1));
                    const int jx = (bxi << lbx) + (j & (wb.bx - 1));
                    if (cg < g.C) {
                        const float2 v = ow[j * (H + 1) + c];
                        if (extra_mode) {
                            slot[((int64_t)(jz * T1 + jy) * T2 + jx) * g.C + cg] = v;
                        } else {
                            const int64_t gi = ((int64_t)(org0 + jz) * nf1 + (org1 + jy)) * nf2 + (org2 + jx);
                            gridf[gi * g.C + cg] = v;
                        }
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();  // the next coil chunk restages into the region
    }
}

// ---- interpolation with compile-time width ---------------------------------------------------
// Lanes of a warp map to (point slot, transform). Each lane keeps its point's first cells and tap
// weights in registers, so the W^d gathers of a point are independent loads the compiler can
// keep in flight together.
template <int CC, int W, bool FR>
__global__ void __launch_bounds__(kGridThreads) k_interp_w(const GridArgs a) {
    extern __shared__ float sm[];
    constexpr int NS = 32 / CC;
    float* coef = sm;
    float* wts_all = coef + kCoefFloats;
    const GridGeom& g = a.g;
    for (int i = threadIdx.x; i < kCoefFloats; i += blockDim.x) coef[i] = (&a.kb.coef[0][0])[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / CC, coil = lane % CC;
    float* wts = wts_all + (warp * NS + slot) * kSlotFloats;
    const int64_t gwarp = (int64_t)blockIdx.x * kGridWarps + warp;
    const int64_t nwarps = (int64_t)gridDim.x * kGridWarps;
    const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
    const int wz = g.wa[0], wy = g.wa[1];
    for (int64_t base = gwarp * NS; base < g.M; base += nwarps * NS) {
        const int64_t s = base + slot;
        const bool valid = s < g.M;
        int i0[3];
        point_setup(a, coef, s, valid, coil, CC, wts, i0);
        __syncwarp();
        if (valid) {
            // element offsets of the taps along axis 2 (x C transforms), 32-bit: a grid holds
            // fewer than 2^32 complex values (checked when the plan is made)
            unsigned colofs[W];
            float wx[W];
#pragma unroll
            for (int d = 0; d < W; ++d) {
                int v = i0[2] + d;
                if (v >= nf2) v -= nf2;
                colofs[d] = (unsigned)v * (unsigned)g.C;
                wx[d] = wts[2 * kMaxWidth + d];
            }
            const int pj = a.perm[s];
            // frames (FR): the grid block of the point's frame; one frame reads a.grid itself
            const float2* const gridf = FR ? a.grid + frame_of_point(a.foff, g.nfr, s) * g.fgrid : a.grid;
            const unsigned rowstride = (unsigned)nf2 * (unsigned)g.C;
            // Common case: the footprint wraps neither along axis 2 nor axis 1 and the lanes hold
            // all C transforms, so a tap's column stride is the compile-time CC: one row pointer,
            // W loads at constant offsets.
            const bool slab_fast = (W <= 6) && g.C % CC == 0 && wy == W && i0[2] + W <= nf2 && i0[1] + W <= nf1;
            const unsigned cs = (unsigned)g.C;  // column stride of a tap along axis 2
            for (int cc0 = 0; cc0 < g.C; cc0 += CC) {
                if (cc0 + coil >= g.C) break;
                const float2* gridc = gridf + cc0 + coil;
                float ar = 0.f, ai = 0.f;
                for (int dz = 0; dz < wz; ++dz) {
                    int gz = i0[0] + dz;
                    if (gz >= nf0) gz -= nf0;
                    const float wzv = wts[dz];
                    if constexpr (W <= 6) {
                        if (slab_fast) {
                            const float2* p0 =
                                gridc + (((unsigned)gz * (unsigned)nf1 + (unsigned)i0[1]) * (unsigned)nf2 + (unsigned)i0[2]) * cs;
                            float2 v[W * W];
#pragma unroll
                            for (int dy = 0; dy < W; ++dy) {
                                const float2* pr = p0 + (size_t)dy * rowstride;
#pragma unroll
                                for (int dx = 0; dx < W; ++dx) v[dy * W + dx] = pr[dx * (g.C == CC ? CC : cs)];
                            }
#pragma unroll
                            for (int dy = 0; dy < W; ++dy) {
                                float rr = 0.f, ri = 0.f;
#pragma unroll
                                for (int dx = 0; dx < W; ++dx) {
                                    rr = fmaf(wx[dx], v[dy * W + dx].x, rr);
                                    ri = fmaf(wx[dx], v[dy * W + dx].y, ri);
                                }
                                const float wzy = wzv * wts[kMaxWidth + dy];
                                ar = fmaf(wzy, rr, ar);
                                ai = fmaf(wzy, ri, ai);
                            }
                            continue;
                        }
                    }
                    unsigned rowbase[W];
#pragma unroll
                    for (int dy = 0; dy < W; ++dy) {
                        int gy = i0[1] + dy;
                        if (gy >= nf1) gy -= nf1;
                        rowbase[dy] = ((unsigned)gz * (unsigned)nf1 + (unsigned)gy) * rowstride;
                    }
                    if constexpr (W <= 6) {
                        // issue the whole W x W slab of gathers before any multiply
                        float2 v[W * W];
#pragma unroll
                        for (int dy = 0; dy < W; ++dy) {
                            const float2* rowp = gridc + rowbase[dy];
#pragma unroll
                            for (int dx = 0; dx < W; ++dx)
                                v[dy * W + dx] = dy < wy ? rowp[colofs[dx]] : make_float2(0.f, 0.f);
                        }
#pragma unroll
                        for (int dy = 0; dy < W; ++dy) {
                            // row partial sum with the axis-2 weights, then one multiply by the row weight
                            float rr = 0.f, ri = 0.f;
#pragma unroll
                            for (int dx = 0; dx < W; ++dx) {
                                rr = fmaf(wx[dx], v[dy * W + dx].x, rr);
                                ri = fmaf(wx[dx], v[dy * W + dx].y, ri);
                            }
                            const float wzy = dy < wy ? wzv * wts[kMaxWidth + dy] : 0.f;
                            ar = fmaf(wzy, rr, ar);
                            ai = fmaf(wzy, ri, ai);
                        }
                    } else {
#pragma unroll
                        for (int dy = 0; dy < W; ++dy) {
                            if (dy < wy) {
                                const float wzy = wzv * wts[kMaxWidth + dy];
                                const float2* rowp = gridc + rowbase[dy];
                                float2 v[W];
#pragma unroll
                                for (int dx = 0; dx < W; ++dx) v[dx] = rowp[colofs[dx]];
                                float rr = 0.f, ri = 0.f;
#pragma unroll
                                for (int dx = 0; dx < W; ++dx) {
                                    rr = fmaf(wx[dx], v[dx].x, rr);
                                    ri = fmaf(wx[dx], v[dx].y, ri);
                                }
                                ar = fmaf(wzy, rr, ar);
                                ai = fmaf(wzy, ri, ai);
                            }
                        }
                    }
                }
                a.out[(int64_t)(cc0 + coil) * g.M + pj] = make_float2(ar, ai);
            }
        }
        __syncwarp();
    }
}

// ---- coordinate gradient by kernel-derivative interpolation ---------------------------------
// grad_x[a][j] = -(nf_a / 2 pi) Re( sum_c h[c][j] sum_l G_c[l] dphi_a(l - u_j) prod_{b!=a} phi_b(l - u_j) )
// G is the plan's fine grid after the type-2 passes, h a per-point complex factor:
//   type 2 (c = A f):      h = conj(dL/dc),          G = grid of f
//   type 1 (f = B c):      h = conj(c),              G = grid of dL/df through the opposite-sign
//                          type-2 passes (the adjoint of deapodise + FFT)
// This is the exact derivative of the implemented gridding operator with respect to the points.
template <int CC, int W>
__global__ void __launch_bounds__(kGridThreads) k_interp_grad(const GridArgs a, const float2* __restrict__ h,
                                                             float* __restrict__ grad, int gdim) {
    extern __shared__ float sm[];
    constexpr int NS = 32 / CC;
    float* coef = sm;
    float* wts_all = coef + kCoefFloats;                                  // [slot][3][kMaxWidth]
    float* dwt_all = wts_all + kGridWarps * NS * kSlotFloats;            // [slot][3][kMaxWidth]
    const GridGeom& g = a.g;
    for (int i = threadIdx.x; i < kCoefFloats; i += blockDim.x) coef[i] = (&a.kb.coef[0][0])[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slot = lane / CC, coil = lane % CC;
    float* wts = wts_all + (warp * NS + slot) * kSlotFloats;
    float* dwt = dwt_all + (warp * NS + slot) * kSlotFloats;
    const int64_t gwarp = (int64_t)blockIdx.x * kGridWarps + warp;
    const int64_t nwarps = (int64_t)gridDim.x * kGridWarps;
    const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];
    const int wz = g.wa[0], wy = g.wa[1];
    for (int64_t base = gwarp * NS; base < g.M; base += nwarps * NS) {
        const int64_t s = base + slot;
        const bool valid = s < g.M;
        int i0[3];
        point_setup(a, coef, s, valid, coil, CC, wts, i0);
        // derivative taps (unit axes keep 0)
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const int w = g.wa[ax];
            if (w == 1) {
                if (coil == 0) dwt[ax * kMaxWidth] = 0.f;
                continue;
            }
            const float u = valid ? a.su[ax][s] : 0.f;
            const float v = __fsub_rn(u, a.kb.hw);
            const float t = __fsub_rn(ceilf(v), v);
            const float sarg = fmaf(2.f, t, -1.f);
            for (int d = coil; d < w; d += CC) dwt[ax * kMaxWidth + d] = kb_tap_deriv(coef, a.kb.deg, d, sarg);
        }
        __syncwarp();
        float r0 = 0.f, r1 = 0.f, r2 = 0.f;
        int pj = 0;
        if (valid) {
            unsigned colofs[W];
            float wx[W], dx_[W];
#pragma unroll
            for (int d = 0; d < W; ++d) {
                int v = i0[2] + d;
                if (v >= nf2) v -= nf2;
                colofs[d] = (unsigned)v * (unsigned)g.C;
                wx[d] = wts[2 * kMaxWidth + d];
                dx_[d] = dwt[2 * kMaxWidth + d];
            }
            pj = a.perm[s];
            const float2* const gridf = a.grid + frame_of_point(a.foff, g.nfr, s) * g.fgrid;
            const unsigned rowstride = (unsigned)nf2 * (unsigned)g.C;
            for (int cc0 = 0; cc0 < g.C; cc0 += CC) {
                if (cc0 + coil >= g.C) break;
                const float2* gridc = gridf + cc0 + coil;
                float2 az = make_float2(0.f, 0.f), ay = az, axx = az;
                for (int dz = 0; dz < wz; ++dz) {
                    int gz = i0[0] + dz;
                    if (gz >= nf0) gz -= nf0;
                    const float wzv = wts[dz], dzv = dwt[dz];
#pragma unroll
                    for (int dy = 0; dy < W; ++dy) {
                        if (dy < wy) {
                            int gy = i0[1] + dy;
                            if (gy >= nf1) gy -= nf1;
                            const float wyv = wts[kMaxWidth + dy], dyv = dwt[kMaxWidth + dy];
                            const float c_zy = wzv * wyv, c_dz = dzv * wyv, c_dy = wzv * dyv;
                            const unsigned rowbase = ((unsigned)gz * (unsigned)nf1 + (unsigned)gy) * rowstride;
#pragma unroll
                            for (int dx = 0; dx < W; ++dx) {
                                const float2 v = gridc[rowbase + colofs[dx]];
                                const float t0 = c_dz * wx[dx], t1 = c_dy * wx[dx], t2 = c_zy * dx_[dx];
                                az.x = fmaf(t0, v.x, az.x);
                                az.y = fmaf(t0, v.y, az.y);
                                ay.x = fmaf(t1, v.x, ay.x);
                                ay.y = fmaf(t1, v.y, ay.y);
                                axx.x = fmaf(t2, v.x, axx.x);
                                axx.y = fmaf(t2, v.y, axx.y);
                            }
                        }
                    }
                }
                const float2 hv = h[(int64_t)(cc0 + coil) * g.M + pj];
                r0 += hv.x * az.x - hv.y * az.y;
                r1 += hv.x * ay.x - hv.y * ay.y;
                r2 += hv.x * axx.x - hv.y * axx.y;
            }
        }
        // sum over the CC lanes of this slot
#pragma unroll
        for (int o = CC / 2; o >= 1; o >>= 1) {
            r0 += __shfl_xor_sync(0xffffffffu, r0, o);
            r1 += __shfl_xor_sync(0xffffffffu, r1, o);
            r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        }
        if (valid && coil == 0) {
            const float r[3] = {r0, r1, r2};
            for (int i = 0; i < gdim; ++i) {
                const int ax = 3 - gdim + i;
                grad[(int64_t)i * g.M + pj] = -r[ax] * g.scale[ax];
            }
        }
        __syncwarp();
    }
}

// ---- x-axis passes between the caller's [C][N..] modes and the interleaved buffers ----------
// Load modes f[e][a][l] (a = row over axes 0,1; l = axis 2) pre-scaled by 1/phihat.
struct OpModesIn {
    static constexpr bool kLoadLFast = true;
    static constexpr bool kStoreLFast = false;
    static constexpr bool kFusedK = false;
    static constexpr bool kChunkLoop = false;
    static constexpr bool kSenseReduce = false;
    const float2* f;
    float2* dst;  // [rows][nf2][C]
    const float* d0;
    const float* d1;
    const float* d2;
    int64_t N1, N2, nm;  // modes of axis 1, 2; modes per transform
    int64_t d_a, d_l;
    int64_t rows_f, fstride;  // frames: rows (N0 N1) and mode values (C nm) per frame; rows_f 0: one frame
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const {
        // row a -> (frame, row of the frame) -> (mode 0, mode 1); 32-bit: F N0 N1 < 2^32 (setpts)
        uint32_t al = (uint32_t)a;
        int64_t fo = 0;
        if (rows_f) {
            const uint32_t fr = al / (uint32_t)rows_f;
            al -= fr * (uint32_t)rows_f;
            fo = (int64_t)fr * fstride;
        }
        const uint32_t i0 = al / (uint32_t)N1, i1 = al - i0 * (uint32_t)N1;
        const float sc = d0[i0] * d1[i1] * d2[l];
        return cscale(f[fo + e * nm + (int64_t)al * N2 + l], sc);
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

// Store modes f[e][a][o] scaled by 1/phihat from the interleaved buffer.
struct OpModesOut {
    static constexpr bool kLoadLFast = false;
    static constexpr bool kStoreLFast = true;
    static constexpr bool kFusedK = false;
    static constexpr bool kChunkLoop = false;
    static constexpr bool kSenseReduce = false;
    const float2* src;  // [rows][nf2][C]
    float2* f;
    const float* d0;
    const float* d1;
    const float* d2;
    int64_t N1, N2, nm;
    int64_t s_a, s_l;
    int64_t rows_f, fstride;  // frames: rows (N0 N1) and mode values (C nm) per frame; rows_f 0: one frame
    __device__ __forceinline__ float2 load(int64_t a, int l, int64_t e) const { return src[a * s_a + (int64_t)l * s_l + e]; }
    __device__ __forceinline__ int64_t kcol(int64_t) const { return 0; }
    __device__ __forceinline__ const float2* kptr(int64_t) const { return nullptr; }
    __device__ __forceinline__ const float2* srow(int64_t, int64_t) const { return nullptr; }
    __device__ __forceinline__ float2 product_s(float2 v, float2) const { return v; }
    __device__ __forceinline__ int64_t group(int64_t) const { return 0; }
    __device__ __forceinline__ int ngroups() const { return 1; }
    __device__ __forceinline__ float2 kval(int64_t, int, int64_t) const { return make_float2(0.f, 0.f); }
    __device__ __forceinline__ void store(int64_t a, int o, int64_t e, float2 v) const {
        uint32_t al = (uint32_t)a;
        int64_t fo = 0;
        if (rows_f) {
            const uint32_t fr = al / (uint32_t)rows_f;
            al -= fr * (uint32_t)rows_f;
            fo = (int64_t)fr * fstride;
        }
        const uint32_t i0 = al / (uint32_t)N1, i1 = al - i0 * (uint32_t)N1;
        const float sc = d0[i0] * d1[i1] * d2[o];
        f[fo + e * nm + (int64_t)al * N2 + o] = cscale(v, sc);
    }
    __device__ __forceinline__ float2 product(int64_t, int, int64_t, float2 v) const { return v; }
    __device__ __forceinline__ void write_row(int64_t, int, int, float2) const {}
    __device__ __forceinline__ void store_phase(const float2* res, const PassCfg& c, int64_t a0, int64_t e0, int, int,
                                                float2*) const {
        for_each_output<true>(res, c, a0, e0, [&](int64_t a, int o, int64_t e, float2 v) { store(a, o, e, v); });
    }
    __device__ __forceinline__ void finish(const PassCfg&, int64_t, float2*) const {}
};

// ---------------------------------------------------------------------------------------------
// plan lifecycle

static int dev_alloc(NufftPlan* p, void** ptr, size_t bytes, const char* what) {
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        set_error(std::string("cudaMalloc(") + what + ", " + std::to_string(bytes) + " bytes) failed: " +
                  cudaGetErrorString(e));
        return HB_ERR_ALLOC;
    }
    p->device_bytes += bytes;
    return HB_OK;
}

int plan_make(NufftPlan* p, int type, int dim, const int64_t* nmodes, int sign, int ntransf, float tol, int width,
              double upsampfac, int method) {
    HB_REQUIRE(type == 1 || type == 2, HB_ERR_INVALID_ARG, "nufft type must be 1 or 2");
    HB_REQUIRE(dim >= 1 && dim <= 3, HB_ERR_INVALID_ARG, "dim must be 1, 2 or 3");
    HB_REQUIRE(nmodes != nullptr, HB_ERR_INVALID_ARG, "nmodes is null");
    HB_REQUIRE(ntransf >= 1, HB_ERR_INVALID_ARG, "ntransf must be >= 1");
    HB_REQUIRE(method >= 0 && method <= 3, HB_ERR_INVALID_ARG, "invalid method");
    HB_REQUIRE(sign == 0 || sign == 1 || sign == -1, HB_ERR_INVALID_ARG, "sign must be -1, 0 or +1");
    p->type = type;
    p->sign = sign != 0 ? sign : (type == 1 ? 1 : -1);
    p->method = method;
    p->sigma = upsampfac > 0 ? upsampfac : 2.0;
    HB_REQUIRE(p->sigma >= 1.1 && p->sigma <= 4.0, HB_ERR_INVALID_ARG, "upsampfac must be in [1.1, 4]");
    int w = width;
    if (w <= 0) {
        HB_REQUIRE(tol > 0.f && tol < 1.f, HB_ERR_INVALID_ARG, "tol must be in (0,1) when kernel_width <= 0");
        w = (int)std::ceil(std::log10(10.0 / (double)tol));
        if (p->sigma < 2.0) {
            // cufinufft's width rule for low upsampling: ceil(-ln(tol) / (pi sqrt(1 - 1/sigma)))
            w = (int)std::ceil(-std::log((double)tol) / (M_PI * std::sqrt(1.0 - 1.0 / p->sigma)));
        }
        w = std::max(2, std::min(kMaxWidth, w));
    }
    HB_REQUIRE(w >= 2 && w <= kMaxWidth, HB_ERR_INVALID_ARG, "kernel width must be in [2, 16]");

    GridGeom& g = p->g;
    g.dim = dim;
    g.C = ntransf;
    for (int ax = 0; ax < 3; ++ax) g.Nm[ax] = 1;
    for (int i = 0; i < dim; ++i) {
        HB_REQUIRE(nmodes[i] >= 1 && nmodes[i] <= (1 << 20), HB_ERR_INVALID_ARG, "nmodes out of range");
        g.Nm[3 - dim + i] = nmodes[i];
    }
    // tiles: 8^3 (3-D), 16x32 (2-D), 256 (1-D); wider kernels need tiles >= w-1
    int Tt[3];
    if (dim == 3) {
        const int e = (w <= 9) ? 8 : 16;
        Tt[0] = Tt[1] = Tt[2] = e;
    } else if (dim == 2) {
        Tt[0] = 1;
        Tt[1] = 16;
        Tt[2] = 32;
    } else {
        Tt[0] = Tt[1] = 1;
        Tt[2] = 256;
    }
    for (int ax = 0; ax < 3; ++ax) {
        const bool unit = (ax < 3 - dim);
        g.T[ax] = unit ? 1 : Tt[ax];
        g.wa[ax] = unit ? 1 : w;
        g.nf[ax] = unit ? 1 : fine_size(g.Nm[ax], p->sigma, w, g.T[ax]);
        g.nb[ax] = g.nf[ax] / g.T[ax];
        g.scale[ax] = (float)((double)g.nf[ax] / (2.0 * M_PI));
    }
    if (dim == 2) {
        p->wb[0] = 1;
        p->wb[1] = 4;
        p->wb[2] = 8;
    }
    // lanes-on-transforms spreading: 8^3 (3-D) or 16x32 (2-D) tiles, widths 4..8, more than four
    // transforms, and at least two tiles along every non-unit axis (so no footprint wraps onto its
    // own tile)
    {
        bool ok = (dim == 3 || dim == 2) && w >= 4 && w <= 8 && ntransf >= 5;
        for (int ax = 3 - dim; ax < 3; ++ax) ok = ok && g.nb[ax] >= 2;
        p->lc = p->lc_ok = ok;
        p->lc_cc = ntransf >= 17 ? 32 : (ntransf >= 9 ? 16 : 8);
        p->st_ok = type == 2 && dim == 3 && w >= 4 && w <= 7;
        p->st = false;
    }
    p->beta = kb_beta(w, p->sigma);
    const double fit_err = kb_fit(&p->kb, w, p->beta);
    if (!(fit_err < 1e-6)) {
        set_error("kernel polynomial fit failed");
        return HB_ERR_INVALID_ARG;
    }
    p->nbins = (int64_t)g.nb[0] * g.nb[1] * g.nb[2];
    g.nfr = 1;
    g.ntf = p->nbins;

    // FFT plans and deapodisation factors per axis
    for (int ax = 0; ax < 3; ++ax) {
        if (g.nf[ax] > 1) HB_TRY(fftlen_make(&p->fl[ax], g.nf[ax]));
        std::vector<float> dv((size_t)g.Nm[ax], 1.0f);
        if (g.nf[ax] > 1) {
            const int64_t half = g.Nm[ax] / 2;
            for (int64_t i = 0; i < g.Nm[ax]; ++i) {
                const double k = (double)(i - half);
                dv[(size_t)i] = (float)(1.0 / kb_phihat(k / (double)g.nf[ax], w, p->beta));
            }
        }
        HB_TRY(dev_alloc(p, (void**)&p->deapod[ax], sizeof(float) * dv.size(), "deapod"));
        HB_CUDA(cudaMemcpy(p->deapod[ax], dv.data(), sizeof(float) * dv.size(), cudaMemcpyHostToDevice));
    }
    p->X_elems = (size_t)g.nf[0] * g.nf[1] * g.nf[2] * g.C;
    HB_REQUIRE(p->X_elems < ((size_t)1 << 32), HB_ERR_INVALID_ARG,
               "fine grid x ntransf must hold fewer than 2^32 values; split the transforms");
    p->Y_elems = (size_t)g.Nm[0] * g.nf[1] * g.nf[2] * g.C;
    g.fgrid = (int64_t)p->X_elems;
    p->frames_cap = 1;
    HB_TRY(dev_alloc(p, (void**)&p->X, sizeof(float2) * p->X_elems, "fine grid"));
    HB_TRY(dev_alloc(p, (void**)&p->Y, sizeof(float2) * p->Y_elems, "pass buffer"));
    HB_TRY(dev_alloc(p, (void**)&p->bin_start, sizeof(int) * (p->nbins + 1), "bins"));
    p->nbins_cap = p->nbins;
    HB_TRY(dev_alloc(p, (void**)&p->d_err, sizeof(int), "error flag"));
    return HB_OK;
}

// Candidates per spread subproblem when the caller has not set one: every point is a candidate
// of up to 2^d tiles; aim at about 32 subproblems per SM so that the dense tiles of centre-heavy
// trajectories (radial, spirals) split across the GPU, with at least 256 and at most 4096
// candidates (large problems keep long chunks per CTA).
static int auto_subproblem(int64_t M, const GridGeom& g) {
    int64_t cand = M;
    for (int ax = 0; ax < 3; ++ax)
        if (g.nb[ax] > 1) cand *= 2;
    const int64_t want = cand / ((int64_t)kNumSMs * 32);
    int m = 256;
    while (m < want && m < 4096) m <<= 1;
    return m;
}

// Job list of the staged interpolation kernel for the current points (type-2 plans).
static int st_build_jobs(NufftPlan* p, cudaStream_t s) {
    int n_jobs = 0;
    HB_TRY(interp_st_jobs(p->bin_start, p->nbins, p->g.wa[2], p->tmp_ecnt, p->tmp_eoff, p->tmp_sums, nullptr, &n_jobs, 0, s));
    if (n_jobs > p->st_cap) {
        if (p->st_jobs) cudaFree(p->st_jobs);
        p->st_jobs = nullptr;
        p->st_cap = 0;
        HB_TRY(dev_alloc(p, (void**)&p->st_jobs, sizeof(int4) * n_jobs, "staged interpolation jobs"));
        p->st_cap = n_jobs;
    }
    HB_TRY(interp_st_jobs(p->bin_start, p->nbins, p->g.wa[2], p->tmp_ecnt, p->tmp_eoff, p->tmp_sums, p->st_jobs, &n_jobs,
                          p->st_cap, s));
    p->n_st_jobs = n_jobs;
    p->st_built = true;
    return HB_OK;
}

int plan_setpts(NufftPlan* p, int64_t M, const float* c0, const float* c1, const float* c2, cudaStream_t s) {
    return plan_setpts_frames(p, 1, &M, c0, c1, c2, s);
}

int plan_setpts_frames(NufftPlan* p, int nframes, const int64_t* npts, const float* c0, const float* c1,
                       const float* c2, cudaStream_t s) {
    GridGeom& g = p->g;
    HB_REQUIRE(nframes >= 1 && nframes <= (1 << 16), HB_ERR_INVALID_ARG, "nframes must be in [1, 65536]");
    HB_REQUIRE(npts != nullptr, HB_ERR_INVALID_ARG, "npts is null");
    int64_t M = 0;
    std::vector<int> hoff((size_t)nframes + 1, 0);
    for (int f = 0; f < nframes; ++f) {
        HB_REQUIRE(npts[f] >= 0, HB_ERR_INVALID_ARG, "a frame's point count is negative");
        M += npts[f];
        HB_REQUIRE(M < (int64_t)0x7fffffff, HB_ERR_INVALID_ARG, "M must be in [0, 2^31)");
        hoff[(size_t)f + 1] = (int)M;
    }
    HB_REQUIRE((int64_t)p->g.ntf * nframes < (int64_t)0x7fffffff, HB_ERR_INVALID_ARG, "too many frames for the grid");
    HB_REQUIRE(p->g.Nm[0] * p->g.Nm[1] * nframes < ((int64_t)1 << 32), HB_ERR_INVALID_ARG, "too many frames for the modes");
    // grids and per-bin scratch for nframes frames (grown, never shrunk)
    if (nframes > p->frames_cap) {
        if (p->X) cudaFree(p->X);
        if (p->Y) cudaFree(p->Y);
        p->X = p->Y = nullptr;
        p->frames_cap = 0;
        p->pts_set = false;
        HB_TRY(dev_alloc(p, (void**)&p->X, sizeof(float2) * p->X_elems * nframes, "fine grid (frames)"));
        HB_TRY(dev_alloc(p, (void**)&p->Y, sizeof(float2) * p->Y_elems * nframes, "pass buffer (frames)"));
        p->frames_cap = nframes;
    }
    const int64_t nbins_all = p->g.ntf * nframes;
    if (nbins_all > p->nbins_cap) {
        for (int** q : {&p->bin_start, &p->tmp_count, &p->tmp_ecnt, &p->tmp_eoff, &p->tmp_sums}) {
            if (*q) cudaFree(*q);
            *q = nullptr;
        }
        p->nbins_cap = 0;
        p->pts_set = false;
        HB_TRY(dev_alloc(p, (void**)&p->bin_start, sizeof(int) * (nbins_all + 1), "bins (frames)"));
        p->nbins_cap = nbins_all;
    }
    if (nframes > 1 && nframes + 1 > p->foff_cap) {
        if (p->foff) cudaFree(p->foff);
        p->foff = nullptr;
        p->foff_cap = 0;
        HB_TRY(dev_alloc(p, (void**)&p->foff, sizeof(int) * (nframes + 1), "frame offsets"));
        p->foff_cap = nframes + 1;
    }
    if (nframes > 1) HB_CUDA(cudaMemcpyAsync(p->foff, hoff.data(), sizeof(int) * (nframes + 1), cudaMemcpyHostToDevice, s));
    g.nfr = nframes;
    p->nbins = nbins_all;
    const float* cu[3] = {c0, c1, c2};
    const float* ca[3] = {nullptr, nullptr, nullptr};
    for (int i = 0; i < g.dim; ++i) {
        HB_REQUIRE(M == 0 || cu[i] != nullptr, HB_ERR_INVALID_ARG, "coordinate array is null");
        ca[3 - g.dim + i] = cu[i];
    }
    if (M > p->M_cap) {
        for (int ax = 0; ax < 3; ++ax) {
            if (p->su[ax]) cudaFree(p->su[ax]);
            p->su[ax] = nullptr;
        }
        if (p->perm) cudaFree(p->perm);
        if (p->inT) cudaFree(p->inT);
        p->perm = nullptr;
        p->inT = nullptr;
        for (int ax = 0; ax < 3; ++ax)
            if (ca[ax] || g.nf[ax] > 1) HB_TRY(dev_alloc(p, (void**)&p->su[ax], sizeof(float) * M, "sorted coords"));
        HB_TRY(dev_alloc(p, (void**)&p->perm, sizeof(int) * M, "perm"));
        if (p->type == 1) HB_TRY(dev_alloc(p, (void**)&p->inT, sizeof(float2) * M * g.C, "interleaved input"));
        p->M_cap = M;
    }
    g.M = M;
    p->pts_set = false;

    // scratch held by the plan (allocated on the first setpts, per-point arrays grown with M)
    int st = HB_OK;
    if (p->tmp_count == nullptr) {
        const int64_t nb = ceil_div(std::max<int64_t>(p->nbins_cap, 1), kScanBlock);
        HB_TRY(dev_alloc(p, (void**)&p->tmp_count, sizeof(int) * (p->nbins_cap + 1), "bin counts"));
        HB_TRY(dev_alloc(p, (void**)&p->tmp_ecnt, sizeof(int) * (p->nbins_cap + 1), "subproblem counts"));
        HB_TRY(dev_alloc(p, (void**)&p->tmp_eoff, sizeof(int) * (p->nbins_cap + 1), "subproblem offsets"));
        HB_TRY(dev_alloc(p, (void**)&p->tmp_sums, sizeof(int) * nb, "scan sums"));
    }
    if (M > p->tmp_cap) {
        for (int ax = 0; ax < 3; ++ax) {
            if (p->tmp_u[ax]) cudaFree(p->tmp_u[ax]);
            p->tmp_u[ax] = nullptr;
        }
        if (p->tmp_binid) cudaFree(p->tmp_binid);
        if (p->tmp_rank) cudaFree(p->tmp_rank);
        p->tmp_binid = p->tmp_rank = nullptr;
        p->tmp_cap = 0;
        for (int ax = 0; ax < 3; ++ax)
            if (ca[ax]) HB_TRY(dev_alloc(p, (void**)&p->tmp_u[ax], sizeof(float) * M, "fine coordinates"));
        HB_TRY(dev_alloc(p, (void**)&p->tmp_binid, sizeof(int) * M, "bin ids"));
        HB_TRY(dev_alloc(p, (void**)&p->tmp_rank, sizeof(int) * M, "bin ranks"));
        p->tmp_cap = M;
    }
    float* u[3] = {ca[0] ? p->tmp_u[0] : nullptr, ca[1] ? p->tmp_u[1] : nullptr, ca[2] ? p->tmp_u[2] : nullptr};
    int *binid = p->tmp_binid, *rank = p->tmp_rank, *count = p->tmp_count, *ecnt = p->tmp_ecnt, *eoff = p->tmp_eoff;
    do {
        cudaError_t e = cudaSuccess;
        if ((e = cudaMemsetAsync(count, 0, sizeof(int) * (p->nbins + 1), s)) != cudaSuccess ||
            (e = cudaMemsetAsync(p->d_err, 0, sizeof(int), s)) != cudaSuccess) {
            set_error(std::string("setpts memset: ") + cudaGetErrorString(e));
            st = HB_ERR_CUDA;
            break;
        }
        if (M > 0) {
            FoldArgs fa{};
            for (int ax = 0; ax < 3; ++ax) {
                fa.c[ax] = ca[ax];
                fa.u[ax] = u[ax];
                fa.nf[ax] = g.nf[ax];
                fa.T[ax] = g.T[ax];
                fa.nb[ax] = g.nb[ax];
                fa.scale[ax] = g.scale[ax];
            }
            fa.binid = binid;
            fa.rank = rank;
            fa.count = count;
            fa.err = p->d_err;
            fa.hw = p->kb.hw;
            fa.M = M;
            fa.foff = nframes > 1 ? p->foff : nullptr;
            fa.nfr = nframes;
            fa.ntf = (int)g.ntf;
            k_fold_bin<<<(unsigned)ceil_div(M, 256), 256, 0, s>>>(fa);
            if ((st = check_launch("k_fold_bin")) != HB_OK) break;
        }
        if ((st = exclusive_scan_int(count, p->bin_start, p->nbins, s, p->tmp_sums)) != HB_OK) break;
        if (M > 0) {
            k_scatter_sorted<<<(unsigned)ceil_div(M, 256), 256, 0, s>>>(u[0], u[1], u[2], binid, rank, p->bin_start,
                                                                       ca[0] ? p->su[0] : nullptr, ca[1] ? p->su[1] : nullptr,
                                                                       ca[2] ? p->su[2] : nullptr, p->perm, M);
            if ((st = check_launch("k_scatter_sorted")) != HB_OK) break;
        }
        // unit axes: sorted coordinate arrays hold zeros
        for (int ax = 0; ax < 3; ++ax)
            if (!ca[ax] && p->su[ax] && M > 0) cudaMemsetAsync(p->su[ax], 0, sizeof(float) * M, s);
        if (p->type == 1 && p->lc) {
            if (p->maxp_auto) p->maxp = auto_subproblem(M, g);
            TileNbr tn;
            for (int ax = 0; ax < 3; ++ax) tn.nb[ax] = g.nb[ax];
            tn.nfr = nframes;
            tn.ntf = (int)g.ntf;
            k_tile_parts_count<<<(unsigned)ceil_div(p->nbins, 256), 256, 0, s>>>(p->bin_start, tn, p->nbins, p->maxp, ecnt);
            if ((st = check_launch("k_tile_parts_count")) != HB_OK) break;
            if ((st = exclusive_scan_int(ecnt, eoff, p->nbins, s, p->tmp_sums)) != HB_OK) break;
            int n_parts = 0;
            if ((e = cudaMemcpyAsync(&n_parts, eoff + p->nbins, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                set_error(std::string("setpts sync: ") + cudaGetErrorString(e));
                st = HB_ERR_CUDA;
                break;
            }
            if (n_parts > p->parts_cap) {
                if (p->dense_parts) cudaFree(p->dense_parts);
                p->dense_parts = nullptr;
                p->parts_cap = 0;
                if ((st = dev_alloc(p, (void**)&p->dense_parts, sizeof(int4) * n_parts, "dense tile parts")) != HB_OK) break;
                p->parts_cap = n_parts;
            }
            const size_t need = sizeof(float2) * (size_t)n_parts * g.T[0] * g.T[1] * g.T[2] * g.C;
            if (need > p->scratch_cap) {
                if (p->dense_scratch) cudaFree(p->dense_scratch);
                p->dense_scratch = nullptr;
                p->scratch_cap = 0;
                if ((st = dev_alloc(p, (void**)&p->dense_scratch, need, "dense tile partials")) != HB_OK) break;
                p->scratch_cap = need;
            }
            p->n_parts = n_parts;
            if (n_parts > 0) {
                k_tile_parts_fill<<<(unsigned)ceil_div(p->nbins, 256), 256, 0, s>>>(ecnt, eoff, p->nbins, p->dense_parts);
                if ((st = check_launch("k_tile_parts_fill")) != HB_OK) break;
            }
            p->n_extra = 0;
        } else if (p->type == 1) {
            if (p->maxp_auto) p->maxp = auto_subproblem(M, g);
            TileNbr tn;
            for (int ax = 0; ax < 3; ++ax) tn.nb[ax] = g.nb[ax];
            tn.nfr = nframes;
            tn.ntf = (int)g.ntf;
            k_tile_extra_count<<<(unsigned)ceil_div(p->nbins, 256), 256, 0, s>>>(p->bin_start, tn, p->nbins,
                                                                                p->maxp, ecnt);
            if ((st = check_launch("k_tile_extra_count")) != HB_OK) break;
            if ((st = exclusive_scan_int(ecnt, eoff, p->nbins, s, p->tmp_sums)) != HB_OK) break;
            int n_extra = 0, err = 0;
            if ((e = cudaMemcpyAsync(&n_extra, eoff + p->nbins, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaMemcpyAsync(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                set_error(std::string("setpts sync: ") + cudaGetErrorString(e));
                st = HB_ERR_CUDA;
                break;
            }
            if (err) {
                set_error("setpts: non-finite coordinate");
                st = HB_ERR_RANGE;
                break;
            }
            if (n_extra > p->extra_cap) {
                if (p->extra) cudaFree(p->extra);
                p->extra = nullptr;
                p->extra_cap = 0;
                if ((st = dev_alloc(p, (void**)&p->extra, sizeof(int4) * n_extra, "spread work list")) != HB_OK) break;
                p->extra_cap = n_extra;
            }
            const size_t need = sizeof(float2) * (size_t)n_extra * g.T[0] * g.T[1] * g.T[2] * g.C;
            if (need > p->extra_scratch_cap) {
                if (p->extra_scratch) cudaFree(p->extra_scratch);
                p->extra_scratch = nullptr;
                p->extra_scratch_cap = 0;
                if ((st = dev_alloc(p, (void**)&p->extra_scratch, need, "spread partial tiles")) != HB_OK) break;
                p->extra_scratch_cap = need;
            }
            p->n_extra = n_extra;
            if (n_extra > 0) {
                k_tile_extra_fill<<<(unsigned)ceil_div(p->nbins, 256), 256, 0, s>>>(ecnt, eoff, p->nbins, p->extra);
                if ((st = check_launch("k_tile_extra_fill")) != HB_OK) break;
            }
        }
        p->st_built = false;
        if (p->type == 2 && p->st && (st = st_build_jobs(p, s)) != HB_OK) break;
        {
            int err = 0;
            if ((e = cudaMemcpyAsync(&err, p->d_err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess) {
                set_error(std::string("setpts sync: ") + cudaGetErrorString(e));
                st = HB_ERR_CUDA;
                break;
            }
            if (err) {
                set_error("setpts: non-finite coordinate");
                st = HB_ERR_RANGE;
                break;
            }
        }
    } while (0);
    if (st == HB_OK) p->pts_set = true;
    return st;
}

static GridArgs grid_args(const NufftPlan* p) {
    GridArgs a{};
    a.g = p->g;
    for (int ax = 0; ax < 3; ++ax) a.su[ax] = p->su[ax];
    a.perm = p->perm;
    a.bin_start = p->bin_start;
    a.foff = p->g.nfr > 1 ? p->foff : nullptr;
    a.inT = p->inT;
    a.grid = p->X;
    a.extra = p->extra;
    a.extra_scratch = p->extra_scratch;
    a.maxp = p->maxp;
    a.kb = p->kb;
    return a;
}

template <int CC>
static int launch_spread_cc(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    const GridGeom& g = p->g;
    const int cells = g.T[0] * g.T[1] * g.T[2];
    if (cells == 512 && g.dim >= 2) {
        // output-stationary kernel: one thread per cell of an 8x8x8 (3-D) or 16x32 (2-D) tile
        SpreadTileShape wb{p->wb[0], p->wb[1], p->wb[2]};
        const size_t smem = sizeof(float) * (size_t)SpreadSmem<CC>::kFloats;
        HB_CUDA(cudaFuncSetAttribute(k_spread_reg<CC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        {
            TimedSection ts("spread", s);
            k_spread_reg<CC><<<(unsigned)p->nbins, kSpreadThreads, smem, s>>>(a, 0, wb);
            HB_TRY(check_launch("k_spread_reg"));
        }
        if (p->n_extra > 0) {
            TimedSection ts("spread_dense", s);
            k_spread_reg<CC><<<(unsigned)p->n_extra, kSpreadThreads, smem, s>>>(a, 1, wb);
            HB_TRY(check_launch("k_spread_reg(extra)"));
            k_spread_extra_reduce<<<(unsigned)p->n_extra, 256, 0, s>>>(a);
            HB_TRY(check_launch("k_spread_extra_reduce"));
        }
        return HB_OK;
    }
    const size_t smem = sizeof(float) * ((size_t)2 * cells * CC + kCoefFloats + (size_t)kGridWarps * (32 / CC) * kSlotFloats);
    HB_CUDA(cudaFuncSetAttribute(k_spread<CC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
        TimedSection ts("spread", s);
        k_spread<CC><<<(unsigned)p->nbins, kGridThreads, smem, s>>>(a, 0);
        HB_TRY(check_launch("k_spread"));
    }
    if (p->n_extra > 0) {
        TimedSection ts("spread_dense", s);
        k_spread<CC><<<(unsigned)p->n_extra, kGridThreads, smem, s>>>(a, 1);
        HB_TRY(check_launch("k_spread(extra)"));
        k_spread_extra_reduce<<<(unsigned)p->n_extra, 256, 0, s>>>(a);
        HB_TRY(check_launch("k_spread_extra_reduce"));
    }
    return HB_OK;
}

template <int CC, int W>
static int launch_interp_w(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    const int64_t per_block = (int64_t)kGridWarps * (32 / CC);
    int64_t blocks = ceil_div(std::max<int64_t>(p->g.M, 1), per_block);
    blocks = std::min<int64_t>(blocks, (int64_t)kNumSMs * 64);
    const size_t smem = sizeof(float) * (kCoefFloats + (size_t)kGridWarps * (32 / CC) * kSlotFloats);
    TimedSection ts("interp", s);
    if (a.foff) {
        HB_CUDA(cudaFuncSetAttribute(k_interp_w<CC, W, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_interp_w<CC, W, true><<<(unsigned)blocks, kGridThreads, smem, s>>>(a);
    } else {
        HB_CUDA(cudaFuncSetAttribute(k_interp_w<CC, W, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_interp_w<CC, W, false><<<(unsigned)blocks, kGridThreads, smem, s>>>(a);
    }
    return check_launch("k_interp");
}

template <int CC>
static int launch_interp_cc(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    switch (p->kb.w) {
        case 2: return launch_interp_w<CC, 2>(p, a, s);
        case 3: return launch_interp_w<CC, 3>(p, a, s);
        case 4: return launch_interp_w<CC, 4>(p, a, s);
        case 5: return launch_interp_w<CC, 5>(p, a, s);
        case 6: return launch_interp_w<CC, 6>(p, a, s);
        case 7: return launch_interp_w<CC, 7>(p, a, s);
        case 8: return launch_interp_w<CC, 8>(p, a, s);
        case 9: return launch_interp_w<CC, 9>(p, a, s);
        case 10: return launch_interp_w<CC, 10>(p, a, s);
        case 11: return launch_interp_w<CC, 11>(p, a, s);
        case 12: return launch_interp_w<CC, 12>(p, a, s);
        case 13: return launch_interp_w<CC, 13>(p, a, s);
        case 14: return launch_interp_w<CC, 14>(p, a, s);
        case 15: return launch_interp_w<CC, 15>(p, a, s);
        default: return launch_interp_w<CC, 16>(p, a, s);
    }
}

static int dispatch_cc(int cc, const NufftPlan* p, const GridArgs& a, cudaStream_t s, bool spread) {
    switch (cc) {
        case 1: return spread ? launch_spread_cc<1>(p, a, s) : launch_interp_cc<1>(p, a, s);
        case 2: return spread ? launch_spread_cc<2>(p, a, s) : launch_interp_cc<2>(p, a, s);
        case 4: return spread ? launch_spread_cc<4>(p, a, s) : launch_interp_cc<4>(p, a, s);
        case 8: return spread ? launch_spread_cc<8>(p, a, s) : launch_interp_cc<8>(p, a, s);
        case 16: return spread ? launch_spread_cc<16>(p, a, s) : launch_interp_cc<16>(p, a, s);
        default: return spread ? launch_spread_cc<32>(p, a, s) : launch_interp_cc<32>(p, a, s);
    }
}

// Type-2 passes: caller modes [C][N..] -> fine grid (returned in *G, one of the plan buffers).
static int type2_grid(NufftPlan* p, const float2* in, float2** G, cudaStream_t s) {
    const GridGeom& g = p->g;
    const int C = g.C;
    const int64_t nm = g.Nm[0] * g.Nm[1] * g.Nm[2];
    const bool inv = p->sign > 0;
    const int64_t h0 = g.Nm[0] / 2, h1 = g.Nm[1] / 2, h2 = g.Nm[2] / 2;
    const int npass = 1 + (g.nf[1] > 1) + (g.nf[0] > 1);
    const int64_t F = g.nfr;  // frames: one block of rows each in every pass
    float2* cur = (npass % 2 == 1) ? p->X : p->Y;
    float2* other = (cur == p->X) ? p->Y : p->X;
    {
        OpModesIn op{in, cur, p->deapod[0], p->deapod[1], p->deapod[2], g.Nm[1], g.Nm[2], nm, (int64_t)g.nf[2] * C, C,
                     F > 1 ? g.Nm[0] * g.Nm[1] : 0, (int64_t)C * nm};
        HB_TRY(launch_fft_pass(op, p->fl[2], F * g.Nm[0] * g.Nm[1], C, (int)g.Nm[2], (int)-h2, g.nf[2], 0, inv, 0, s,
                               "type2 axis2"));
    }
    if (g.nf[1] > 1) {
        const int64_t E = (int64_t)g.nf[2] * C;
        OpStrided op{cur, other, g.Nm[1] * E, E, (int64_t)g.nf[1] * E, E, 1.0f};
        HB_TRY(launch_fft_pass(op, p->fl[1], F * g.Nm[0], E, (int)g.Nm[1], (int)-h1, g.nf[1], 0, inv, 0, s, "type2 axis1"));
        std::swap(cur, other);
    }
    if (g.nf[0] > 1) {
        const int64_t E = (int64_t)g.nf[1] * g.nf[2] * C;
        OpStrided op{cur, other, g.Nm[0] * E, E, (int64_t)g.nf[0] * E, E, 1.0f};
        HB_TRY(launch_fft_pass(op, p->fl[0], F, E, (int)g.Nm[0], (int)-h0, g.nf[0], 0, inv, 0, s, "type2 axis0"));
        std::swap(cur, other);
    }
    *G = cur;
    return HB_OK;
}

int plan_execute(NufftPlan* p, const float2* in, float2* out, cudaStream_t s) {
    HB_REQUIRE(p->pts_set, HB_ERR_STATE, "execute called before setpts");
    const GridGeom& g = p->g;
    // the nonuniform side may be empty (M == 0), the mode side never is
    const bool in_ok = in != nullptr || (p->type == 1 && g.M == 0);
    const bool out_ok = out != nullptr || (p->type == 2 && g.M == 0);
    HB_REQUIRE(in_ok && out_ok, HB_ERR_INVALID_ARG, "null data pointer");
    const int C = g.C;
    const int64_t M = g.M;
    const int64_t nm = g.Nm[0] * g.Nm[1] * g.Nm[2];
    const bool inv = p->sign > 0;
    const int64_t h0 = g.Nm[0] / 2, h1 = g.Nm[1] / 2, h2 = g.Nm[2] / 2;

    if (p->type == 1) {
        if (M > 0) {
            TimedSection ts("interleave_in", s);
            k_interleave_in<<<dim3((unsigned)ceil_div(M, 32), (unsigned)ceil_div(C, 32)), dim3(32, 8), 0, s>>>(
                in, p->inT, M, C);
            HB_TRY(check_launch("k_interleave_in"));
        }
        GridArgs a = grid_args(p);
        if (p->lc)
            HB_TRY(p->lc_cc == 8 ? spread_lc_cc8(p, a, s) : (p->lc_cc == 16 ? spread_lc_cc16(p, a, s) : spread_lc_cc32(p, a, s)));
        else
            HB_TRY(dispatch_cc(spread_cc(g), p, a, s, true));
        float2* cur = p->X;
        float2* other = p->Y;
        const int64_t F = g.nfr;  // frames: one block of rows each in every pass
        // axis 0: [F][nf0][nf1*nf2*C] -> [F][Nm0][...]
        if (g.nf[0] > 1) {
            const int64_t E = (int64_t)g.nf[1] * g.nf[2] * C;
            OpStrided op{cur, other, (int64_t)g.nf[0] * E, E, g.Nm[0] * E, E, 1.0f};
            HB_TRY(launch_fft_pass(op, p->fl[0], F, E, g.nf[0], 0, (int)g.Nm[0], (int)-h0, inv, 0, s, "type1 axis0"));
            std::swap(cur, other);
        }
        // axis 1: [F Nm0][nf1][nf2*C] -> [F Nm0][Nm1][nf2*C]
        if (g.nf[1] > 1) {
            const int64_t E = (int64_t)g.nf[2] * C;
            OpStrided op{cur, other, (int64_t)g.nf[1] * E, E, g.Nm[1] * E, E, 1.0f};
            HB_TRY(launch_fft_pass(op, p->fl[1], F * g.Nm[0], E, g.nf[1], 0, (int)g.Nm[1], (int)-h1, inv, 0, s, "type1 axis1"));
            std::swap(cur, other);
        }
        // axis 2 -> caller's modes [F][C][Nm..] with deapodisation
        {
            OpModesOut op{cur, out, p->deapod[0], p->deapod[1], p->deapod[2], g.Nm[1], g.Nm[2], nm,
                          (int64_t)g.nf[2] * C, C, F > 1 ? g.Nm[0] * g.Nm[1] : 0, (int64_t)C * nm};
            HB_TRY(launch_fft_pass(op, p->fl[2], F * g.Nm[0] * g.Nm[1], C, g.nf[2], 0, (int)g.Nm[2], (int)-h2, inv, 0, s,
                                   "type1 axis2"));
        }
        return HB_OK;
    }

    // type 2: passes x, y, z into the fine grid, then interpolate
    float2* G = nullptr;
    HB_TRY(type2_grid(p, in, &G, s));
    if (M > 0) {
        GridArgs a = grid_args(p);
        a.grid = G;
        a.out = out;
        if (p->st)
            HB_TRY(interp_st_run(p, a, s));
        else
            HB_TRY(dispatch_cc(p->interp_cc ? p->interp_cc : spread_cc(g), p, a, s, false));
    }
    return HB_OK;
}

template <int CC, int W>
static int launch_grad_w(const NufftPlan* p, const GridArgs& a, const float2* h, float* grad, cudaStream_t s) {
    const int64_t per_block = (int64_t)kGridWarps * (32 / CC);
    int64_t blocks = ceil_div(std::max<int64_t>(p->g.M, 1), per_block);
    blocks = std::min<int64_t>(blocks, (int64_t)kNumSMs * 64);
    const size_t smem = sizeof(float) * (kCoefFloats + (size_t)2 * kGridWarps * (32 / CC) * kSlotFloats);
    HB_CUDA(cudaFuncSetAttribute(k_interp_grad<CC, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TimedSection ts("interp_grad", s);
    k_interp_grad<CC, W><<<(unsigned)blocks, kGridThreads, smem, s>>>(a, h, grad, p->g.dim);
    return check_launch("k_interp_grad");
}

template <int CC>
static int launch_grad_cc(const NufftPlan* p, const GridArgs& a, const float2* h, float* grad, cudaStream_t s) {
    switch (p->kb.w) {
        case 2: return launch_grad_w<CC, 2>(p, a, h, grad, s);
        case 3: return launch_grad_w<CC, 3>(p, a, h, grad, s);
        case 4: return launch_grad_w<CC, 4>(p, a, h, grad, s);
        case 5: return launch_grad_w<CC, 5>(p, a, h, grad, s);
        case 6: return launch_grad_w<CC, 6>(p, a, h, grad, s);
        case 7: return launch_grad_w<CC, 7>(p, a, h, grad, s);
        case 8: return launch_grad_w<CC, 8>(p, a, h, grad, s);
        default: return HB_ERR_INVALID_ARG;
    }
}

int plan_set_spread_tuning(NufftPlan* p, int maxp, int bz, int by, int bx) {
    HB_REQUIRE(!p->pts_set, HB_ERR_STATE, "set the spread tuning before setpts");
    HB_REQUIRE(maxp >= 32 && maxp <= (1 << 16), HB_ERR_INVALID_ARG, "max candidates must be in [32, 65536]");
    const int b[3] = {bz, by, bx};
    HB_REQUIRE(bz * by * bx == 32, HB_ERR_INVALID_ARG, "warp block must hold 32 cells");
    for (int ax = 0; ax < 3; ++ax) {
        HB_REQUIRE(b[ax] >= 1 && (b[ax] & (b[ax] - 1)) == 0 && p->g.T[ax] % b[ax] == 0, HB_ERR_INVALID_ARG,
                   "warp block edges must be powers of two that tile the spread tile");
        HB_REQUIRE(p->g.T[ax] > 1 || b[ax] == 1, HB_ERR_INVALID_ARG, "unit axes take a block edge of 1");
    }
    p->maxp = maxp;
    p->maxp_auto = false;
    for (int ax = 0; ax < 3; ++ax) p->wb[ax] = b[ax];
    return HB_OK;
}

int plan_set_spread_kernel(NufftPlan* p, int kind, int transforms_per_cta) {
    HB_REQUIRE(!p->pts_set, HB_ERR_STATE, "set the spreading kernel before setpts");
    const int base = kind;
    HB_REQUIRE(base == HB_SPREAD_AUTO || base == HB_SPREAD_CELLS || base == HB_SPREAD_TRANSFORMS, HB_ERR_INVALID_ARG,
               "spreading kernel must be HB_SPREAD_AUTO, HB_SPREAD_CELLS or HB_SPREAD_TRANSFORMS");
    HB_REQUIRE(base != HB_SPREAD_TRANSFORMS || p->lc_ok, HB_ERR_INVALID_ARG,
               "this plan cannot spread with the transforms on the lanes (needs 8^3 / 16x32 tiles, width 4..8, "
               ">= 5 transforms, >= 2 tiles per axis)");
    HB_REQUIRE(transforms_per_cta == 0 || transforms_per_cta == 8 || transforms_per_cta == 16 || transforms_per_cta == 32,
               HB_ERR_INVALID_ARG, "transforms per CTA must be 0 (automatic), 8, 16 or 32");
    p->lc = base == HB_SPREAD_CELLS ? false : p->lc_ok;
    if (transforms_per_cta) p->lc_cc = transforms_per_cta;
    return HB_OK;
}

int plan_set_interp_tuning(NufftPlan* p, int transforms_per_group) {
    HB_REQUIRE(transforms_per_group == 0 || transforms_per_group == 1 || transforms_per_group == 2 ||
                   transforms_per_group == 4 || transforms_per_group == 8 || transforms_per_group == 16 ||
                   transforms_per_group == 32,
               HB_ERR_INVALID_ARG, "transforms per lane group must be 0 (automatic) or a power of two up to 32");
    p->interp_cc = transforms_per_group;
    return HB_OK;
}

int plan_set_interp_kernel(NufftPlan* p, int kind) {
    HB_REQUIRE(kind == HB_INTERP_AUTO || kind == HB_INTERP_GATHER || kind == HB_INTERP_STAGED, HB_ERR_INVALID_ARG,
               "interpolation kernel must be HB_INTERP_AUTO, HB_INTERP_GATHER or HB_INTERP_STAGED");
    HB_REQUIRE(kind != HB_INTERP_STAGED || p->st_ok, HB_ERR_INVALID_ARG,
               "staged interpolation needs a 3-D type-2 plan with kernel width 4..7");
    p->st = kind == HB_INTERP_STAGED;
    // points already set: build the staged kernel's job list now (setpts builds it otherwise)
    if (p->st && p->pts_set && !p->st_built) {
        HB_TRY(st_build_jobs(p, nullptr));
        HB_CUDA(cudaStreamSynchronize(nullptr));
    }
    return HB_OK;
}

int plan_coord_grad(NufftPlan* p, const float2* modes, const float2* h, float* grad, cudaStream_t s) {
    HB_REQUIRE(p->type == 2, HB_ERR_INVALID_ARG, "coordinate gradient needs a type-2 plan");
    HB_REQUIRE(p->pts_set, HB_ERR_STATE, "coordinate gradient called before setpts");
    HB_REQUIRE(p->kb.w <= 8, HB_ERR_INVALID_ARG, "coordinate gradient supports kernel widths up to 8");
    HB_REQUIRE(modes && grad && (h || p->g.M == 0), HB_ERR_INVALID_ARG, "null argument");
    if (p->g.M == 0) return HB_OK;
    float2* G = nullptr;
    HB_TRY(type2_grid(p, modes, &G, s));
    GridArgs a = grid_args(p);
    a.grid = G;
    switch (spread_cc(p->g)) {
        case 1: return launch_grad_cc<1>(p, a, h, grad, s);
        case 2: return launch_grad_cc<2>(p, a, h, grad, s);
        case 4: return launch_grad_cc<4>(p, a, h, grad, s);
        case 8: return launch_grad_cc<8>(p, a, h, grad, s);
        case 16: return launch_grad_cc<16>(p, a, h, grad, s);
        default: return launch_grad_cc<32>(p, a, h, grad, s);
    }
}

void plan_free(NufftPlan* p) {
    for (int ax = 0; ax < 3; ++ax) {
        fftlen_free(&p->fl[ax]);
        if (p->deapod[ax]) cudaFree(p->deapod[ax]);
        if (p->su[ax]) cudaFree(p->su[ax]);
        p->deapod[ax] = nullptr;
        p->su[ax] = nullptr;
    }
    if (p->X) cudaFree(p->X);
    if (p->Y) cudaFree(p->Y);
    if (p->foff) cudaFree(p->foff);
    p->foff = nullptr;
    if (p->perm) cudaFree(p->perm);
    if (p->inT) cudaFree(p->inT);
    if (p->bin_start) cudaFree(p->bin_start);
    if (p->extra) cudaFree(p->extra);
    if (p->extra_scratch) cudaFree(p->extra_scratch);
    p->extra_scratch = nullptr;
    if (p->d_err) cudaFree(p->d_err);
    for (int ax = 0; ax < 3; ++ax) {
        if (p->tmp_u[ax]) cudaFree(p->tmp_u[ax]);
        p->tmp_u[ax] = nullptr;
    }
    if (p->dense_parts) cudaFree(p->dense_parts);
    if (p->dense_scratch) cudaFree(p->dense_scratch);
    if (p->st_jobs) cudaFree(p->st_jobs);
    p->st_jobs = nullptr;
    p->n_st_jobs = p->st_cap = 0;
    p->dense_parts = nullptr;
    p->dense_scratch = nullptr;
    p->parts_cap = 0;
    p->scratch_cap = 0;
    for (int** q : {&p->tmp_binid, &p->tmp_rank, &p->tmp_count, &p->tmp_ecnt, &p->tmp_eoff, &p->tmp_sums}) {
        if (*q) cudaFree(*q);
        *q = nullptr;
    }
    p->tmp_cap = 0;
    p->X = p->Y = nullptr;
    p->perm = nullptr;
    p->inT = nullptr;
    p->bin_start = nullptr;
    p->extra = nullptr;
    p->d_err = nullptr;
}

}  // namespace hb
