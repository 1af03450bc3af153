// Type-1 spreading with the transforms on the lanes.
//
// One CTA owns one tile of the fine grid (8x8x8 in 3-D, 16x32 in 2-D) for CC transforms. The 32
// lanes of a warp are G = 32/CC groups of CC transforms; every thread keeps 4 rows x 8 cells of
// its tile in registers for its one transform (64 accumulators): rows (2 z x 2 y) in 3-D, 4 y
// in 2-D, 8 consecutive x cells per row. A warp's block is 1 x-segment of 8 cells x 4 rows per
// group (groups take consecutive y rows).
//
// Candidate points (the tile's bin and its lower neighbours) pass through shared memory in
// double-buffered chunks: per point the CC values (cp.async) and its tile-relative weight rows
// along z, y and x (the kernel taps at the cells the footprint covers, zero elsewhere), so a
// visit multiplies whole rows with no per-cell range or index logic. A warp visits only the points
// whose footprint meets its block (ballots per 32 candidates, one per quarter of the block's 8 x
// cells). For a visited point every lane forms its 4 row products u_r = w_z w_y v and adds
// w_x[x] u_r to the 4 x 2 cells of each quarter of the block that the footprint touches (the
// multiply-adds of the other quarters would add zero weights).
//
// Dense tiles (more candidates than a subproblem holds, maxp) are spread in ceil(total / maxp)
// parts, one CTA each, however many that is, so the k-space centre of radial and spiral
// trajectories spreads over the whole GPU; each part writes its partial tile (all transforms) to a
// scratch slot held by the plan, and a second kernel sums a tile's partial tiles in part order and
// stores the cells. No atomics anywhere; every cell is written exactly once, the sum order is
// fixed, and no sequential FP32 sum runs over more than maxp candidates.
#pragma once

#include <algorithm>

#include "fft2.cuh"
#include "nufft.cuh"
#include "timing.cuh"

namespace hb {

template <int CC, bool D3>
struct LcShape {
    static constexpr int G = 32 / CC;  // lane groups per warp
    static constexpr int RZ = D3 ? 2 : 1;
    static constexpr int RY = D3 ? 2 : 4;
    static constexpr int T0 = D3 ? 8 : 1, T1 = D3 ? 8 : 16, T2 = D3 ? 8 : 32;
    static constexpr int NZB = T0 / RZ, NYB = T1 / (G * RY), NXS = T2 / 8;
    static constexpr int WARPS = NZB * NYB * NXS;
    static constexpr int THREADS = WARPS * 32;
    static constexpr int CELLS = T0 * T1 * T2;
    // weight floats per staged point: tile-relative rows wz[T0] (3-D) | wy[T1] | wx[T2]
    static constexpr int OY = D3 ? T0 : 0, OX = OY + T1;
    static constexpr int kRec = OX + T2;
    // candidates staged per chunk: the 32-transform 3-D CTA is alone on its SM (registers), so it
    // takes long chunks (fewer barriers, even warp loads); the others keep several per SM
    static constexpr int kLcChunk = (CC == 32 && D3) ? 256 : 128;
    // staging buffer: values float2[chunk][CC] | weights float[chunk][kRec] | packed first cells
    static constexpr int kValF = kLcChunk * CC * 2;
    static constexpr int kBufF = kValF + kLcChunk * kRec + kLcChunk;
    static size_t smem_bytes() { return sizeof(float) * (size_t)(kCoefFloats + 2 * kBufF); }
};
static_assert(LcShape<32, true>::kRec % 4 == 0 && LcShape<32, false>::kRec % 4 == 0, "16-byte weight rows");
static_assert(LcShape<32, true>::THREADS == 512 && LcShape<8, true>::THREADS == 128, "tile shape");
static_assert(LcShape<32, false>::THREADS == 512 && LcShape<8, false>::THREADS == 128, "tile shape");

// acc[r][X0 + x] += wx[x] * u_r, x < 4
template <int X0>
__device__ __forceinline__ void lc_half(float (&ar)[4][8], float (&ai)[4][8], const float4 wx, const float (&ur)[4],
                                        const float (&ui)[4]) {
    const float w[4] = {wx.x, wx.y, wx.z, wx.w};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            ar[r][X0 + x] = fmaf(w[x], ur[r], ar[r][X0 + x]);
            ai[r][X0 + x] = fmaf(w[x], ui[r], ai[r][X0 + x]);
        }
    }
}

// acc[r][X0 + x] += w_x * u_r, x < 2 (a quarter of the block's 8 cells)
template <int X0>
__device__ __forceinline__ void lc_quarter(float (&ar)[4][8], float (&ai)[4][8], const float w0, const float w1,
                                           const float (&ur)[4], const float (&ui)[4]) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ar[r][X0] = fmaf(w0, ur[r], ar[r][X0]);
        ai[r][X0] = fmaf(w0, ui[r], ai[r][X0]);
        ar[r][X0 + 1] = fmaf(w1, ur[r], ar[r][X0 + 1]);
        ai[r][X0 + 1] = fmaf(w1, ui[r], ai[r][X0 + 1]);
    }
}

// A visit's operands: the row products u_r = w_z w_y v of staged point q for this lane's transform
// and rows, and the x weights of the warp's two halves of 4 cells
template <int CC, bool D3>
__device__ __forceinline__ void lc_prep(const float2* bval, const float* bwt, int q, int coil, int z0, int y0g, int x0,
                                        float (&ur)[4], float (&ui)[4], float4& x0w, float4& x1w) {
    using S = LcShape<CC, D3>;
    const float2 v = bval[q * CC + coil];
    const float* rec = bwt + q * S::kRec;
    float rw[4];
    if constexpr (D3) {
        const float2 wz2 = *reinterpret_cast<const float2*>(rec + z0);
        const float2 wy2 = *reinterpret_cast<const float2*>(rec + S::OY + y0g);
        rw[0] = wz2.x * wy2.x;
        rw[1] = wz2.x * wy2.y;
        rw[2] = wz2.y * wy2.x;
        rw[3] = wz2.y * wy2.y;
    } else {
        const float4 wy4 = *reinterpret_cast<const float4*>(rec + S::OY + y0g);
        rw[0] = wy4.x;
        rw[1] = wy4.y;
        rw[2] = wy4.z;
        rw[3] = wy4.w;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ur[r] = rw[r] * v.x;
        ui[r] = rw[r] * v.y;
    }
    const float4* wx = reinterpret_cast<const float4*>(rec + S::OX + x0);
    x0w = wx[0];
    x1w = wx[1];
}

// parts == nullptr: one CTA per tile (blockIdx.x), storing the tile; tiles with more than maxp
// candidates are left to the parts launch. Otherwise CTA blockIdx.x spreads part e.y of e.z of
// tile e.x (e = parts[blockIdx.x]) into scratch slot e.w + e.y ([slot][cell][C]).
template <int CC, int W, bool D3>
__global__ void __launch_bounds__(LcShape<CC, D3>::THREADS)
    k_spread_lc(const GridArgs a, const int4* __restrict__ parts, float2* __restrict__ scratch) {
    using S = LcShape<CC, D3>;
    extern __shared__ float4 sm_f4[];
    float* coef = reinterpret_cast<float*>(sm_f4);
    float* region = coef + kCoefFloats;
    __shared__ int s_start[8], s_pref[9], s_nbin;
    const GridGeom& g = a.g;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = lane / CC, coil = lane % CC;

    const int4 job = parts ? parts[blockIdx.x] : make_int4((int)blockIdx.x, 0, 1, 0);
    int tile = job.x;
    const int part = job.y, K = job.z;
    const int fr = split_frame_tile(g, tile);
    const int fbin = fr * (int)g.ntf;
    float2* const gridf = a.grid + fr * g.fgrid;
    const int tx = tile % g.nb[2], ty = (tile / g.nb[2]) % g.nb[1], tz = tile / (g.nb[2] * g.nb[1]);
    const int org0 = tz * S::T0, org1 = ty * S::T1, org2 = tx * S::T2;
    const int nf1 = g.nf[1], nf2 = g.nf[2];

    // this warp's block and this group's rows
    const int xs = warp % S::NXS, yb = (warp / S::NXS) % S::NYB, zb = warp / (S::NXS * S::NYB);
    const int x0 = xs * 8, z0 = zb * S::RZ, y0w = yb * S::G * S::RY;
    const int y0g = y0w + grp * S::RY;
    constexpr int WZ = D3 ? W : 1;

    for (int i = tid; i < kCoefFloats; i += S::THREADS) coef[i] = (&a.kb.coef[0][0])[i];
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
    if (!parts) {
        if (total > a.maxp) return;  // the parts launch spreads this tile
        if (total == 0) {
            if (blockIdx.y != 0) return;
            // no point reaches the tile: 16-byte zero stores (a tile row of T2 cells x C values is
            // contiguous and 16-byte aligned: T2 and the tile origin are multiples of 8)
            const int rowf4 = (S::T2 * g.C) >> 1;
            const int nrow = S::T0 * S::T1;
            for (int i = tid; i < nrow * rowf4; i += S::THREADS) {
                const int r = i / rowf4, c4 = i - r * rowf4;
                const int zz = r / S::T1, yy = r - zz * S::T1;
                float4* dst = reinterpret_cast<float4*>(
                    gridf + (((int64_t)(org0 + zz) * nf1 + (org1 + yy)) * nf2 + org2) * g.C);
                dst[c4] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
            return;
        }
    }
    const int k_begin = (int)((int64_t)part * total / K);
    const int k_end = (int)((int64_t)(part + 1) * total / K);
    const float hw = a.kb.hw;
    const bool vec = (g.C % 2) == 0;

    // candidates visited interleaved across the tile's bins (8 segments, k -> segment k % 8)
    const int seg_len = total >> 3, seg_rem = total & 7;
    auto sorted_index = [&](int k0) -> int {
        const int sgm = k0 & 7;
        const int k = sgm * seg_len + min(sgm, seg_rem) + (k0 >> 3);
        int b = 0;
#pragma unroll
        for (int j = 1; j < 8; ++j) b += (j < nbin && s_pref[j] <= k) ? 1 : 0;
        return s_start[b] + (k - s_pref[b]);
    };

    // Stages candidates base .. base+n-1: thread (q, axis) finds candidate q's sorted index once,
    // folds all three coordinates to tile-relative first cells, and -- only when the footprint
    // reaches the tile along every axis (about half of the lower neighbours' points do not) --
    // writes its axis's weights and a third of the point's CC values (cp.async). A point that
    // misses the tile is marked so no warp visits it.
    auto stage = [&](int base, int cc0, float* buf) {
        const int n = min(S::kLcChunk, k_end - base);
        float2* bval = reinterpret_cast<float2*>(buf);
        float* bwt = buf + S::kValF;
        unsigned char* brel = reinterpret_cast<unsigned char*>(bwt + S::kLcChunk * S::kRec);
        constexpr int CP = CC / 2;               // 16-byte pieces of a point's values
        constexpr int PPA = (CP + 2) / 3;        // pieces per axis thread
        for (int i = tid; i < 3 * n; i += S::THREADS) {
            const int q = i / 3, ax = i - 3 * q;
            const int sidx = sorted_index(base + q);
            int rel[3];
            bool reach = true;
#pragma unroll
            for (int a3 = 0; a3 < 3; ++a3) {
                rel[a3] = 0;
                if (a3 == 0 && !D3) continue;
                const int T = a3 == 0 ? S::T0 : (a3 == 1 ? S::T1 : S::T2);
                const int nf = g.nf[a3];
                int iw = (int)ceilf(__fsub_rn(a.su[a3][sidx], hw));
                if (iw < 0) iw += nf;
                if (iw >= nf) iw -= nf;
                int r = iw - (a3 == 0 ? org0 : (a3 == 1 ? org1 : org2));
                if (r < 0) r += nf;
                if (r >= T) r -= nf;  // a footprint reaching the tile from below starts at -(W-1) .. -1
                rel[a3] = r;
                reach = reach && r >= -(W - 1);
            }
            if (ax == 0)
                *reinterpret_cast<int*>(brel + q * 4) =
                    reach ? (rel[0] + 16) | ((rel[1] + 16) << 8) | ((rel[2] + 16) << 16) : 0;
            if (!reach) continue;
            if (D3 || ax != 0) {
                // this axis's tile-relative weight row: the W taps at cells rel .. rel+W-1 inside
                // the tile, zero elsewhere
                const float v = __fsub_rn(a.su[ax][sidx], hw);
                const float sarg = fmaf(2.f, __fsub_rn(ceilf(v), v), -1.f);
                float t[W];
#pragma unroll
                for (int d = 0; d < W; ++d) t[d] = kb_tap(coef, a.kb.deg, d, sarg);
                const int T = ax == 0 ? S::T0 : (ax == 1 ? S::T1 : S::T2);
                float* wt = bwt + q * S::kRec + (ax == 0 ? 0 : (ax == 1 ? S::OY : S::OX));
                const int r = ax == 0 ? rel[0] : (ax == 1 ? rel[1] : rel[2]);
                for (int c = 0; c < T; c += 4) *reinterpret_cast<float4*>(wt + c) = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int d = 0; d < W; ++d) {
                    const int c = r + d;
                    if (c >= 0 && c < T) wt[c] = t[d];
                }
            }
            const float2* src = a.inT + (int64_t)a.perm[sidx] * g.C;
            for (int pc = ax * PPA; pc < min(CP, (ax + 1) * PPA); ++pc) {
                const int c = 2 * pc, cg = cc0 + c;
                float2* dst = bval + q * CC + c;
                if (vec && cg < g.C) {
                    cp_async16(dst, src + cg);
                } else {
                    if (cg < g.C) cp_async8(dst, src + cg); else dst[0] = make_float2(0.f, 0.f);
                    if (cg + 1 < g.C) cp_async8(dst + 1, src + cg + 1); else dst[1] = make_float2(0.f, 0.f);
                }
            }
        }
    };

    {
        const int cc0 = (int)blockIdx.y * CC;  // this CTA's transform chunk
        float ar[4][8], ai[4][8];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int x = 0; x < 8; ++x) ar[r][x] = ai[r][x] = 0.f;
        const int nch = (k_end - k_begin + S::kLcChunk - 1) / S::kLcChunk;
        if (nch > 0) stage(k_begin, cc0, region);
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        for (int it = 0; it < nch; ++it) {
            const int base = k_begin + it * S::kLcChunk;
            if (it + 1 < nch) stage(base + S::kLcChunk, cc0, region + ((it + 1) & 1) * S::kBufF);
            cp_async_commit();
            {
                const int n = min(S::kLcChunk, k_end - base);
                const float* buf = region + (it & 1) * S::kBufF;
                const float2* bval = reinterpret_cast<const float2*>(buf);
                const float* bwt = buf + S::kValF;
                const int* brel = reinterpret_cast<const int*>(bwt + S::kLcChunk * S::kRec);
                for (int q0 = 0; q0 < n; q0 += 32) {
                    const int qq = q0 + lane;
                    bool h0 = false, h1 = false, h2 = false, h3 = false;
                    if (qq < n) {
                        const int pk = brel[qq];
                        const int rz = (pk & 0xff) - 16, ry = ((pk >> 8) & 0xff) - 16, rx = ((pk >> 16) & 0xff) - 16;
                        const bool zy = rz <= z0 + S::RZ - 1 && rz + WZ - 1 >= z0 && ry <= y0w + S::G * S::RY - 1 &&
                                        ry + W - 1 >= y0w;
                        // the quarters of the block's 8 x cells the footprint rx .. rx+W-1 covers
                        h0 = zy && rx <= x0 + 1 && rx + W - 1 >= x0;
                        h1 = zy && rx <= x0 + 3 && rx + W - 1 >= x0 + 2;
                        h2 = zy && rx <= x0 + 5 && rx + W - 1 >= x0 + 4;
                        h3 = zy && rx <= x0 + 7 && rx + W - 1 >= x0 + 6;
                    }
                    const unsigned m0 = __ballot_sync(0xffffffffu, h0), m1 = __ballot_sync(0xffffffffu, h1);
                    const unsigned m2 = __ballot_sync(0xffffffffu, h2), m3 = __ballot_sync(0xffffffffu, h3);
                    unsigned bits = m0 | m1 | m2 | m3;
                    // visits two at a time: both points' loads and row products are issued before
                    // either's multiply-adds, so one visit's shared-memory latency hides behind the
                    // other's arithmetic
                    while (bits) {
                        const int ia = __ffs(bits) - 1;
                        bits &= bits - 1;
                        const bool two = bits != 0;
                        const int ib = two ? __ffs(bits) - 1 : ia;
                        if (two) bits &= bits - 1;
                        float ura[4], uia[4], urb[4], uib[4];
                        float4 xa0, xa1, xb0, xb1;
                        lc_prep<CC, D3>(bval, bwt, q0 + ia, coil, z0, y0g, x0, ura, uia, xa0, xa1);
                        lc_prep<CC, D3>(bval, bwt, q0 + ib, coil, z0, y0g, x0, urb, uib, xb0, xb1);
                        // only the quarters the footprint covers (the others would add zero weights)
                        if ((m0 >> ia) & 1u) lc_quarter<0>(ar, ai, xa0.x, xa0.y, ura, uia);
                        if ((m1 >> ia) & 1u) lc_quarter<2>(ar, ai, xa0.z, xa0.w, ura, uia);
                        if ((m2 >> ia) & 1u) lc_quarter<4>(ar, ai, xa1.x, xa1.y, ura, uia);
                        if ((m3 >> ia) & 1u) lc_quarter<6>(ar, ai, xa1.z, xa1.w, ura, uia);
                        if (two) {
                            if ((m0 >> ib) & 1u) lc_quarter<0>(ar, ai, xb0.x, xb0.y, urb, uib);
                            if ((m1 >> ib) & 1u) lc_quarter<2>(ar, ai, xb0.z, xb0.w, urb, uib);
                            if ((m2 >> ib) & 1u) lc_quarter<4>(ar, ai, xb1.x, xb1.y, urb, uib);
                            if ((m3 >> ib) & 1u) lc_quarter<6>(ar, ai, xb1.z, xb1.w, urb, uib);
                        }
                    }
                }
            }
            cp_async_wait_all();
            __syncthreads();
        }
        const bool coil_ok = cc0 + coil < g.C;
        float2* dst = parts ? scratch + (int64_t)(job.w + part) * S::CELLS * g.C : nullptr;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int z = z0 + (D3 ? (r >> 1) : 0), y = y0g + (D3 ? (r & 1) : r);
            float2* row = parts ? dst + ((int64_t)(z * S::T1 + y) * S::T2 + x0) * g.C + cc0 + coil
                                : gridf + (((int64_t)(org0 + z) * nf1 + (org1 + y)) * nf2 + org2 + x0) * g.C + cc0 + coil;
            if (coil_ok) {
#pragma unroll
                for (int x = 0; x < 8; ++x) row[(int64_t)x * g.C] = make_float2(ar[r][x], ai[r][x]);
            }
        }
    }
}

// Sums the partial tiles of the dense tiles: CTA blockIdx.x takes entry e = parts[blockIdx.x] and
// sums the e.z slots e.w .. e.w + e.z - 1 of tile e.x, in slot order, for its share (part e.y of
// e.z) of the tile's cells x transforms, then stores them in the fine grid.
template <bool D3>
__global__ void __launch_bounds__(256) k_spread_lc_reduce(const GridArgs a, const int4* __restrict__ parts,
                                                          const float2* __restrict__ scratch) {
    using S = LcShape<32, D3>;
    const GridGeom& g = a.g;
    const int4 e = parts[blockIdx.x];
    int tile = e.x;
    const int fr = split_frame_tile(g, tile);
    float2* const gridf = a.grid + fr * g.fgrid;
    const int tx = tile % g.nb[2], ty = (tile / g.nb[2]) % g.nb[1], tz = tile / (g.nb[2] * g.nb[1]);
    const int org0 = tz * S::T0, org1 = ty * S::T1, org2 = tx * S::T2;
    const int64_t E = (int64_t)S::CELLS * g.C;
    const int64_t i0 = e.y * E / e.z, i1 = (e.y + 1) * E / e.z;
    const float2* src = scratch + (int64_t)e.w * E;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        float2 sum = src[i];
        for (int q = 1; q < e.z; ++q) {
            const float2 v = src[(int64_t)q * E + i];
            sum.x += v.x;
            sum.y += v.y;
        }
        const int64_t cell = i / g.C;
        const int c = (int)(i - cell * g.C);
        const int x = (int)(cell % S::T2), y = (int)((cell / S::T2) % S::T1), z = (int)(cell / (S::T2 * S::T1));
        gridf[(((int64_t)(org0 + z) * g.nf[1] + (org1 + y)) * g.nf[2] + org2 + x) * g.C + c] = sum;
    }
}

// Host launch: one CTA per tile for the tiles within one subproblem, then (dense tiles) one CTA per
// part into scratch and the reduction of the parts.
template <int CC, int W, bool D3>
inline int launch_spread_lc(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    using S = LcShape<CC, D3>;
    auto kern = k_spread_lc<CC, W, D3>;
    const size_t smem = S::smem_bytes();
    HB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    {
        TimedSection ts("spread", s);
        kern<<<dim3((unsigned)p->nbins, (unsigned)ceil_div(a.g.C, CC)), S::THREADS, smem, s>>>(a, nullptr, nullptr);
        HB_TRY(check_launch("k_spread_lc"));
    }
    if (p->n_parts > 0) {
        TimedSection ts("spread_dense", s);
        kern<<<dim3((unsigned)p->n_parts, (unsigned)ceil_div(a.g.C, CC)), S::THREADS, smem, s>>>(
            a, p->dense_parts, p->dense_scratch);
        HB_TRY(check_launch("k_spread_lc(parts)"));
        k_spread_lc_reduce<D3><<<(unsigned)p->n_parts, 256, 0, s>>>(a, p->dense_parts, p->dense_scratch);
        HB_TRY(check_launch("k_spread_lc_reduce"));
    }
    return HB_OK;
}

template <int CC, bool D3>
inline int launch_spread_lc_w(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    switch (p->g.wa[2]) {
        case 4: return launch_spread_lc<CC, 4, D3>(p, a, s);
        case 5: return launch_spread_lc<CC, 5, D3>(p, a, s);
        case 6: return launch_spread_lc<CC, 6, D3>(p, a, s);
        case 7: return launch_spread_lc<CC, 7, D3>(p, a, s);
        default: return launch_spread_lc<CC, 8, D3>(p, a, s);
    }
}

}  // namespace hb
