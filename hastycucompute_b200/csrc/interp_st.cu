// Type-2 interpolation from a staged region of the fine grid (3-D, widths 4..7).
//
// One CTA owns one tile of the fine grid (8^3 cells, the bin its points' first cells fall in) for
// 8 transforms, or one part of a dense tile's points. It copies the region the tile's footprints
// can reach -- the tile plus W-1 cells above it along every axis, wrapped at the grid edge -- into
// shared memory (cp.async, 16-byte pieces of 2 transforms), stages its points' tap weights, and
// then every group of 4 lanes (one point, 2 transforms per lane) gathers the point's W^3 cells
// from shared memory at compile-time offsets: no wrap or bounds logic in the gather.
//
// Bank layout: a cell is 8 transforms x 8 B = 64 B, half of the 128-byte bank window, and the
// region's row pitches are odd, so a cell's half of the banks is the parity of z + y + x. Every tap
// of a point keeps the parity of its first cell. A 16-byte load is served per quarter-warp (two lane
// groups), so a quarter-warp whose two groups hold points of opposite parity reads its two cells
// in one wavefront: the minimum four per warp load. The CTA orders its points into such pairs
// (even, odd) and runs the unmatched rest after them.
//
// The sums run in the order of the gathering kernel (per row the x taps, then the row weight
// w_z w_y), with the same tap weights, so both kernels give bit-identical samples.
#include <algorithm>

#include "fft2.cuh"
#include "kbkernel.cuh"
#include "nufft.cuh"
#include "timing.cuh"

namespace hb {

constexpr int kStCoils = 8;      // transforms per CTA
constexpr int kStThreads = 512;  // 16 warps x 8 lane groups

template <int W>
struct StShape {
    static constexpr int R = 8 + W - 1;  // region edge: the tile and the footprints' reach
    static constexpr int RP = R | 1;     // odd pitch of the y and x axes
    static constexpr int kRegionF2 = R * RP * RP * kStCoils;
    static constexpr int kMaxPts = W <= 6 ? 256 : 192;  // points per CTA (shared memory)
    static constexpr int kRecF = 24;                   // taps per point: z[8] | y[8] | x[8]
    static constexpr size_t smem_bytes() {
        return sizeof(float2) * (size_t)kRegionF2 + sizeof(float) * (size_t)(kCoefFloats + kMaxPts * kRecF) +
               sizeof(int) * (size_t)(3 * kMaxPts);
    }
};
static_assert(StShape<7>::smem_bytes() <= 227 * 1024, "staged region and points fit one CTA");
static_assert(StShape<4>::kMaxPts <= kStThreads, "one point per thread when ordering");

int interp_st_max_points(int w) { return w <= 6 ? StShape<6>::kMaxPts : StShape<7>::kMaxPts; }

// CTA blockIdx.x: job {tile, first sorted point, end}; blockIdx.y: transform chunk of 8
template <int W>
__global__ void __launch_bounds__(kStThreads, 1) k_interp_st(const GridArgs a, const int4* __restrict__ jobs) {
    using S = StShape<W>;
    constexpr int R = S::R, RP = S::RP;
    extern __shared__ float4 st_f4[];
    float2* region = reinterpret_cast<float2*>(st_f4);
    float* coef = reinterpret_cast<float*>(region + S::kRegionF2);
    float* rec = coef + kCoefFloats;
    int* rel = reinterpret_cast<int*>(rec + S::kMaxPts * S::kRecF);  // packed region-relative first cells
    int* pidx = rel + S::kMaxPts;                                    // caller's index of the point
    int* order = pidx + S::kMaxPts;                                  // visit order (parity pairs)
    __shared__ int s_cnt[2];
    const GridGeom& g = a.g;
    const int tid = threadIdx.x;
    const int4 job = jobs[blockIdx.x];
    int tile = job.x;
    const int k0 = job.y, n = job.z - job.y;
    const int cc0 = (int)blockIdx.y * kStCoils;
    const int fr = split_frame_tile(g, tile);
    const float2* const gridf = a.grid + fr * g.fgrid;
    const int tx = tile % g.nb[2], ty = (tile / g.nb[2]) % g.nb[1], tz = tile / (g.nb[2] * g.nb[1]);
    const int org0 = tz * 8, org1 = ty * 8, org2 = tx * 8;
    const int nf0 = g.nf[0], nf1 = g.nf[1], nf2 = g.nf[2];

    if (tid < 2) s_cnt[tid] = 0;
    for (int i = tid; i < kCoefFloats; i += kStThreads) coef[i] = (&a.kb.coef[0][0])[i];
    // the region: one warp per (z, y) row of R cells x 4 pieces of 2 transforms; every wrapped
    // coordinate needs at most two subtractions (org + r < 8 nb + 15 <= 3 nf)
    const bool vec = (g.C % 2) == 0;
    {
        const int warp = tid >> 5, lane = tid & 31;
        for (int row = warp; row < R * R; row += kStThreads / 32) {
            const int z = row / R, y = row - z * R;
            int gz = org0 + z, gy = org1 + y;
            if (gz >= nf0) gz -= nf0;
            if (gz >= nf0) gz -= nf0;
            if (gy >= nf1) gy -= nf1;
            if (gy >= nf1) gy -= nf1;
            const float2* srow = gridf + ((int64_t)gz * nf1 + gy) * nf2 * g.C + cc0;
            float2* drow = region + (z * RP + y) * RP * kStCoils;
            for (int i = lane; i < R * 4; i += 32) {
                const int x = i >> 2, pc = i & 3;
                int gx = org2 + x;
                if (gx >= nf2) gx -= nf2;
                if (gx >= nf2) gx -= nf2;
                const int c = cc0 + 2 * pc;
                const float2* src = srow + (int64_t)gx * g.C + 2 * pc;
                float2* dst = drow + x * kStCoils + 2 * pc;
                if (vec && c < g.C) {
                    cp_async16(dst, src);
                } else {
                    if (c < g.C) cp_async8(dst, src); else dst[0] = make_float2(0.f, 0.f);
                    if (c + 1 < g.C) cp_async8(dst + 1, src + 1); else dst[1] = make_float2(0.f, 0.f);
                }
            }
        }
    }
    cp_async_commit();
    __syncthreads();  // coef, counters

    // points: thread (q, axis) evaluates its axis's taps; the region-relative first cell is in
    // [0, 8) for the tile's own points (clamped, so a stray value cannot index past the region)
    for (int i = tid; i < 3 * n; i += kStThreads) {
        const int q = i / 3, ax = i - 3 * q;
        const int sidx = k0 + q;
        const float v = __fsub_rn(a.su[ax][sidx], a.kb.hw);
        const int ic = (int)ceilf(v);
        const float t = __fsub_rn((float)ic, v);
        const float sarg = fmaf(2.f, t, -1.f);
        const int nf = ax == 0 ? nf0 : (ax == 1 ? nf1 : nf2);
        int iw = ic;
        if (iw < 0) iw += nf;
        if (iw >= nf) iw -= nf;
        const int r = min(max(iw - (ax == 0 ? org0 : (ax == 1 ? org1 : org2)), 0), 7);
        float* rr = rec + q * S::kRecF + ax * 8;
#pragma unroll
        for (int d = 0; d < W; ++d) rr[d] = kb_tap(coef, a.kb.deg, d, sarg);
        reinterpret_cast<unsigned char*>(rel + q)[ax] = (unsigned char)r;
        if (ax == 0) pidx[q] = a.perm[sidx];
    }
    __syncthreads();
    // parity classes, then the visit order: pairs (even, odd), then the rest
    for (int q = tid; q < n; q += kStThreads) {
        const int pk = rel[q];
        const int par = ((pk & 0xff) + ((pk >> 8) & 0xff) + ((pk >> 16) & 0xff)) & 1;
        const int pos = atomicAdd(&s_cnt[par], 1);
        order[q] = pos | (par << 30);  // temporary: list position and parity
    }
    __syncthreads();
    {
        const int ne = s_cnt[0], no = s_cnt[1];
        const int m = min(ne, no);  // matched pairs
        const int o = tid < n ? order[tid] : 0;
        __syncthreads();
        if (tid < n) {
            const int par = o >> 30, i = o & 0x3fffffff;
            const int slot = i < m ? 2 * i + par : 2 * m + (par ? ne - m : 0) + (i - m);
            order[slot] = tid;
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // gathers: a group of 4 lanes = one point, each lane 2 transforms (16-byte loads, served per
    // quarter-warp: two points of opposite parity per quarter-warp, one wavefront)
    const int warp = tid >> 5, lane = tid & 31, grp = lane >> 2, c2 = lane & 3;
    const int cA = cc0 + 2 * c2;
    float2* outA = a.out + (int64_t)cA * g.M;
    float2* outB = outA + g.M;
    for (int base = 0; base < n; base += kStThreads / 4) {
        const int o = base + warp * 8 + grp;
        if (o >= n) continue;
        const int q = order[o];
        const int pk = rel[q];
        const int rz = pk & 0xff, ry = (pk >> 8) & 0xff, rx = (pk >> 16) & 0xff;
        const float* rq = rec + q * S::kRecF;
        float wx[W];
#pragma unroll
        for (int d = 0; d < W; ++d) wx[d] = rq[16 + d];
        const float4* p0 = reinterpret_cast<const float4*>(region + ((rz * RP + ry) * RP + rx) * kStCoils) + c2;
        float ar0 = 0.f, ai0 = 0.f, ar1 = 0.f, ai1 = 0.f;
#pragma unroll 1
        for (int dz = 0; dz < W; ++dz) {
            const float wzd = rq[dz];
#pragma unroll 2
            for (int dy = 0; dy < W; ++dy) {
                const float4* pr = p0 + (dz * RP + dy) * RP * (kStCoils / 2);
                float rr0 = 0.f, ri0 = 0.f, rr1 = 0.f, ri1 = 0.f;
#pragma unroll
                for (int dx = 0; dx < W; ++dx) {
                    const float4 v = pr[dx * (kStCoils / 2)];
                    rr0 = fmaf(wx[dx], v.x, rr0);
                    ri0 = fmaf(wx[dx], v.y, ri0);
                    rr1 = fmaf(wx[dx], v.z, rr1);
                    ri1 = fmaf(wx[dx], v.w, ri1);
                }
                const float wzy = wzd * rq[8 + dy];
                ar0 = fmaf(wzy, rr0, ar0);
                ai0 = fmaf(wzy, ri0, ai0);
                ar1 = fmaf(wzy, rr1, ar1);
                ai1 = fmaf(wzy, ri1, ai1);
            }
        }
        const int pj = pidx[q];
        if (cA < g.C) outA[pj] = make_float2(ar0, ai0);
        if (cA + 1 < g.C) outB[pj] = make_float2(ar1, ai1);
    }
}

// jobs per tile: ceil(points / P), 0 for an empty tile
__global__ void k_st_jobs_count(const int* bin_start, int64_t ntiles, int P, int* cnt) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int n = bin_start[t + 1] - bin_start[t];
    cnt[t] = (n + P - 1) / P;
}

// the tile's points split evenly over its jobs
__global__ void k_st_jobs_fill(const int* bin_start, const int* cnt, const int* off, int64_t ntiles, int4* jobs) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const int k = cnt[t], o = off[t], s0 = bin_start[t], n = bin_start[t + 1] - s0;
    for (int q = 0; q < k; ++q)
        jobs[o + q] = make_int4((int)t, s0 + (int)((int64_t)q * n / k), s0 + (int)((int64_t)(q + 1) * n / k), 0);
}

int interp_st_jobs(const int* bin_start, int64_t ntiles, int w, int* cnt, int* off, int* sums, int4* jobs, int* n_jobs,
                   int64_t jobs_cap, cudaStream_t s) {
    const int P = interp_st_max_points(w);
    const unsigned blocks = (unsigned)ceil_div(ntiles, 256);
    if (jobs == nullptr) {
        k_st_jobs_count<<<blocks, 256, 0, s>>>(bin_start, ntiles, P, cnt);
        HB_TRY(check_launch("k_st_jobs_count"));
        HB_TRY(exclusive_scan_int(cnt, off, ntiles, s, sums));
        HB_CUDA(cudaMemcpyAsync(n_jobs, off + ntiles, sizeof(int), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        return HB_OK;
    }
    HB_REQUIRE(*n_jobs <= jobs_cap, HB_ERR_INVALID_ARG, "staged interpolation job list too small");
    if (*n_jobs > 0) {
        k_st_jobs_fill<<<blocks, 256, 0, s>>>(bin_start, cnt, off, ntiles, jobs);
        HB_TRY(check_launch("k_st_jobs_fill"));
    }
    return HB_OK;
}

template <int W>
static int launch_st(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    using S = StShape<W>;
    HB_CUDA(cudaFuncSetAttribute(k_interp_st<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::smem_bytes()));
    TimedSection ts("interp", s);
    k_interp_st<W><<<dim3((unsigned)p->n_st_jobs, (unsigned)ceil_div(a.g.C, kStCoils)), kStThreads, S::smem_bytes(), s>>>(
        a, p->st_jobs);
    return check_launch("k_interp_st");
}

int interp_st_run(const NufftPlan* p, const GridArgs& a, cudaStream_t s) {
    if (p->n_st_jobs == 0) return HB_OK;
    switch (p->g.wa[2]) {
        case 4: return launch_st<4>(p, a, s);
        case 5: return launch_st<5>(p, a, s);
        case 6: return launch_st<6>(p, a, s);
        case 7: return launch_st<7>(p, a, s);
        default: set_error("staged interpolation takes widths 4..7"); return HB_ERR_INVALID_ARG;
    }
}

}  // namespace hb
