// NUFFT plan internals (type 1 / type 2, 1-3 dimensions, complex64, Kaiser-Bessel).
//
// Internally every problem is 3-D with unit leading axes: a 2-D plan of [N1, N2] is
// [1, N1, N2]. Axis 0 is the slowest. A unit axis has one mode, one fine cell, tap width 1.
//
// Device data layout:
//   fine grid     X[nf0][nf1][nf2][C]   (transforms interleaved: one cell holds all C values)
//   pass buffer   Y[Nm0][nf1][nf2][C]   (the grid after/before the axis-0 transform)
//   sorted points su_a[M] (fine coordinates in [0, nf_a)), perm[M] (sorted -> caller index)
//   bins          bin_start[nbins+1]   (tiles of T0 x T1 x T2 cells; bins == tiles)
#pragma once

#include <stdint.h>

#include "fft.cuh"
#include "kbkernel.cuh"

namespace hb {

struct GridGeom {
    int dim;          // caller's dimensionality (1..3)
    int C;            // transforms (ntransf)
    int64_t Nm[3];    // modes per axis
    int nf[3];        // fine cells per axis
    int wa[3];        // taps per axis (1 on unit axes)
    int T[3];         // tile edge per axis
    int nb[3];        // tiles (bins) per axis
    float scale[3];   // nf / (2 pi), float32
    int64_t M;        // points (all frames)
    // frames: independent trajectories of one plan. Frame f owns fine grid block f (fgrid values),
    // bins f * ntf .. f * ntf + ntf - 1 and the points foff[f] .. foff[f+1] - 1 (caller and sorted
    // order alike: the bins are frame-major, so sorting keeps every frame's points together).
    int nfr;          // frames (1: a single trajectory)
    int64_t ntf;      // tiles (bins) per frame
    int64_t fgrid;    // fine grid values per frame (cells x C)
};

struct NufftPlan {
    int type = 1;
    int sign = 1;
    int method = HB_METHOD_DEFAULT;
    double sigma = 2.0;
    double beta = 0.0;
    GridGeom g{};
    KbPoly kb{};
    FftLen fl[3];
    float* deapod[3] = {nullptr, nullptr, nullptr};
    float2* X = nullptr;
    float2* Y = nullptr;
    size_t X_elems = 0, Y_elems = 0;
    // points
    int64_t M_cap = 0;
    float* su[3] = {nullptr, nullptr, nullptr};
    int* perm = nullptr;
    float2* inT = nullptr;  // type 1: [M][C] input with the transforms interleaved (caller point order)
    int* bin_start = nullptr;
    int64_t nbins = 0;
    // spread subproblems beyond the first chunk of each tile ({tile, chunk, extra chunks of the
    // tile, first entry of the tile}); each writes its partial tile to its scratch slot (slot =
    // entry), and a reduction adds a tile's slots into the grid in slot order
    int4* extra = nullptr;
    int64_t n_extra = 0;
    int64_t extra_cap = 0;
    float2* extra_scratch = nullptr;
    size_t extra_scratch_cap = 0;  // bytes
    int* d_err = nullptr;
    bool pts_set = false;
    // frames: grids are allocated for frames_cap frames; foff holds the current frames' point
    // offsets (device, g.nfr + 1 entries)
    int frames_cap = 1;
    int* foff = nullptr;
    int64_t foff_cap = 0;
    int64_t nbins_cap = 0;  // entries of the per-bin scratch (bin counts, subproblem counts)
    // setpts scratch, kept by the plan so that re-pointing it allocates nothing: per point
    // (grown with M) and per bin (allocated at the first setpts)
    float* tmp_u[3] = {nullptr, nullptr, nullptr};
    int* tmp_binid = nullptr;
    int* tmp_rank = nullptr;
    int64_t tmp_cap = 0;
    int* tmp_count = nullptr;
    int* tmp_ecnt = nullptr;
    int* tmp_eoff = nullptr;
    int* tmp_sums = nullptr;  // scan block sums
    // spreading knobs (autotuned): candidates per subproblem and the warp's cell block. Unless set
    // explicitly, the subproblem size is chosen at setpts from the number of points.
    int maxp = 4096;
    bool maxp_auto = true;
    int wb[3] = {2, 4, 4};
    // lanes-on-transforms spreading (k_spread_lc): usable for this plan's shape (lc_ok), chosen
    // (lc), its transform chunk; the parts of the dense tiles of the current points ({tile, part,
    // parts of the tile, first scratch slot of the tile}) and the scratch their partial tiles
    // go to (one tile of all transforms per part)
    bool lc = false;
    bool lc_ok = false;
    int lc_cc = 0;
    int interp_cc = 0;  // interpolation: transforms per lane group (0 = the spreading rule)
    int4* dense_parts = nullptr;
    int64_t n_parts = 0, parts_cap = 0;
    float2* dense_scratch = nullptr;
    size_t scratch_cap = 0;  // bytes
    // staged interpolation (k_interp_st, 3-D, widths 4..7): usable for this plan (st_ok), chosen
    // (st); the jobs of the current points ({tile, first sorted point, end, 0}), built at setpts
    bool st_ok = false;
    bool st = false;
    bool st_built = false;  // st_jobs match the current points
    int4* st_jobs = nullptr;
    int64_t n_st_jobs = 0, st_cap = 0;
    size_t device_bytes = 0;
};


// Arguments of the gridding kernels (spreading and interpolation).
struct GridArgs {
    GridGeom g;
    const float* su[3];
    const int* perm;
    const int* bin_start;
    const float2* inT;  // spread input [M][C], transforms interleaved, caller's point order
    float2* grid;       // [nf0][nf1][nf2][C]
    float2* out;        // interp output [C][M]
    const int* foff;    // frame point offsets [nfr + 1] (nullptr with one frame)
    const int4* extra;
    float2* extra_scratch;  // [entry][tile cell][C] partial tiles of the extra subproblems
    int maxp;
    KbPoly kb;
};

constexpr int kCoefFloats = kMaxWidth * (kMaxDeg + 1);

#ifdef __CUDACC__
// Frame of point s (caller or sorted index: both keep every frame's points contiguous). Empty
// frames are skipped: the last f with foff[f] <= s.
__device__ __forceinline__ int frame_of_point(const int* foff, int nfr, int64_t s) {
    if (nfr <= 1) return 0;
    int lo = 0, hi = nfr;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (foff[mid] <= s) lo = mid; else hi = mid;
    }
    return lo;
}
// Tile over all frames (frame-major) -> its frame; `tile` becomes the frame's own tile index.
__device__ __forceinline__ int split_frame_tile(const GridGeom& g, int& tile) {
    if (g.nfr <= 1) return 0;
    const int fr = (int)(tile / g.ntf);
    tile -= fr * (int)g.ntf;
    return fr;
}
#endif

// Type-1 spreading with the transforms on the lanes (spread_lc.cuh; instances in
// spread_lc{8,16,32}.cu) for plans with p->lc set, by transform chunk.
int spread_lc_cc8(const NufftPlan* p, const GridArgs& a, cudaStream_t s);
int spread_lc_cc16(const NufftPlan* p, const GridArgs& a, cudaStream_t s);
int spread_lc_cc32(const NufftPlan* p, const GridArgs& a, cudaStream_t s);

int plan_make(NufftPlan* p, int type, int dim, const int64_t* nmodes, int sign, int ntransf, float tol,
              int width, double upsampfac, int method);
int plan_setpts(NufftPlan* p, int64_t M, const float* c0, const float* c1, const float* c2, cudaStream_t s);
// Points of nframes frames at once: frame f has npts[f] (host) points, stored one frame after the
// other in c0 / c1 / c2. Grows the plan's grids to nframes frames when needed.
int plan_setpts_frames(NufftPlan* p, int nframes, const int64_t* npts, const float* c0, const float* c1,
                       const float* c2, cudaStream_t s);
int plan_execute(NufftPlan* p, const float2* in, float2* out, cudaStream_t s);
int plan_coord_grad(NufftPlan* p, const float2* modes, const float2* h, float* grad, cudaStream_t s);
int plan_set_spread_tuning(NufftPlan* p, int maxp, int bz, int by, int bx);
int plan_set_spread_kernel(NufftPlan* p, int kind, int transforms_per_cta);
int plan_set_interp_tuning(NufftPlan* p, int transforms_per_group);
int plan_set_interp_kernel(NufftPlan* p, int kind);

// Type-2 interpolation from staged regions of the fine grid (interp_st.cu). interp_st_jobs with
// jobs == nullptr counts the jobs (per tile in cnt, offsets in off, total in *n_jobs; syncs s);
// with a job array of jobs_cap >= *n_jobs entries it fills them.
int interp_st_max_points(int w);
int interp_st_jobs(const int* bin_start, int64_t ntiles, int w, int* cnt, int* off, int* sums, int4* jobs, int* n_jobs,
                   int64_t jobs_cap, cudaStream_t s);
int interp_st_run(const NufftPlan* p, const GridArgs& a, cudaStream_t s);
void plan_free(NufftPlan* p);

// Pieces reused by the Toeplitz kernel builder.
// `sums` (optional): ceil(n / 1024) ints of scratch; without it the scan allocates stream-ordered.
int exclusive_scan_int(const int* in, int* out, int64_t n, cudaStream_t s, int* sums = nullptr);

}  // namespace hb
