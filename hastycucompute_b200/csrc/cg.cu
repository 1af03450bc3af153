// Conjugate-gradient vector steps with device-resident scalars and FP64, fixed-order dots.
//
// Restates conjugate_gradient of cpp/corelib/lib/op/cg.cppm:122-184 (TorchScript step at
// :139-150, loop and break test at :166-178):
//   r = b - A x; p = r; rzold = Re<r,r>
//   loop: if sqrt(rzold) < tol: break
//         Ap = A p; alpha = rzold / Re<p,Ap>; x += alpha p; r -= alpha Ap
//         rznew = Re<r,r>; p = r + (rznew / rzold) p; rzold = rznew
// The break test runs on the device at the start of each step; once it fires the step leaves
// x, r, p untouched, so a fixed number of captured steps reproduces the early exit.
//
// Every reduction is: per-block partial sums in double over a grid-stride range (fixed grid
// for a given n), then the last block to finish adds the partials in block order.
#include <algorithm>

#include "common.cuh"
#include "timing.cuh"

namespace hb {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 1184;  // 8 per SM

struct CgState {
    double rzold;
    double pAp;
    double alpha;
    double beta;
    double tol;
    long long iters;
    int run;                // 1 while the loop has not broken
    unsigned int counter;   // last-block detection
    double partial[kRedMaxBlocks];
};

static int red_blocks(int64_t n) {
    int64_t b = ceil_div(std::max<int64_t>(n, 1), (int64_t)kRedThreads * 4);
    return (int)std::min<int64_t>(b, kRedMaxBlocks);
}

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[i];
    }
    __syncthreads();
    return t;  // valid in thread 0
}

// Publishes this block's partial; returns true in the block that finished last, which then
// holds the ordered total in *total (thread 0).
__device__ __forceinline__ bool finish_reduction(double part, double* partial, unsigned int* counter, double* total) {
    __shared__ double sh[kRedThreads / 32];
    __shared__ bool is_last;
    const double bt = block_sum(part, sh);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = bt;
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double acc = 0;
    const volatile double* vp = partial;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) acc += vp[i];
    // ordered: thread i holds blocks i, i+256, ...; the tree below is fixed
    const double tot = block_sum(acc, sh);
    if (threadIdx.x == 0) {
        *total = tot;
        *counter = 0u;
    }
    return true;
}

// Every kernel below serves gridDim.y independent systems (frames): system f uses vector segment
// [f*n, (f+1)*n) and state st[f]; one system is gridDim.y == 1.
__global__ void __launch_bounds__(kRedThreads) k_cg_init(int64_t n, const float2* __restrict__ b, const float2* __restrict__ Ax,
                                                          float2* __restrict__ r, float2* __restrict__ p, CgState* st, double tol) {
    const int64_t fo = (int64_t)blockIdx.y * n;
    b += fo;
    Ax += fo;
    r += fo;
    p += fo;
    st += blockIdx.y;
    double part = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = csub(b[i], Ax[i]);
        r[i] = v;
        p[i] = v;
        part += (double)v.x * v.x + (double)v.y * v.y;
    }
    double tot;
    if (finish_reduction(part, st->partial, &st->counter, &tot) && threadIdx.x == 0) {
        st->rzold = tot;
        st->tol = tol;
        st->iters = 0;
        st->run = 1;
        st->alpha = 0;
        st->beta = 0;
        st->pAp = 0;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_cg_alpha(int64_t n, const float2* __restrict__ p, const float2* __restrict__ Ap,
                                                           CgState* st) {
    const int64_t fo = (int64_t)blockIdx.y * n;
    p += fo;
    Ap += fo;
    st += blockIdx.y;
    double part = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 a = p[i], c = Ap[i];
        part += (double)a.x * c.x + (double)a.y * c.y;
    }
    double tot;
    if (finish_reduction(part, st->partial, &st->counter, &tot) && threadIdx.x == 0) {
        const int run = st->run && !(sqrt(st->rzold) < st->tol);
        st->run = run;
        st->pAp = tot;
        st->alpha = run ? st->rzold / tot : 0.0;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_cg_update(int64_t n, float2* __restrict__ x, float2* __restrict__ r,
                                                            const float2* __restrict__ p, const float2* __restrict__ Ap,
                                                            CgState* st) {
    const int64_t fo = (int64_t)blockIdx.y * n;
    x += fo;
    r += fo;
    p += fo;
    Ap += fo;
    st += blockIdx.y;
    if (!st->run) return;
    const float alpha = (float)st->alpha;
    double part = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 pv = p[i], av = Ap[i];
        float2 xv = x[i], rv = r[i];
        xv.x = fmaf(alpha, pv.x, xv.x);
        xv.y = fmaf(alpha, pv.y, xv.y);
        rv.x = fmaf(-alpha, av.x, rv.x);
        rv.y = fmaf(-alpha, av.y, rv.y);
        x[i] = xv;
        r[i] = rv;
        part += (double)rv.x * rv.x + (double)rv.y * rv.y;
    }
    double tot;
    if (finish_reduction(part, st->partial, &st->counter, &tot) && threadIdx.x == 0) {
        st->beta = tot / st->rzold;
        st->rzold = tot;
        st->iters += 1;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_cg_dir(int64_t n, const float2* __restrict__ r, float2* __restrict__ p,
                                                         const CgState* st) {
    const int64_t fo = (int64_t)blockIdx.y * n;
    r += fo;
    p += fo;
    st += blockIdx.y;
    if (!st->run) return;
    const float beta = (float)st->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 rv = r[i];
        float2 pv = p[i];
        pv.x = fmaf(beta, pv.x, rv.x);
        pv.y = fmaf(beta, pv.y, rv.y);
        p[i] = pv;
    }
}

// ---- preconditioned / restarted CG (cpp/corelib/lib/op/cg.cppm:16-119) -------------------------
//   r = b - A x; z = P r; p = z; rzold = Re<r,z>; resid = sqrt(rzold)
//   loop: if resid < tol: break
//         Ap = A p; alpha = rzold / Re<p,Ap>; x += alpha p; r -= alpha Ap          (step 1)
//         z = P r                                                                   (caller)
//         rznew = Re<r,z>; p = restart ? z : z + (rznew / rzold) p; rzold = rznew  (step 2)
// Step 1 reuses k_cg_alpha (break test, Re<p,Ap>, alpha); the break leaves every vector as is.
__global__ void k_pcg_residual(int64_t n, const float2* __restrict__ b, const float2* __restrict__ Ax,
                               float2* __restrict__ r) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = csub(b[i], Ax[i]);
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_start(int64_t n, const float2* __restrict__ r,
                                                            const float2* __restrict__ z, float2* __restrict__ p,
                                                            CgState* st, double tol) {
    double part = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 rv = r[i], zv = z[i];
        p[i] = zv;
        part += (double)rv.x * zv.x + (double)rv.y * zv.y;
    }
    double tot;
    if (finish_reduction(part, st->partial, &st->counter, &tot) && threadIdx.x == 0) {
        st->rzold = tot;
        st->tol = tol;
        st->iters = 0;
        st->run = 1;
        st->alpha = 0;
        st->beta = 0;
        st->pAp = 0;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_xr(int64_t n, float2* __restrict__ x, float2* __restrict__ r,
                                                         const float2* __restrict__ p, const float2* __restrict__ Ap,
                                                         const CgState* st) {
    if (!st->run) return;
    const float alpha = (float)st->alpha;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 pv = p[i], av = Ap[i];
        float2 xv = x[i], rv = r[i];
        xv.x = fmaf(alpha, pv.x, xv.x);
        xv.y = fmaf(alpha, pv.y, xv.y);
        rv.x = fmaf(-alpha, av.x, rv.x);
        rv.y = fmaf(-alpha, av.y, rv.y);
        x[i] = xv;
        r[i] = rv;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_rz(int64_t n, const float2* __restrict__ r,
                                                         const float2* __restrict__ z, CgState* st) {
    if (!st->run) return;
    double part = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 rv = r[i], zv = z[i];
        part += (double)rv.x * zv.x + (double)rv.y * zv.y;
    }
    double tot;
    if (finish_reduction(part, st->partial, &st->counter, &tot) && threadIdx.x == 0) {
        st->beta = tot / st->rzold;
        st->rzold = tot;
        st->iters += 1;
    }
}

__global__ void __launch_bounds__(kRedThreads) k_pcg_dir(int64_t n, const float2* __restrict__ z, float2* __restrict__ p,
                                                          const CgState* st, int restart) {
    if (!st->run) return;
    const float beta = restart ? 0.f : (float)st->beta;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 zv = z[i];
        float2 pv = p[i];
        pv.x = restart ? zv.x : fmaf(beta, pv.x, zv.x);
        pv.y = restart ? zv.y : fmaf(beta, pv.y, zv.y);
        p[i] = pv;
    }
}

struct DotScratch {
    unsigned int counter;
    double partial[kRedMaxBlocks];
};

__global__ void __launch_bounds__(kRedThreads) k_vdot_real(int64_t n, const float2* __restrict__ a, const float2* __restrict__ b,
                                                            DotScratch* sc, double* out) {
    double part = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 u = a[i], v = b[i];
        part += (double)u.x * v.x + (double)u.y * v.y;
    }
    double tot;
    if (finish_reduction(part, sc->partial, &sc->counter, &tot) && threadIdx.x == 0) *out = tot;
}

size_t cg_state_bytes() { return sizeof(CgState); }
size_t cgb_state_bytes(int64_t nframes) { return sizeof(CgState) * (size_t)std::max<int64_t>(nframes, 1); }

int cgb_init(int64_t n, int64_t nf, const void* b, const void* Ax, void* r, void* p, void* state, double tol,
             cudaStream_t s) {
    HB_REQUIRE(n >= 1 && nf >= 1 && nf <= 65535, HB_ERR_INVALID_ARG, "n >= 1 and 1 <= nframes <= 65535");
    HB_REQUIRE(b && Ax && r && p && state, HB_ERR_INVALID_ARG, "null argument");
    HB_CUDA(cudaMemsetAsync(state, 0, sizeof(CgState) * (size_t)nf, s));
    dim3 grid(red_blocks(n), (unsigned)nf);
    k_cg_init<<<grid, kRedThreads, 0, s>>>(n, (const float2*)b, (const float2*)Ax, (float2*)r, (float2*)p,
                                          (CgState*)state, tol);
    return check_launch("k_cg_init (frames)");
}

int cgb_step(int64_t n, int64_t nf, void* x, void* r, void* p, const void* Ap, void* state, cudaStream_t s) {
    HB_REQUIRE(n >= 1 && nf >= 1 && nf <= 65535, HB_ERR_INVALID_ARG, "n >= 1 and 1 <= nframes <= 65535");
    HB_REQUIRE(x && r && p && Ap && state, HB_ERR_INVALID_ARG, "null argument");
    dim3 grid(red_blocks(n), (unsigned)nf);
    CgState* st = (CgState*)state;
    TimedSection ts("cg_step", s);
    k_cg_alpha<<<grid, kRedThreads, 0, s>>>(n, (const float2*)p, (const float2*)Ap, st);
    k_cg_update<<<grid, kRedThreads, 0, s>>>(n, (float2*)x, (float2*)r, (const float2*)p, (const float2*)Ap, st);
    k_cg_dir<<<grid, kRedThreads, 0, s>>>(n, (const float2*)r, (float2*)p, st);
    return check_launch("cg_step (frames)");
}

int cgb_read_state(const void* state, int64_t nf, double* rzold, int64_t* iters, int* converged, cudaStream_t s) {
    HB_REQUIRE(state && nf >= 1, HB_ERR_INVALID_ARG, "bad argument");
    for (int64_t f = 0; f < nf; ++f) {
        CgState h;
        HB_CUDA(cudaMemcpyAsync(&h, (const CgState*)state + f, offsetof(CgState, partial), cudaMemcpyDeviceToHost, s));
        HB_CUDA(cudaStreamSynchronize(s));
        if (rzold) rzold[f] = h.rzold;
        if (iters) iters[f] = h.iters;
        if (converged) converged[f] = (h.run == 0) || (sqrt(h.rzold) < h.tol);
    }
    return HB_OK;
}

int cg_init(int64_t n, const void* b, const void* Ax, void* r, void* p, void* state, double tol, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(b && Ax && r && p && state, HB_ERR_INVALID_ARG, "null argument");
    HB_CUDA(cudaMemsetAsync(state, 0, sizeof(CgState), s));
    k_cg_init<<<red_blocks(n), kRedThreads, 0, s>>>(n, (const float2*)b, (const float2*)Ax, (float2*)r, (float2*)p,
                                                   (CgState*)state, tol);
    return check_launch("k_cg_init");
}

int cg_step(int64_t n, void* x, void* r, void* p, const void* Ap, void* state, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(x && r && p && Ap && state, HB_ERR_INVALID_ARG, "null argument");
    const int g = red_blocks(n);
    CgState* st = (CgState*)state;
    TimedSection ts("cg_step", s);
    k_cg_alpha<<<g, kRedThreads, 0, s>>>(n, (const float2*)p, (const float2*)Ap, st);
    k_cg_update<<<g, kRedThreads, 0, s>>>(n, (float2*)x, (float2*)r, (const float2*)p, (const float2*)Ap, st);
    k_cg_dir<<<g, kRedThreads, 0, s>>>(n, (const float2*)r, (float2*)p, st);
    return check_launch("cg_step");
}

int cg_read_state(const void* state, double* rzold, int64_t* iters, int* converged, cudaStream_t s) {
    HB_REQUIRE(state, HB_ERR_INVALID_ARG, "null state");
    CgState h;
    HB_CUDA(cudaMemcpyAsync(&h, state, offsetof(CgState, partial), cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    if (rzold) *rzold = h.rzold;
    if (iters) *iters = h.iters;
    if (converged) *converged = (h.run == 0) || (sqrt(h.rzold) < h.tol);
    return HB_OK;
}

int pcg_residual(int64_t n, const void* b, const void* Ax, void* r, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(b && Ax && r, HB_ERR_INVALID_ARG, "null argument");
    k_pcg_residual<<<red_blocks(n), kRedThreads, 0, s>>>(n, (const float2*)b, (const float2*)Ax, (float2*)r);
    return check_launch("k_pcg_residual");
}

int pcg_start(int64_t n, const void* r, const void* z, void* p, void* state, double tol, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(r && z && p && state, HB_ERR_INVALID_ARG, "null argument");
    HB_CUDA(cudaMemsetAsync(state, 0, sizeof(CgState), s));
    k_pcg_start<<<red_blocks(n), kRedThreads, 0, s>>>(n, (const float2*)r, (const float2*)z, (float2*)p,
                                                     (CgState*)state, tol);
    return check_launch("k_pcg_start");
}

int pcg_step1(int64_t n, void* x, void* r, const void* p, const void* Ap, void* state, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(x && r && p && Ap && state, HB_ERR_INVALID_ARG, "null argument");
    const int g = red_blocks(n);
    CgState* st = (CgState*)state;
    TimedSection ts("pcg_step", s);
    k_cg_alpha<<<g, kRedThreads, 0, s>>>(n, (const float2*)p, (const float2*)Ap, st);
    k_pcg_xr<<<g, kRedThreads, 0, s>>>(n, (float2*)x, (float2*)r, (const float2*)p, (const float2*)Ap, st);
    return check_launch("pcg_step1");
}

int pcg_step2(int64_t n, const void* r, const void* z, void* p, void* state, int restart, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(r && z && p && state, HB_ERR_INVALID_ARG, "null argument");
    const int g = red_blocks(n);
    CgState* st = (CgState*)state;
    TimedSection ts("pcg_step", s);
    k_pcg_rz<<<g, kRedThreads, 0, s>>>(n, (const float2*)r, (const float2*)z, st);
    k_pcg_dir<<<g, kRedThreads, 0, s>>>(n, (const float2*)z, (float2*)p, st, restart ? 1 : 0);
    return check_launch("pcg_step2");
}

int vdot_real(int64_t n, const void* a, const void* b, double* out, cudaStream_t s) {
    HB_REQUIRE(n >= 1, HB_ERR_INVALID_ARG, "n must be >= 1");
    HB_REQUIRE(a && b && out, HB_ERR_INVALID_ARG, "null argument");
    DotScratch* sc = nullptr;
    HB_CUDA(cudaMallocAsync((void**)&sc, sizeof(DotScratch), s));
    cudaMemsetAsync(sc, 0, sizeof(unsigned int), s);
    k_vdot_real<<<red_blocks(n), kRedThreads, 0, s>>>(n, (const float2*)a, (const float2*)b, sc, out);
    int st = check_launch("k_vdot_real");
    HB_CUDA(cudaFreeAsync(sc, s));
    return st;
}

}  // namespace hb
