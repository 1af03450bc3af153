// extern "C" entry points of libhasty_b200.so (declared in include/hasty_b200.h). Each one
// validates its arguments, forwards to the hb:: implementation and turns any C++ exception
// into a status code; nothing throws across the boundary.
#include <new>
#include <string>

#include "common.cuh"
#include "nufft.cuh"

namespace hb {
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* get_error() { return g_last_error.c_str(); }

// implemented in toeplitz.cu / cg.cu
int toeplitz_kernel(int dim, const int64_t* kshape, int64_t M, const float* c0, const float* c1, const float* c2,
                    const void* nudata, void* kout, int width, cudaStream_t s);
int toeplitz_kernel_frames(int dim, const int64_t* kshape, int nframes, const int64_t* npts, const float* c0,
                           const float* c1, const float* c2, const void* nudata, void* kout, int width, cudaStream_t s);
int transform_toeplitz_kernel(int dim, const int64_t* kshape, const void* kin, void* kout, cudaStream_t s);
int toeplitz_workspace_size(int dim, const int64_t* shape, int64_t nbatch, size_t* bytes);
int toeplitz_multiplication(int dim, const int64_t* shape, int64_t nbatch, const void* input, void* output,
                            const void* kernel, void* workspace, size_t workspace_bytes, const void* mult1,
                            const void* mult2, int io_mult, int in_m1, int out_m1, int in_m2, int out_m2, int accumulate,
                            cudaStream_t s);
int sense_normal(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps, const void* kernel,
                 void* out, void* workspace, size_t workspace_bytes, cudaStream_t s);
int sense_normal_noalloc(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps,
                         const void* kernel, void* out, cudaStream_t s);
int sense_normal_ex(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps_in,
                    const void* smaps_out, const void* diag, int accumulate, const void* kernel, void* out,
                    void* workspace, size_t workspace_bytes, cudaStream_t s);
int sense_normal_batched(int dim, const int64_t* shape, int64_t nframes, int64_t ncoils, const void* x,
                         const void* smaps, const void* kernels, void* out, void* workspace, size_t workspace_bytes,
                         cudaStream_t s);
int transform_toeplitz_kernels(int dim, const int64_t* kshape, int64_t nframes, const void* kin, void* kout,
                               cudaStream_t s);
size_t cgb_state_bytes(int64_t nframes);
int cgb_init(int64_t n, int64_t nf, const void* b, const void* Ax, void* r, void* p, void* state, double tol,
             cudaStream_t s);
int cgb_step(int64_t n, int64_t nf, void* x, void* r, void* p, const void* Ap, void* state, cudaStream_t s);
int cgb_read_state(const void* state, int64_t nf, double* rzold, int64_t* iters, int* converged, cudaStream_t s);
size_t cg_state_bytes();
int cg_init(int64_t n, const void* b, const void* Ax, void* r, void* p, void* state, double tol, cudaStream_t s);
int cg_step(int64_t n, void* x, void* r, void* p, const void* Ap, void* state, cudaStream_t s);
int pcg_residual(int64_t n, const void* b, const void* Ax, void* r, cudaStream_t s);
int pcg_start(int64_t n, const void* r, const void* z, void* p, void* state, double tol, cudaStream_t s);
int pcg_step1(int64_t n, void* x, void* r, const void* p, const void* Ap, void* state, cudaStream_t s);
int pcg_step2(int64_t n, const void* r, const void* z, void* p, void* state, int restart, cudaStream_t s);
int cg_read_state(const void* state, double* rzold, int64_t* iters, int* converged, cudaStream_t s);
int vdot_real(int64_t n, const void* a, const void* b, double* out, cudaStream_t s);
}  // namespace hb

struct hb_nufft_plan_s {
    hb::NufftPlan p;
};

#define HB_GUARD(body)                                  \
    try {                                               \
        body                                            \
    } catch (const std::bad_alloc&) {                   \
        hb::set_error("host allocation failed");        \
        return HB_ERR_ALLOC;                            \
    } catch (const std::exception& ex) {                \
        hb::set_error(std::string("exception: ") + ex.what()); \
        return HB_ERR_INVALID_ARG;                      \
    } catch (...) {                                     \
        hb::set_error("unknown exception");             \
        return HB_ERR_INVALID_ARG;                      \
    }

static inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

const char* hb_last_error(void) { return hb::get_error(); }

int hb_version(void) { return 10000; }

int hb_nufft_makeplan(int type, int dim, const int64_t* nmodes, int sign, int ntransf, float tol, int kernel_width,
                      double upsampfac, int method, hb_nufft_plan* plan_out) {
    HB_GUARD({
        if (!plan_out) {
            hb::set_error("plan_out is null");
            return HB_ERR_INVALID_ARG;
        }
        *plan_out = nullptr;
        hb_nufft_plan_s* h = new hb_nufft_plan_s();
        int st = hb::plan_make(&h->p, type, dim, nmodes, sign, ntransf, tol, kernel_width, upsampfac, method);
        if (st != HB_OK) {
            hb::plan_free(&h->p);
            delete h;
            return st;
        }
        *plan_out = h;
        return HB_OK;
    })
}

int hb_nufft_setpts(hb_nufft_plan plan, int64_t M, const float* coord0, const float* coord1, const float* coord2,
                    void* stream) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_setpts(&plan->p, M, coord0, coord1, coord2, as_stream(stream));
    })
}

int hb_nufft_setpts_frames(hb_nufft_plan plan, int nframes, const int64_t* npts, const float* coord0,
                           const float* coord1, const float* coord2, void* stream) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_setpts_frames(&plan->p, nframes, npts, coord0, coord1, coord2, as_stream(stream));
    })
}

int hb_nufft_execute(hb_nufft_plan plan, const void* in, void* out, void* stream) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_execute(&plan->p, (const float2*)in, (float2*)out, as_stream(stream));
    })
}

int hb_nufft_set_spread_tuning(hb_nufft_plan plan, int max_candidates, int block_z, int block_y, int block_x) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_set_spread_tuning(&plan->p, max_candidates, block_z, block_y, block_x);
    })
}

int hb_nufft_set_spread_kernel(hb_nufft_plan plan, int kind, int transforms_per_cta) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_set_spread_kernel(&plan->p, kind, transforms_per_cta);
    })
}

int hb_nufft_set_interp_tuning(hb_nufft_plan plan, int transforms_per_group) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_set_interp_tuning(&plan->p, transforms_per_group);
    })
}

int hb_nufft_set_interp_kernel(hb_nufft_plan plan, int kind) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_set_interp_kernel(&plan->p, kind);
    })
}

int hb_nufft_coord_grad(hb_nufft_plan plan, const void* modes, const void* h, float* grad, void* stream) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        return hb::plan_coord_grad(&plan->p, (const float2*)modes, (const float2*)h, grad, as_stream(stream));
    })
}

int hb_nufft_destroy(hb_nufft_plan plan) {
    HB_GUARD({
        if (!plan) return HB_OK;
        hb::plan_free(&plan->p);
        delete plan;
        return HB_OK;
    })
}

int hb_nufft_get_info(hb_nufft_plan plan, int64_t* fine_out3, int* width_out, double* beta_out,
                      size_t* device_bytes_out) {
    HB_GUARD({
        if (!plan) {
            hb::set_error("plan is null");
            return HB_ERR_INVALID_ARG;
        }
        const hb::GridGeom& g = plan->p.g;
        if (fine_out3) {
            for (int i = 0; i < 3; ++i) fine_out3[i] = 1;
            for (int i = 0; i < g.dim; ++i) fine_out3[i] = g.nf[3 - g.dim + i];
        }
        if (width_out) *width_out = plan->p.kb.w;
        if (beta_out) *beta_out = plan->p.beta;
        if (device_bytes_out) *device_bytes_out = plan->p.device_bytes;
        return HB_OK;
    })
}

int hb_toeplitz_kernel(int dim, const int64_t* kernel_shape, int64_t M, const float* coord0, const float* coord1,
                       const float* coord2, const void* nudata, void* kernel_out, int kernel_width, void* stream) {
    HB_GUARD({
        return hb::toeplitz_kernel(dim, kernel_shape, M, coord0, coord1, coord2, nudata, kernel_out, kernel_width,
                                   as_stream(stream));
    })
}

int hb_toeplitz_kernels_frames(int dim, const int64_t* kernel_shape, int nframes, const int64_t* npts,
                               const float* coord0, const float* coord1, const float* coord2, const void* nudata,
                               void* kernel_out, int kernel_width, void* stream) {
    HB_GUARD({
        return hb::toeplitz_kernel_frames(dim, kernel_shape, nframes, npts, coord0, coord1, coord2, nudata, kernel_out,
                                          kernel_width, as_stream(stream));
    })
}

int hb_transform_toeplitz_kernel(int dim, const int64_t* kernel_shape, const void* kernel_in, void* kernel_out,
                                 void* stream) {
    HB_GUARD({ return hb::transform_toeplitz_kernel(dim, kernel_shape, kernel_in, kernel_out, as_stream(stream)); })
}

int hb_toeplitz_workspace_size(int dim, const int64_t* shape, int64_t nbatch, size_t* bytes) {
    HB_GUARD({ return hb::toeplitz_workspace_size(dim, shape, nbatch, bytes); })
}

int hb_toeplitz_multiplication(int dim, const int64_t* shape, int64_t nbatch, const void* input, void* output,
                               const void* kernel, void* workspace, size_t workspace_bytes, const void* mult1,
                               const void* mult2, int io_mult, int in_m1, int out_m1, int in_m2, int out_m2,
                               int accumulate, void* stream) {
    HB_GUARD({
        return hb::toeplitz_multiplication(dim, shape, nbatch, input, output, kernel, workspace, workspace_bytes, mult1,
                                           mult2, io_mult, in_m1, out_m1, in_m2, out_m2, accumulate, as_stream(stream));
    })
}

int hb_sense_normal(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps, const void* kernel,
                    void* out, void* workspace, size_t workspace_bytes, void* stream) {
    HB_GUARD({
        return hb::sense_normal(dim, shape, ncoils, x, smaps, kernel, out, workspace, workspace_bytes,
                                as_stream(stream));
    })
}

int hb_sense_normal_noalloc(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps,
                            const void* kernel, void* out, void* stream) {
    HB_GUARD({ return hb::sense_normal_noalloc(dim, shape, ncoils, x, smaps, kernel, out, as_stream(stream)); })
}

int hb_sense_normal_ex(int dim, const int64_t* shape, int64_t ncoils, const void* x, const void* smaps_in,
                       const void* smaps_out, const void* diag, int accumulate, const void* kernel, void* out,
                       void* workspace, size_t workspace_bytes, void* stream) {
    HB_GUARD({
        return hb::sense_normal_ex(dim, shape, ncoils, x, smaps_in, smaps_out, diag, accumulate, kernel, out, workspace,
                                   workspace_bytes, as_stream(stream));
    })
}

int hb_sense_normal_batched(int dim, const int64_t* shape, int64_t nframes, int64_t ncoils, const void* x,
                            const void* smaps, const void* kernels, void* out, void* workspace, size_t workspace_bytes,
                            void* stream) {
    HB_GUARD({
        return hb::sense_normal_batched(dim, shape, nframes, ncoils, x, smaps, kernels, out, workspace, workspace_bytes,
                                        as_stream(stream));
    })
}

int hb_transform_toeplitz_kernels(int dim, const int64_t* kernel_shape, int64_t nframes, const void* kernels_in,
                                  void* kernels_out, void* stream) {
    HB_GUARD({
        return hb::transform_toeplitz_kernels(dim, kernel_shape, nframes, kernels_in, kernels_out, as_stream(stream));
    })
}

size_t hb_cgb_state_bytes(int64_t nframes) { return hb::cgb_state_bytes(nframes); }

int hb_cgb_init(int64_t n, int64_t nframes, const void* b, const void* Ax, void* r, void* p, void* state, double tol,
                void* stream) {
    HB_GUARD({ return hb::cgb_init(n, nframes, b, Ax, r, p, state, tol, as_stream(stream)); })
}

int hb_cgb_step(int64_t n, int64_t nframes, void* x, void* r, void* p, const void* Ap, void* state, void* stream) {
    HB_GUARD({ return hb::cgb_step(n, nframes, x, r, p, Ap, state, as_stream(stream)); })
}

int hb_cgb_read_state(const void* state, int64_t nframes, double* rzold, int64_t* iters, int* converged,
                      void* stream) {
    HB_GUARD({ return hb::cgb_read_state(state, nframes, rzold, iters, converged, as_stream(stream)); })
}

size_t hb_cg_state_bytes(void) { return hb::cg_state_bytes(); }

int hb_cg_init(int64_t n, const void* b, const void* Ax, void* r, void* p, void* state, double tol, void* stream) {
    HB_GUARD({ return hb::cg_init(n, b, Ax, r, p, state, tol, as_stream(stream)); })
}

int hb_cg_step(int64_t n, void* x, void* r, void* p, const void* Ap, void* state, void* stream) {
    HB_GUARD({ return hb::cg_step(n, x, r, p, Ap, state, as_stream(stream)); })
}

int hb_pcg_residual(int64_t n, const void* b, const void* Ax, void* r, void* stream) {
    HB_GUARD({ return hb::pcg_residual(n, b, Ax, r, as_stream(stream)); })
}

int hb_pcg_start(int64_t n, const void* r, const void* z, void* p, void* state, double tol, void* stream) {
    HB_GUARD({ return hb::pcg_start(n, r, z, p, state, tol, as_stream(stream)); })
}

int hb_pcg_step1(int64_t n, void* x, void* r, const void* p, const void* Ap, void* state, void* stream) {
    HB_GUARD({ return hb::pcg_step1(n, x, r, p, Ap, state, as_stream(stream)); })
}

int hb_pcg_step2(int64_t n, const void* r, const void* z, void* p, void* state, int restart, void* stream) {
    HB_GUARD({ return hb::pcg_step2(n, r, z, p, state, restart, as_stream(stream)); })
}

int hb_cg_read_state(const void* state, double* rzold, int64_t* iters, int* converged, void* stream) {
    HB_GUARD({ return hb::cg_read_state(state, rzold, iters, converged, as_stream(stream)); })
}

int hb_vdot_real(int64_t n, const void* a, const void* b, double* result_dev, void* stream) {
    HB_GUARD({ return hb::vdot_real(n, a, b, result_dev, as_stream(stream)); })
}

}  // extern "C"
