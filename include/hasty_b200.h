/*
 * hasty_b200.h -- C ABI of libhasty_b200.so, the B200 (sm_100a) implementation of the
 * HastyCuCompute MRI reconstruction hot path:
 *
 *   - non-uniform FFT type 1 (adjoint gridding) and type 2 (forward interpolation),
 *     1-3 dimensions, complex64 data, float32 coordinates in radians;
 *   - the Toeplitz-embedded normal operator (2x zero pad, FFT, pointwise kernel, crop),
 *     its kernel construction, and the SENSE coil expand / reduce around it;
 *   - the conjugate-gradient vector steps that drive the normal operator.
 *
 * Conventions (all shared with the reference C++ library):
 *   - arrays are C-order; an image of shape [N0, N1, N2] has N2 fastest;
 *   - coordinate array coordI pairs with image dimension I (the reference hands
 *     coords[DIM-1] to cufinufft as "x", cpp/corelib/lib/fft/nufft.cppm:191-199);
 *   - mode index i of a dimension of size N holds frequency k = i - floor(N/2)
 *     (cufinufft default mode order);
 *   - type 1:  f[k]  = sum_j c_j exp(+i*sign1 k.x_j), default sign +1;
 *     type 2:  c_j   = sum_k f[k] exp(+i*sign2 k.x_j), default sign -1
 *     (cpp/corelib/lib/fft/nufft.cppm:50-55);
 *   - every device pointer is caller-owned unless a function says otherwise;
 *   - every launch goes on the caller's stream (`stream` is a cudaStream_t, NULL means the
 *     legacy default stream); nothing synchronises the device except where stated.
 *
 * Errors: every function returns an int status (HB_OK == 0). On failure the message is
 * kept per thread and returned by hb_last_error(). Nothing throws across this boundary.
 */
#ifndef HASTY_B200_H
#define HASTY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define HB_OK               0
#define HB_ERR_INVALID_ARG  1  /* bad enum value, null pointer, bad sizes              */
#define HB_ERR_SHAPE        2  /* shapes that do not agree (kernel vs image, ...)       */
#define HB_ERR_CUDA         3  /* a CUDA runtime call failed                             */
#define HB_ERR_ALLOC        4  /* device allocation failed                               */
#define HB_ERR_STATE        5  /* call order violated (execute before setpts, ...)      */
#define HB_ERR_RANGE        6  /* non-finite coordinate met during setpts                */
#define HB_ERR_WORKSPACE    7  /* caller-provided workspace smaller than required        */

/* ---- enums (values identical to the reference) --------------------------------------- */
/* nufft_type, cpp/corelib/lib/fft/nufft.cppm:42-48 */
#define HB_NUFFT_TYPE_1 1      /* BACKWARD / adjoint */
#define HB_NUFFT_TYPE_2 2      /* FORWARD            */
/* nufft_method_cuda, cpp/corelib/lib/fft/nufft.cppm:65-70. Every value selects the same
 * bin-sorted tile kernels here; the value is kept so callers port unchanged. */
#define HB_METHOD_GM_NO_SORT 0
#define HB_METHOD_GM_SORT    1
#define HB_METHOD_SM         2
#define HB_METHOD_DEFAULT    3
/* ToeplitzMultType, cpp/corelib/lib/fft/toeplitz.cppm:47-51 */
#define HB_MULT_NONE      0
#define HB_MULT_MULT      1
#define HB_MULT_MULT_CONJ 2
/* ToeplitzAccumulateType, cpp/corelib/lib/fft/toeplitz.cppm:53-56 */
#define HB_ACC_NONE       0
#define HB_ACC_ACCUMULATE 1

/* ---- library ---------------------------------------------------------------------- */
const char* hb_last_error(void);
int hb_version(void);

/* ---- NUFFT plan ---------------------------------------------------------------------
 * Replaces nufft_plan<cuda_t,f32_t,DIM,NT> (cpp/corelib/lib/fft/nufft.cppm:103-310), i.e.
 * cufinufftf_makeplan / setpts / execute / destroy.
 *
 * Kernel: Kaiser-Bessel, phi(z) = I0(beta*sqrt(1-(2z/w)^2)) / I0(beta) on |z| < w/2 (fine
 * grid units), beta = pi*sqrt((w/sigma)^2 (sigma-1/2)^2 - 0.8). Width w comes from
 * `kernel_width` when > 0, else from `tol` as w = ceil(log10(10/tol)) (2 <= w <= 16).
 * Fine grid per dimension: the smallest 2,3,5-smooth multiple of the spread tile edge that
 * is >= max(upsampfac*N, 2w).
 */
typedef struct hb_nufft_plan_s* hb_nufft_plan;

/* nufft_plan::make, nufft.cppm:107-172. nmodes has `dim` entries in image order (dim 0
 * slowest). sign: +1 / -1, or 0 for the type's default. upsampfac <= 0 means 2.0. */
int hb_nufft_makeplan(int type, int dim, const int64_t* nmodes, int sign, int ntransf,
                      float tol, int kernel_width, double upsampfac, int method,
                      hb_nufft_plan* plan_out);

/* nufft_plan::setpts, nufft.cppm:175-203. Coordinates are device float arrays of length M
 * (coord1/coord2 NULL below 2/3 dims). The plan keeps its own sorted copy; the caller's
 * arrays may be freed afterwards. Bin-sorts the points on `stream` and synchronises it once
 * to size the spread work list. A non-finite coordinate returns HB_ERR_RANGE. */
int hb_nufft_setpts(hb_nufft_plan plan, int64_t M, const float* coord0, const float* coord1,
                    const float* coord2, void* stream);

/* Frames in one plan: replaces the per-frame loop of plans (one setpts + execute per frame's
 * trajectory, hasty_python/simul_op.py:39-91, right_precond_test.py:48-73) with one bin sort
 * and one launch per pass over every frame's points. Frame f has npts[f] points (host array of
 * nframes counts, zeros allowed); the device coordinate arrays hold the frames one after the
 * other (M = sum npts). Grows the plan's grids to nframes frames on first use. After it, execute
 * reads and writes (M_f = npts[f], rows of all frames back to back):
 *   type 1: in = c64 [ntransf, M],  out = c64 [nframes, ntransf, N0, ..];
 *   type 2: in = c64 [nframes, ntransf, N0, ..], out = c64 [ntransf, M].
 * hb_nufft_setpts is this call with one frame. */
int hb_nufft_setpts_frames(hb_nufft_plan plan, int nframes, const int64_t* npts,
                           const float* coord0, const float* coord1, const float* coord2,
                           void* stream);

/* nufft_plan::execute, nufft.cppm:205-250.
 *   type 1: in = c64 [ntransf, M] nonuniform data, out = c64 [ntransf, N0, ..] modes;
 *   type 2: in = c64 [ntransf, N0, ..] modes,      out = c64 [ntransf, M].
 * Allocation free, graph capturable. */
int hb_nufft_execute(hb_nufft_plan plan, const void* in, void* out, void* stream);

/* Spreading knobs (no counterpart in the reference; set by the autotuner, before setpts): points
 * per spread subproblem (32..65536; when never set, setpts picks a power of two in 512..4096 from
 * the number of points) and the cell block a warp owns inside a spread tile (32 cells; default
 * 2x4x4 in 3-D, 1x4x8 in 2-D; power-of-two edges dividing the tile edge, unit axes 1). */
int hb_nufft_set_spread_tuning(hb_nufft_plan plan, int max_candidates, int block_z, int block_y,
                               int block_x);

/* Spreading kernel of a type-1 plan, before its setpts (no counterpart in the reference, whose
 * spreading method is cufinufft's GM / GM_SORT / SM choice, fft/nufft.cppm:119-139):
 * HB_SPREAD_AUTO (transforms on the lanes when the plan allows it: 8^3 or 16x32 tiles, widths
 * 4..8, 5 or more transforms, two or more tiles per axis), HB_SPREAD_CELLS (one cell per lane,
 * any plan), HB_SPREAD_TRANSFORMS (transforms on the lanes; HB_ERR_INVALID_ARG where the plan
 * does not allow it). transforms_per_cta (8, 16 or 32; 0 = automatic) sets how many transforms
 * one CTA of the transforms kernel spreads; larger transform counts run as several CTAs per tile.
 * Every choice computes the same sums. */
#define HB_SPREAD_AUTO       0
#define HB_SPREAD_CELLS      1
#define HB_SPREAD_TRANSFORMS 2
int hb_nufft_set_spread_kernel(hb_nufft_plan plan, int kind, int transforms_per_cta);

/* Interpolation of a type-2 plan (no counterpart in the reference): the transforms one group of
 * lanes gathers per point (1, 2, 4, 8, 16 or 32; 0 = automatic), i.e. 32 / that many points per
 * warp in flight at once. Every choice computes the same sums. */
int hb_nufft_set_interp_tuning(hb_nufft_plan plan, int transforms_per_group);

/* Interpolation kernel of a type-2 plan (no counterpart in the reference): HB_INTERP_GATHER
 * (warps gather each point's cells from global memory, any plan), HB_INTERP_STAGED (one CTA per
 * 8^3 tile and 8 transforms copies the region the tile's footprints reach into shared memory and
 * gathers from there; 3-D plans with kernel width 4..7, else HB_ERR_INVALID_ARG) or HB_INTERP_AUTO.
 * Both kernels give bit-identical samples; callable before or after setpts. */
#define HB_INTERP_AUTO   0
#define HB_INTERP_GATHER 1
#define HB_INTERP_STAGED 2
int hb_nufft_set_interp_kernel(hb_nufft_plan plan, int kind);

/* Coordinate gradient (no counterpart in the reference, which has no derivatives): with a
 * type-2 plan (sign s) whose points are set, writes to grad ([dim][M] float, image order)
 *   grad[i][j] = -(nf_i / 2 pi) Re( sum_c h[c][j] sum_l G_c[l] dPhi_i(l - u_j) )
 * where G is the plan's fine grid of `modes` ([ntransf, N..]) after the type-2 passes and dPhi_i
 * the kernel with its derivative along dimension i: the exact derivative of the implemented
 * gridding operator with respect to the points. For c = A f (this plan) and a real loss L,
 * h = conj(dL/dc) gives dL/dx. For f = B c (a type-1 plan of sign -s on the same points),
 * modes = dL/df and h = conj(c) give dL/dx. Kernel widths up to 8. */
int hb_nufft_coord_grad(hb_nufft_plan plan, const void* modes, const void* h, float* grad,
                        void* stream);

/* nufft_plan::free / ~nufft_plan, nufft.cppm:279-301. Safe on NULL. */
int hb_nufft_destroy(hb_nufft_plan plan);

/* Plan introspection: fine grid sizes (image order), kernel width, beta, device bytes held. */
int hb_nufft_get_info(hb_nufft_plan plan, int64_t* fine_out3, int* width_out,
                      double* beta_out, size_t* device_bytes_out);

/* ---- Toeplitz ------------------------------------------------------------------------
 * toeplitz_kernel, cpp/corelib/lib/fft/nufft.cppm:386-441:
 *   kernel (shape [2N0, .., 2N{dim-1}], c64) = FFT( embed_{[0,2N-1)}( type1(nudata; 2N-1
 *   modes) ) ) / prod(N).
 * nudata is c64 [M] (the reference's [1, M]). The type-1 uses this library's NUFFT with the
 * given kernel width (<= 0: from tol = 1e-5 as the reference asks for f32).
 * Allocates and frees a temporary NUFFT plan and grid (not graph capturable). */
int hb_toeplitz_kernel(int dim, const int64_t* kernel_shape, int64_t M, const float* coord0,
                       const float* coord1, const float* coord2, const void* nudata,
                       void* kernel_out, int kernel_width, void* stream);

/* toeplitz_kernel for nframes frames in one call (the per-frame kernel builds of
 * hasty_python/simul_op.py:39-91 and right_precond_test.py:48-73, there one cufinufft plan and
 * toeplitz_kernel call per frame): one frame-batched type-1 NUFFT over all frames' points
 * (frame f has npts[f] points, frames back to back in coord* and nudata, as for
 * hb_nufft_setpts_frames) and one launch per FFT pass over all frames. kernel_out is
 * c64 [nframes, 2N0, ..]. Allocates and frees its temporaries (about nframes times the
 * one-frame call's). */
int hb_toeplitz_kernels_frames(int dim, const int64_t* kernel_shape, int nframes,
                               const int64_t* npts, const float* coord0, const float* coord1,
                               const float* coord2, const void* nudata, void* kernel_out,
                               int kernel_width, void* stream);

/* transform_toeplitz_kernel, cpp/corelib/lib/fft/toeplitz.cppm:510-609: re-lays the
 * straight kernel ([2N..] c64, from hb_toeplitz_kernel) into the layout
 * hb_toeplitz_multiplication / hb_sense_normal read (same element count, c64), with the
 * inverse-FFT normalisation 1/prod(2N) and, per axis, the phase ramp exp(+2 pi i k (N-1) / 2N)
 * folded in (it moves the crop [N-1, 2N-1) of the inverse transform to [0, N)). in and out must
 * not alias. */
int hb_transform_toeplitz_kernel(int dim, const int64_t* kernel_shape, const void* kernel_in,
                                 void* kernel_out, void* stream);

/* Bytes of device workspace hb_toeplitz_multiplication / hb_sense_normal need for images of
 * shape `shape` ([N0..], dim entries) with `nbatch` batches (coils). */
int hb_toeplitz_workspace_size(int dim, const int64_t* shape, int64_t nbatch, size_t* bytes);

/* toeplitz_multiplication / ops_toeplitz_multiplication, cpp/corelib/lib/fft/toeplitz.cppm:
 * 611-712 and 722-857 (kernel code fft/kernels/toeplitz_load_3D.cu:18-79). For each batch b:
 *   t      = input[b] * m(mult1, in_m1) * m(mult2, in_m2)
 *   v      = crop_{[N-1,2N-1)}( IFFT( FFT(pad_{2N}(t)) * K ) )
 *   v      = v * m(mult1, out_m1) * m(mult2, out_m2) * m(input[b], io_mult)
 *   out[b] = v (+ out[b] if accumulate)
 * m(a, NONE) = 1, m(a, MULT) = a, m(a, MULT_CONJ) = conj(a). mult1/mult2 are [N..] or NULL.
 * kernel is the transformed kernel. `workspace` must hold hb_toeplitz_workspace_size bytes;
 * NULL makes the call allocate it stream-ordered (cudaMallocAsync) and free it after. */
int hb_toeplitz_multiplication(int dim, const int64_t* shape, int64_t nbatch,
                               const void* input, void* output, const void* kernel,
                               void* workspace, size_t workspace_bytes,
                               const void* mult1, const void* mult2,
                               int io_mult, int in_m1, int out_m1, int in_m2, int out_m2,
                               int accumulate, void* stream);

/* NORMAL_T_T1_OP::operator(), cpp/corelib/lib/mri/normal.cppm:65-88, fused:
 *   out = sum_c conj(S_c) * T(S_c * x)     (x, out: [N..]; smaps: [C, N..])
 * with T the Toeplitz operator of `kernel` (transformed). The coil sum happens inside the
 * last FFT pass; no [C, N..] intermediate is written. out must not alias x.
 * Workspace as for hb_toeplitz_multiplication with nbatch = C. */
int hb_sense_normal(int dim, const int64_t* shape, int64_t ncoils, const void* x,
                    const void* smaps, const void* kernel, void* out,
                    void* workspace, size_t workspace_bytes, void* stream);

/* One time segment of NORMAL_IDT_T1_OP / NORMAL_IDTW_T1_OP (cpp/corelib/lib/mri/normal.cppm:
 * 218-266 and 441-535), fused like hb_sense_normal:
 *   out (+)= conj(R) * sum_c conj(U_c) * T(R * S_c * x)
 * S = smaps_in [C, N..]; U = smaps_out [C, N..] (NULL: U = S); R = diag [N..] (NULL: 1).
 * NORMAL_IDT_T1_OP is the sum of these over its L (kernel, diagonal) pairs, the first call with
 * accumulate = HB_ACC_NONE and the rest HB_ACC_ACCUMULATE. NORMAL_IDTW_T1_OP's coil mixing
 * sum_i conj(S_i) sum_j W_ij v_j equals sum_j conj(U_j) v_j with U_j = sum_i conj(W_ij) S_i, so it
 * runs with U = W^H S. out must not alias an input; workspace as for hb_sense_normal. */
int hb_sense_normal_ex(int dim, const int64_t* shape, int64_t ncoils, const void* x,
                       const void* smaps_in, const void* smaps_out, const void* diag, int accumulate,
                       const void* kernel, void* out, void* workspace, size_t workspace_bytes,
                       void* stream);

/* ---- frames: many systems in one launch per pass (no counterpart in the reference) -------
 * hb_sense_normal over F frames that share the coil maps, each with its own Toeplitz kernel:
 *   out[f] = sum_c conj(S_c) T_f(S_c x[f])     x, out: [F, N..]; smaps: [C, N..]
 * kernels from hb_transform_toeplitz_kernels. All F*C columns run through each of the five passes
 * in one launch. Workspace: hb_toeplitz_workspace_size(dim, shape, F*C). The per-frame loop it
 * replaces is NORMAL_T_T1_OP::operator() (cpp/corelib/lib/mri/normal.cppm:65-88) once per frame. */
int hb_sense_normal_batched(int dim, const int64_t* shape, int64_t nframes, int64_t ncoils,
                            const void* x, const void* smaps, const void* kernels, void* out,
                            void* workspace, size_t workspace_bytes, void* stream);
/* transform_toeplitz_kernel (cpp/corelib/lib/fft/toeplitz.cppm:510-609) for F straight kernels
 * [F, 2N..] at once, into the layout hb_sense_normal_batched reads. */
int hb_transform_toeplitz_kernels(int dim, const int64_t* kernel_shape, int64_t nframes,
                                  const void* kernels_in, void* kernels_out, void* stream);

/* Allocation-free variant of hb_sense_normal (no counterpart in the reference). For callers
 * that cannot allocate device memory -- a runtime embedded in another framework that owns all
 * allocations, a driver layer handing out fixed buffers, code running where cudaMalloc is off
 * limits. It allocates nothing: the workspace (32 MiB) and the FFT twiddle tables sit in fixed
 * device arrays inside this library, which every GPU that loads it keeps until exit. Limits:
 * the workspace need, 3-D 6 * prod(N) * ncoils * 8 bytes and 2-D 2 * prod(N) * ncoils * 8
 * bytes, must be <= 32 MiB (else HB_ERR_WORKSPACE, nothing launched), and 2N <= 4096 per axis.
 * The first call on a device (and the first after a device reset, which reloads the arrays at
 * new addresses) looks up the arrays' device addresses; make that first call before any stream
 * capture. All calls share the arrays, so calls that overlap on the GPU (different streams,
 * threads or processes sharing a context) race: serialise them. Result as hb_sense_normal. */
int hb_sense_normal_noalloc(int dim, const int64_t* shape, int64_t ncoils, const void* x,
                            const void* smaps, const void* kernel, void* out, void* stream);

/* ---- conjugate gradient --------------------------------------------------------------
 * Vector steps of conjugate_gradient, cpp/corelib/lib/op/cg.cppm:122-184, with all scalars
 * on the device (no host read per iteration) and every inner product accumulated in FP64
 * in a fixed order. The state block is opaque device memory of hb_cg_state_bytes() bytes.
 * An iteration is  Ap = A(p); hb_cg_step(...). Once sqrt(rzold) < tol the steps leave x, r,
 * p unchanged (the reference breaks out of its loop), so a fixed-length captured loop gives
 * the reference's result. */
size_t hb_cg_state_bytes(void);
/* r = b - Ax; p = r; rzold = Re<r,r>; state.tol = tol. */
int hb_cg_init(int64_t n, const void* b, const void* Ax, void* r, void* p, void* state,
               double tol, void* stream);
/* pAp = Re<p,Ap>; alpha = rzold/pAp; x += alpha p; r -= alpha Ap; rznew = Re<r,r>;
 * p = r + (rznew/rzold) p; rzold = rznew. */
int hb_cg_step(int64_t n, void* x, void* r, void* p, const void* Ap, void* state, void* stream);
/* Preconditioned / restarted CG, cpp/corelib/lib/op/cg.cppm:16-119, on the same state block:
 *   hb_pcg_residual: r = b - Ax;   caller: z = P(r);   hb_pcg_start: p = z, rzold = Re<r,z>
 *   iteration:  Ap = A(p); hb_pcg_step1 (break test sqrt(rzold) < tol, alpha, x, r);
 *               z = P(r);  hb_pcg_step2 (rznew = Re<r,z>, p = z (restart != 0) or
 *               z + (rznew/rzold) p, rzold = rznew).
 * After the break test fires both steps leave x, r and p unchanged. */
int hb_pcg_residual(int64_t n, const void* b, const void* Ax, void* r, void* stream);
int hb_pcg_start(int64_t n, const void* r, const void* z, void* p, void* state, double tol,
                 void* stream);
int hb_pcg_step1(int64_t n, void* x, void* r, const void* p, const void* Ap, void* state,
                 void* stream);
int hb_pcg_step2(int64_t n, const void* r, const void* z, void* p, void* state, int restart,
                 void* stream);
/* Copies {rzold, iterations done, converged flag} to host (synchronises the stream). */
int hb_cg_read_state(const void* state, double* rzold, int64_t* iters, int* converged,
                     void* stream);

/* The same steps for F independent systems at once (vectors [F, n], one state block per frame,
 * hb_cgb_state_bytes(F) bytes); each frame keeps its own scalars and its own early exit. */
size_t hb_cgb_state_bytes(int64_t nframes);
int hb_cgb_init(int64_t n, int64_t nframes, const void* b, const void* Ax, void* r, void* p,
                void* state, double tol, void* stream);
int hb_cgb_step(int64_t n, int64_t nframes, void* x, void* r, void* p, const void* Ap,
                void* state, void* stream);
int hb_cgb_read_state(const void* state, int64_t nframes, double* rzold, int64_t* iters,
                      int* converged, void* stream);

/* ---- vector helpers ------------------------------------------------------------------ */
/* Re<a,b> in FP64, written to *result_dev (a device double). Deterministic order. */
int hb_vdot_real(int64_t n, const void* a, const void* b, double* result_dev, void* stream);

/* ---- measurement hooks (no counterpart in the reference) ------------------------------
 * When enabled, every kernel launch of this library is bracketed by CUDA events on the stream
 * it runs on. hb_timing_read synchronises on the recorded events, writes the per-kernel-name
 * summed milliseconds (first-seen order; names '\n'-separated into `names`), the number of
 * names and of launches recorded, then clears the record. Not for use inside stream capture. */
int hb_timing_enable(int on);
int hb_timing_read(char* names, size_t names_cap, float* ms, int cap, int* n_names,
                   int* n_launches);

#ifdef __cplusplus
}
#endif

#endif /* HASTY_B200_H */
