// Host side of the shared-memory FFT passes: radix plans, twiddle tables, block sizing.
#include <cmath>
#include <vector>

#include "fft.cuh"

namespace hb {

int fftlen_make(FftLen* f, int L) {
    f->L = L;
    f->nrad = 0;
    f->tw = nullptr;
    int rest = L;
    const int order[8] = {8, 4, 2, 5, 3, 7, 11, 13};
    for (int r : order) {
        while (rest % r == 0 && rest > 1) {
            if (f->nrad >= kMaxRadices) {
                set_error("FFT length has too many factors");
                return HB_ERR_INVALID_ARG;
            }
            f->rad[f->nrad++] = r;
            rest /= r;
        }
    }
    if (rest != 1) {
        set_error("FFT length " + std::to_string(L) + " has a prime factor other than 2, 3, 5, 7, 11, 13");
        return HB_ERR_INVALID_ARG;
    }
    std::vector<float2> h(L);
    for (int m = 0; m < L; ++m) {
        double ang = 2.0 * M_PI * (double)m / (double)L;
        h[m] = make_float2((float)std::cos(ang), (float)(-std::sin(ang)));
    }
    cudaError_t e = cudaMalloc(&f->tw, sizeof(float2) * (size_t)L);
    if (e != cudaSuccess) {
        set_error(std::string("cudaMalloc(twiddles) failed: ") + cudaGetErrorString(e));
        f->tw = nullptr;
        return HB_ERR_ALLOC;
    }
    HB_CUDA(cudaMemcpy(f->tw, h.data(), sizeof(float2) * (size_t)L, cudaMemcpyHostToDevice));
    return HB_OK;
}

void fftlen_free(FftLen* f) {
    if (f->tw) cudaFree(f->tw);
    f->tw = nullptr;
}

int pass_columns_for(int L) {
    const size_t budget = 100 * 1024;
    int W = 32;
    while (W > 1) {
        int Wp = W | 1;
        size_t bytes = (size_t)(2 * L * Wp + L) * sizeof(float2);
        if (bytes <= budget) break;
        W >>= 1;
    }
    return W;
}

void pass_setup(PassCfg* c, const FftLen& f, int64_t A, int64_t E, int Lin, int in_shift, int Lout,
                int out_shift, int inverse, int max_cols) {
    c->L = f.L;
    c->nrad = f.nrad;
    for (int i = 0; i < kMaxRadices; ++i) c->rad[i] = f.rad[i];
    c->tw = f.tw;
    c->Lin = Lin;
    c->in_shift = in_shift;
    c->Lout = Lout;
    c->out_shift = out_shift;
    c->A = A;
    c->E = E;
    const int W = max_cols > 0 ? max_cols : pass_columns_for(f.L);
    int Eb = (int)(E < W ? E : W);
    if (Eb < 1) Eb = 1;
    int Ab = W / Eb;
    if (Ab < 1) Ab = 1;
    if (Ab > A) Ab = (int)(A > 0 ? A : 1);
    c->E_blk = Eb;
    c->A_blk = Ab;
    c->W = Ab * Eb;
    c->Wp = c->W | 1;
    c->n_eb = ceil_div(E, Eb);
    c->inverse = inverse;
}

}  // namespace hb
