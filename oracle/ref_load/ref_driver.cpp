// Host driver for the reference's toeplitz_load_2D / toeplitz_load_3D kernels
// (cpp/corelib/lib/fft/kernels/toeplitz_load_{2D,3D}.cu, compiled unchanged with cpu_shim.h).
// It emulates the reference's launch (fft/toeplitz.cppm:137-163: 256 threads per block,
// ceil(N/256) blocks) by visiting every (block, thread). Test infrastructure only.
#include "cpu_shim.h"

hb_ref_dim3 blockIdx, blockDim, threadIdx;

struct cuFloatComplex;
extern "C" void toeplitz_load_3D(const cuFloatComplex*, cuFloatComplex*, cuFloatComplex*, const cuFloatComplex*,
                                 const cuFloatComplex*, int, int, int, int, int, int, int, int, int, int, bool);
extern "C" void toeplitz_load_2D(const cuFloatComplex*, cuFloatComplex*, cuFloatComplex*, const cuFloatComplex*,
                                 const cuFloatComplex*, int, int, int, int, int, int, int, int, int, bool);

extern "C" void ref_launch_load_3D(const void* input, void* output, void* scratch, const void* mult1,
                                   const void* mult2, int io, int in1, int out1, int in2, int out2, int batch_in,
                                   int batch_out, int NX, int NY, int NZ, int accumulate) {
    const int threads = 256;
    const long total = (long)NX * NY * NZ;
    const int blocks = (int)((total + threads - 1) / threads);
    blockDim = {(unsigned)threads, 1, 1};
    for (int b = 0; b < blocks; ++b) {
        blockIdx = {(unsigned)b, 0, 0};
        for (int t = 0; t < threads; ++t) {
            threadIdx = {(unsigned)t, 0, 0};
            toeplitz_load_3D((const cuFloatComplex*)input, (cuFloatComplex*)output, (cuFloatComplex*)scratch,
                             (const cuFloatComplex*)mult1, (const cuFloatComplex*)mult2, io, in1, out1, in2, out2,
                             batch_in, batch_out, NX, NY, NZ, accumulate != 0);
        }
    }
}

extern "C" void ref_launch_load_2D(const void* input, void* output, void* scratch, const void* mult1,
                                   const void* mult2, int io, int in1, int out1, int in2, int out2, int batch_in,
                                   int batch_out, int NX, int NY, int accumulate) {
    const int threads = 256;
    const long total = (long)NX * NY;
    const int blocks = (int)((total + threads - 1) / threads);
    blockDim = {(unsigned)threads, 1, 1};
    for (int b = 0; b < blocks; ++b) {
        blockIdx = {(unsigned)b, 0, 0};
        for (int t = 0; t < threads; ++t) {
            threadIdx = {(unsigned)t, 0, 0};
            toeplitz_load_2D((const cuFloatComplex*)input, (cuFloatComplex*)output, (cuFloatComplex*)scratch,
                             (const cuFloatComplex*)mult1, (const cuFloatComplex*)mult2, io, in1, out1, in2, out2,
                             batch_in, batch_out, NX, NY, accumulate != 0);
        }
    }
}
