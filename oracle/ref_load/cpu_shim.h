/* Makes the reference's Toeplitz load/store kernels (plain CUDA C, no intrinsics) compile as
 * host C++: __global__/__device__ vanish and the launch coordinates become host globals that
 * ref_driver.cpp steps through, one (block, thread) at a time. Test infrastructure only. */
#pragma once
#define __global__
#define __device__
struct hb_ref_dim3 { unsigned int x, y, z; };
extern hb_ref_dim3 blockIdx, blockDim, threadIdx;
