"""CPU oracle for the hastycucompute_b200 hot path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product (the ``hastycucompute_b200`` package and its CUDA library) imports this
package. Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use it,
as the checker and as the timed CPU reference.

Contents
--------
- ``nudft``      FP64 direct non-uniform DFT (type 1 / type 2): the mathematical definition the
                 reference's cufinufft calls compute (cpp/corelib/lib/fft/nufft.cppm:205-250,
                 signs :50-55, coordinate pairing :191-199, centred mode order).
- ``kb``         Kaiser-Bessel kernel, its Fourier transform and the fine-grid sizing rule.
- ``gridding``   FP64 restatement of the gridding NUFFT (spread / FFT / deapodise and the
                 reverse) with the same kernel, width, upsampling and fine grid as the GPU path.
- ``toeplitz``   the reference's straight Toeplitz kernel and multiply
                 (cpp/corelib/lib/fft/nufft.cppm:386-479), the flag semantics of
                 toeplitz_multiplication (cpp/corelib/lib/fft/toeplitz.cppm:611-712) and the SENSE
                 normal operator (cpp/corelib/lib/mri/normal.cppm:65-88).
- ``refload``    the reference's own Toeplitz load/store kernels
                 (cpp/corelib/lib/fft/kernels/toeplitz_load_{2D,3D}.cu), compiled for the CPU by
                 ``oracle/ref_load/Makefile`` into ``oracle/_ref/`` and driven from Python.
- ``cg``         conjugate gradient following cpp/corelib/lib/op/cg.cppm:122-184.

Parity status: the reference publishes no golden vectors or fixtures for this path, and its
NUFFT is the third-party finufft/cufinufft (pinned only to ``master`` in CMakeLists.txt:175-181,
absent here). The NUFFT restatement is pinned to the FP64 NUDFT (its definition); the Toeplitz
load/store stage is pinned to the reference's own kernel source compiled here.
"""
