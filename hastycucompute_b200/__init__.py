"""hastycucompute_b200: B200-native (sm_100a) MRI reconstruction hot path of HastyCuCompute.

NUFFT type 1 / 2 (``nufft``), the Toeplitz-embedded normal operator and SENSE A^H A
(``toeplitz``, ``normal``) and conjugate gradient (``cg``), over the C ABI of libhasty_b200.so.
"""
from ._lib import HastyError, load as load_library  # noqa: F401
from .nufft import (  # noqa: F401
    NufftMethod,
    NufftOpts,
    NufftPlan,
    NufftSign,
    NufftType,
    NufftUpsamp,
    nufft_backward_cpu_over_cuda,
    nufft_type1,
    nufft_type2,
)
from .toeplitz import (  # noqa: F401
    ToeplitzAccumulateType,
    ToeplitzMultType,
    sense_normal,
    sense_normal_ex,
    toeplitz_kernel,
    toeplitz_kernels_frames,
    toeplitz_multiplication,
    toeplitz_multiply,
    transform_toeplitz_kernel,
)
from .normal import (  # noqa: F401
    BatchedNormalOp,
    BatchedSenseOp,
    NormalIDTT1Op,
    NormalIDTT2Op,
    NormalIDTWT1Op,
    NormalIDTWT2Op,
    NormalTT1Op,
    NormalTT2Op,
    SenseOffresOp,
    SenseOp,
    build_toeplitz_kernel,
    build_toeplitz_kernels,
)
from .cg import BatchedCGSolver, CGSolver, conjugate_gradient, conjugate_gradient_precond, vdot_real  # noqa: F401
from .alg import max_eig  # noqa: F401
from .pipeline import HostPipeline  # noqa: F401
from . import autograd  # noqa: F401

__version__ = "0.1.0"
