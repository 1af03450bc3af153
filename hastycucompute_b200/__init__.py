"""hastycucompute_b200: B200-native (sm_100a) MRI reconstruction hot path of HastyCuCompute.

NUFFT type 1 / 2 (``nufft``), the Toeplitz-embedded normal operator and SENSE A^H A
(``toeplitz``, ``normal``) and conjugate gradient (``cg``), over the C ABI of libhasty_b200.so.
"""
from ._lib import HastyError, load as load_library  # noqa: F401
from .nufft import NufftMethod, NufftOpts, NufftPlan, NufftSign, NufftType, NufftUpsamp  # noqa: F401
from .toeplitz import (  # noqa: F401
    ToeplitzAccumulateType,
    ToeplitzMultType,
    sense_normal,
    toeplitz_kernel,
    toeplitz_multiplication,
    toeplitz_multiply,
    transform_toeplitz_kernel,
)
from .normal import NormalTT1Op, SenseOp, build_toeplitz_kernel  # noqa: F401
from .cg import CGSolver, conjugate_gradient, vdot_real  # noqa: F401

__version__ = "0.1.0"
