"""partmc_b200: PartMC's particle-resolved coagulation step (mc_coag) on B200.

The hot path is CUDA in libpmc_coag_gpu.so behind the C ABI of
include/pmc_coag_gpu.h; this package is the host-side mirror of the
reference's interface for that path.
"""
from .coagulation import (AeroData, AeroDist, AeroMode, AeroState, AeroWeightArray, EnvState,  # noqa: F401
                          Fractal, HostMirror, mc_coag, mc_coag_batch,
                          COAG_KERNEL_TYPE_ADDITIVE, COAG_KERNEL_TYPE_BROWN, COAG_KERNEL_TYPE_CONSTANT,
                          COAG_KERNEL_TYPE_SEDI, COAG_KERNEL_TYPE_ZERO, COAG_KERNEL_TYPE_BROWN_FREE,
                          COAG_KERNEL_TYPE_BROWN_CONT, MODE_FP64, MODE_MIXED, MODE_REPLAY,
                          AERO_MODE_TYPE_LOG_NORMAL, AERO_MODE_TYPE_EXP, AERO_MODE_TYPE_MONO,
                          AERO_MODE_TYPE_SAMPLED)
from ._lib import PmcError  # noqa: F401
