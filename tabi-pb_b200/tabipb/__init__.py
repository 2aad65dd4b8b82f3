"""tabipb -- B200 TABI-PB solve path (host mirror of the reference interface).

The numerics live in libtabi_gpu.so (sm_100a CUDA, tabi-pb_b200/csrc); this
package binds its C ABI (include/tabi_gpu.h) and provides the input formats.
"""
from ._lib import FLAG_PIVOTED_LU, PREC_FP64, PREC_MIXED, TabiError, load  # noqa: F401
from .solver import (TabiSolver, default_params, kappa, probe_fp32_peak, probe_fp64_peak,  # noqa: F401
                     solve_molecule)
