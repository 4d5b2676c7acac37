"""B200-native time step of the D2Q9 MRT lattice-Boltzmann flapping-airfoil
solver (immersed boundary, implicit velocity correction), behind the C ABI of
include/lbm_b200.h."""
from ._abi import (LBM_DELTA_PESKIN4, LBM_DELTA_SMOOTH, LBM_PREC_BF16, LBM_PREC_FP16, LBM_PREC_FP32,
                   LBM_PREC_FP64, LbmParams, load_library)
from .solver import Batch, Lbm, LbmError

__all__ = ["Batch", "Lbm", "LbmError", "LbmParams", "load_library", "LBM_PREC_FP32", "LBM_PREC_FP64",
           "LBM_PREC_FP16", "LBM_PREC_BF16", "LBM_DELTA_PESKIN4", "LBM_DELTA_SMOOTH"]
