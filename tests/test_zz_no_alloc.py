"""lbm_residual_device (the allocation-free residual on caller-owned device
fields) against lbm_residual on a handle, on two calls in a row.

Tolerance: relative 1e-12; both sum the same FP64 terms (fields widened from
their storage type), in different orders.
"""
import ctypes as C

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Lbm, cases
from fortran_loadfile_mitiwing_b200 import _abi

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _device(a, dtype):
    import torch
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_residual_device_matches_handle_residual(gpu_lib, precision):
    import torch
    dtype = torch.float64 if precision == "fp64" else torch.float32
    code = _abi.LBM_PREC_FP64 if precision == "fp64" else _abi.LBM_PREC_FP32
    case = cases.small_case(precision=precision, n_steps=100)
    g = Lbm.from_case(case, gpu_lib)
    g.run(5)
    _, u0, v0 = g.fields()
    side = torch.cuda.Stream()
    for call, stream in enumerate((None, C.c_void_p(side.cuda_stream))):
        g.evolution()
        _, u, v = g.fields()
        ref = g.erranalysis()
        bufs = [_device(a, dtype) for a in (u, v, u0, v0)]
        torch.cuda.synchronize()
        err = C.c_double(-1.0)
        st = gpu_lib.lbm_residual_device(*[C.c_void_p(b.data_ptr()) for b in bufs], g.nx, g.ny, code,
                                         stream, C.byref(err))
        assert st == _abi.LBM_OK, (call, st)
        assert ref > 0
        assert abs(err.value - ref) <= TOL * ref, (call, err.value, ref)
        u0, v0 = u, v
    g.close()


def test_residual_device_rejects_rows_beyond_its_scratch(gpu_lib):
    import torch
    b = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(b.data_ptr())
    err = C.c_double(-1.0)
    st = gpu_lib.lbm_residual_device(p, p, p, p, 4, _abi.LBM_RESIDUAL_MAX_ROWS + 3, _abi.LBM_PREC_FP64, None, C.byref(err))
    assert st == _abi.LBM_ERR_SIZE
    assert err.value == -1.0
