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


def _host_residual(u, v, u0, v0):
    """erranalysis on host arrays (ny, nx): interior nodes only."""
    s = (slice(1, -1), slice(1, -1))
    du, dv = u[s] - u0[s], v[s] - v0[s]
    return np.sqrt(np.sum(du * du + dv * dv)) / (np.sqrt(np.sum(u[s] ** 2 + v[s] ** 2)) + 1e-30)


def test_residual_device_in_a_context_the_caller_created(gpu_lib):
    """A Fortran driver's CUDA runtime may work in a context it created itself
    instead of the device's primary context, and the scratch array sits at a
    different address in each context. The entry point looks the address up
    once per context: calls in the primary context, then (after a handle was
    created and destroyed) in a context made with the driver API, then in the
    primary context again, all give the residual computed on the host."""
    import torch
    cuda = C.CDLL("libcuda.so.1")
    for name in ("cuInit", "cuDeviceGet", "cuCtxCreate_v2", "cuCtxPopCurrent_v2", "cuCtxPushCurrent_v2",
                 "cuCtxDestroy_v2", "cuMemAlloc_v2", "cuMemFree_v2", "cuMemcpyHtoD_v2"):
        getattr(cuda, name).restype = C.c_int
    rng = np.random.default_rng(5)
    ny, nx = 70, 90
    u, v, u0, v0 = (rng.standard_normal((ny, nx)) * 0.05 for _ in range(4))
    ref = _host_residual(u, v, u0, v0)

    def call(ptrs):
        err = C.c_double(-1.0)
        st = gpu_lib.lbm_residual_device(*ptrs, nx, ny, _abi.LBM_PREC_FP64, None, C.byref(err))
        assert st == _abi.LBM_OK, st
        return err.value

    bufs = [_device(a, torch.float64) for a in (u, v, u0, v0)]
    torch.cuda.synchronize()
    assert abs(call([C.c_void_p(b.data_ptr()) for b in bufs]) - ref) <= TOL * ref
    g = Lbm.from_case(cases.small_case(precision="fp32", n_steps=20), gpu_lib)
    g.close()
    assert cuda.cuInit(0) == 0
    dev = C.c_int()
    assert cuda.cuDeviceGet(C.byref(dev), torch.cuda.current_device()) == 0
    ctx = C.c_void_p()
    assert cuda.cuCtxCreate_v2(C.byref(ctx), 0, dev) == 0   # current on this thread now
    ptrs = []
    try:
        for a in (u, v, u0, v0):
            p = C.c_ulonglong()
            assert cuda.cuMemAlloc_v2(C.byref(p), C.c_size_t(a.nbytes)) == 0
            ptrs.append(p)
            host = np.ascontiguousarray(a)
            assert cuda.cuMemcpyHtoD_v2(p, host.ctypes.data_as(C.c_void_p), C.c_size_t(a.nbytes)) == 0
        for _ in range(2):
            assert abs(call([C.c_void_p(p.value) for p in ptrs]) - ref) <= TOL * ref
    finally:
        for p in ptrs:
            cuda.cuMemFree_v2(p)
        popped = C.c_void_p()
        cuda.cuCtxPopCurrent_v2(C.byref(popped))
        cuda.cuCtxDestroy_v2(ctx)
    torch.cuda.synchronize()
    assert abs(call([C.c_void_p(b.data_ptr()) for b in bufs]) - ref) <= TOL * ref
