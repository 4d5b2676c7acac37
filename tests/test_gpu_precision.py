"""FP16 and BF16 deviation storage against FP64 storage on the GPU (the
precision study of fortran_loadfile_mitiwing_b200.precision, 3 periods of the
400x200 plunge case).

Tolerances: per-period mean C_D within 1% of |mean C_D| of the FP64 run, and
per-period mean C_L within 1% of the FP64 run's RMS of C_L (its mean is close
to zero): the bar stated for the FP16 form; velocity-field L2 error at the end
of period 3 below 1e-3 (FP16) and 3e-2 (BF16, 8-bit mantissa); FP32 storage
within 1e-5 on all of them.
"""
import pytest

from fortran_loadfile_mitiwing_b200 import precision

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def result(gpu_lib):
    return precision.study(periods=3, report=(3,), precisions=("fp16", "bf16", "fp32"), lib=gpu_lib)


@pytest.mark.parametrize("prec,vel_tol,coef_tol", [("fp16", 1e-3, 1e-2), ("bf16", 3e-2, 1e-2), ("fp32", 1e-5, 1e-5)])
def test_storage_precision_against_fp64(result, prec, vel_tol, coef_tol):
    r = result[prec]
    assert r["velocity_l2"]["3"] < vel_tol, r["velocity_l2"]
    for per in r["periods"]:
        assert per["cd_mean_err"] < coef_tol, per
        assert per["cl_mean_err"] < coef_tol, per
