"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances:
  FP64 storage: max |f_gpu - f_oracle| <= 1e-11 (f ~ 0.03..0.44), fields
    likewise, force coefficients within 1e-8 relative (summation order only).
  FP32 storage, 400x200 plunge case, first 1000 steps (the low-Re parity
    window): populations, velocity field and per-step C_D/C_L within 1e-5
    relative; populations as max|df|/max|f|, velocity as ||du||/||u||, forces
    per step against max(|C|, rms C over the window) so that zero crossings of
    C_L are not divided by ~0. The same bars on the benchmarked 4096x2048
    heave + pitch case over its first 24 steps.
  FP32 storage, 400x200 plunge case, two whole periods after step 1000:
    per-period mean C_D within 0.5% of |mean C_D|, mean C_L within 0.5% of
    the RMS of C_L.
  FP64 storage, 400x200 plunge case, 1000 steps: populations and fields
    within 1e-10 absolute, force coefficients 1e-8 relative.
"""
import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Lbm, LbmError, cases, io_formats
from fortran_loadfile_mitiwing_b200 import _abi

pytestmark = pytest.mark.gpu


def run_both(case, nsteps, gpu_lib, oracle_mod, use_run=False):
    g = Lbm.from_case(case, gpu_lib)
    o = oracle_mod.Oracle.from_case(case)
    if use_run:
        rg = g.run(nsteps)
    else:
        rg = np.array([g.evolution() for _ in range(nsteps)])
    ro = o.run(nsteps)
    return g, o, rg, ro


def rel_series(a, b):
    floor = np.sqrt(np.mean(b * b, axis=0, keepdims=True))
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))


def test_fp64_parity_small_case(gpu_lib, oracle_mod):
    case = cases.small_case(precision="fp64", n_steps=200, pitch_deg=10.0)
    g, o, rg, ro = run_both(case, 100, gpu_lib, oracle_mod)
    assert np.abs(g.populations() - o.populations()).max() < 1e-11
    for a, b in zip(g.fields(), o.fields()):
        assert np.abs(a - b).max() < 1e-11
    np.testing.assert_array_equal(rg[:, 0], ro[:, 0])          # time column
    np.testing.assert_array_equal(rg[:, 7:], ro[:, 7:])        # motion columns
    assert rel_series(rg[:, 1:7], ro[:, 1:7]) < 1e-8
    xg, yg, res = g.markers()
    xo, yo, _ = o.markers()
    assert np.abs(xg - xo).max() < 1e-14 and np.abs(yg - yo).max() < 1e-14   # fused multiply-adds


def test_fp64_parity_two_wings_smooth_kernel(gpu_lib, oracle_mod):
    case = cases.small_case(nx=128, wings=2, delta=_abi.LBM_DELTA_SMOOTH, precision="fp64", n_steps=60)
    g, o, rg, ro = run_both(case, 40, gpu_lib, oracle_mod, use_run=True)
    assert np.abs(g.populations() - o.populations()).max() < 1e-11
    assert rel_series(rg[:, 1:10], ro[:, 1:10]) < 1e-8


def test_fp64_parity_without_body(gpu_lib, oracle_mod):
    case = cases.small_case(wings=0, precision="fp64", n_steps=40)
    g, o, rg, ro = run_both(case, 30, gpu_lib, oracle_mod)
    assert np.abs(g.populations() - o.populations()).max() < 1e-12
    for a, b in zip(g.fields(), o.fields()):
        assert np.abs(a - b).max() < 1e-12


def test_fp32_parity_plunge_400x200_first_1000_steps(gpu_lib, oracle_mod):
    case = cases.plunge_case(precision="fp32", n_steps=4000)
    g, o, rg, ro = run_both(case, 1000, gpu_lib, oracle_mod, use_run=True)
    fg, fo = g.populations(), o.populations()
    assert np.abs(fg - fo).max() / np.abs(fo).max() < 1e-5
    _, ug, vg = g.fields()
    _, uo, vo = o.fields()
    vel = np.sqrt(np.sum((ug - uo) ** 2 + (vg - vo) ** 2) / np.sum(uo ** 2 + vo ** 2))
    assert vel < 1e-5
    assert rel_series(rg[:, 1:3], ro[:, 1:3]) < 1e-5


def test_fp32_parity_odd_rows(gpu_lib, oracle_mod):
    """An odd number of interior rows (59) leaves the lattice update's last
    row unpaired; FP32 stays within the parity tolerance of the oracle."""
    case = cases.small_case(nx=100, ny=61, chord=20, pivot=(35, 31), markers=36, precision="fp32", n_steps=300)
    g, o, rg, ro = run_both(case, 200, gpu_lib, oracle_mod, use_run=True)
    fg, fo = g.populations(), o.populations()
    assert np.abs(fg - fo).max() / np.abs(fo).max() < 1e-5
    assert rel_series(rg[:, 1:4], ro[:, 1:4]) < 1e-5


def test_step_and_run_agree_bitwise(gpu_lib):
    case = cases.small_case(precision="fp32", n_steps=100)
    a = Lbm.from_case(case, gpu_lib)
    b = Lbm.from_case(case, gpu_lib)
    ra = np.array([a.evolution() for _ in range(25)])
    rb = b.run(25)
    np.testing.assert_array_equal(a.populations(), b.populations())
    np.testing.assert_array_equal(ra, rb)


def test_timing_modes(gpu_lib):
    """LBM_TIMING_SPAN times the steps with events at the ends of the call
    only (kernel totals stay 0); LBM_TIMING_KERNELS also times the lattice
    kernel and the IB chain of every step. Neither changes the results."""
    import ctypes as C
    case = cases.small_case(precision="fp32", n_steps=100)
    a, b = Lbm.from_case(case, gpu_lib), Lbm.from_case(case, gpu_lib)
    ra = a.run(30)
    out = []
    for mode in (_abi.LBM_TIMING_SPAN, _abi.LBM_TIMING_KERNELS):
        assert gpu_lib.lbm_set_timing(b.h, mode) == 0
        rows = b.run(15)
        t = [C.c_double() for _ in range(3)]
        n = C.c_int()
        gpu_lib.lbm_get_timing(b.h, *(C.byref(x) for x in t), C.byref(n))
        out.append((rows, [x.value for x in t], n.value))
    (r1, t1, n1), (r2, t2, n2) = out
    assert n1 == 15 and n2 == 15
    assert t1[0] > 0 and t1[1] == 0 and t1[2] == 0
    assert t2[0] > 0 and t2[1] > 0 and t2[2] > 0
    np.testing.assert_array_equal(np.concatenate([r1, r2]), ra)


def test_launch_count_per_step(gpu_lib):
    """Per step of one rigid wing: the flow chain (interpolation, solve, update
    of the correction tiles, force row) and the lattice kernel; the residual
    check on the last step of each batch of 4 steps and of the call; the mass
    check at the end of the call; per batch of steps, the six kernels of the
    batched factorization of the marker system (geometry, band assembly,
    factorization, patch-tile lists in three passes)."""
    import ctypes as C
    case = cases.small_case(precision="fp32", n_steps=100)
    g = Lbm.from_case(case, gpu_lib)
    g.run(1)
    n0, n1 = C.c_longlong(), C.c_longlong()
    assert gpu_lib.lbm_get_launch_count(g.h, C.byref(n0)) == 0
    steps = 12
    g.run(steps)
    gpu_lib.lbm_get_launch_count(g.h, C.byref(n1))
    total = n1.value - n0.value
    per_step = 4 + 1
    # steps n = 2 .. 13: checked where (n + 1) % 4 == 0 (3, 7, 11) and the last (13)
    checks = sum(1 for n in range(2, 2 + steps) if (n + 1) % 4 == 0 or n == 1 + steps)
    rest = total - steps * per_step - checks - 1
    assert rest > 0 and rest % 6 == 0, total
    assert 1 <= rest // 6 <= steps, total


def test_residual_matches_oracle(gpu_lib, oracle_mod):
    case = cases.small_case(precision="fp64", n_steps=100)
    g = Lbm.from_case(case, gpu_lib)
    o = oracle_mod.Oracle.from_case(case)
    g.evolution()
    o.evolution()
    assert abs(g.erranalysis() - o.erranalysis()) < 1e-10
    g.run(10)
    o.run(10)
    assert abs(g.erranalysis() - o.erranalysis()) < 1e-10 * max(1.0, o.erranalysis())


def test_range_error_is_reported(gpu_lib):
    case = cases.small_case(pivot=(8, 33), precision="fp32")
    g = Lbm.from_case(case, gpu_lib)
    with pytest.raises(LbmError) as ei:
        g.evolution()
    assert ei.value.status == _abi.LBM_ERR_RANGE


def test_run_stops_at_motion_end(gpu_lib):
    case = cases.small_case(n_steps=7)
    g = Lbm.from_case(case, gpu_lib)
    rows = g.run(20)
    assert rows.shape[0] == 7
    assert g.evolution() is None
    assert g.step_index == 8


def test_step_before_init_is_refused(gpu_lib):
    case = cases.small_case()
    g = Lbm(case.params, gpu_lib)
    with pytest.raises(LbmError) as ei:
        g.evolution()
    assert ei.value.status == _abi.LBM_ERR_STATE


def test_file_inputs_match_memory_inputs(gpu_lib, tmp_path):
    case = cases.small_case(precision="fp64", n_steps=30)
    io_formats.write_boundary(tmp_path / "boundary.dat", *case.contours[0])
    io_formats.write_motion(tmp_path / "motion_params.dat", case.table)
    a = Lbm.from_case(case, gpu_lib)
    b = Lbm(case.params, gpu_lib)
    b.read_boundary(str(tmp_path))
    b.load_motion_table(str(tmp_path / "motion_params.dat"))
    b.init(case.du, case.dv)
    ra, rb = a.run(20), b.run(20)
    np.testing.assert_array_equal(ra, rb)
    np.testing.assert_array_equal(a.populations(), b.populations())


def test_populations_round_trip(gpu_lib):
    case = cases.small_case(precision="fp64", n_steps=30)
    g = Lbm.from_case(case, gpu_lib)
    g.run(5)
    f = g.populations()
    g.set_populations(f)
    np.testing.assert_array_equal(g.populations(), f)


def test_checkpoint_restart_continues_identically(gpu_lib):
    case = cases.small_case(precision="fp32", n_steps=60)
    a = Lbm.from_case(case, gpu_lib)
    a.run(20)
    f = a.populations()
    ra = a.run(10)
    b = Lbm.from_case(case, gpu_lib)
    b.run(20)
    b.set_populations(f)
    rb = b.run(10)
    np.testing.assert_array_equal(ra, rb)


def test_banded_and_dense_solves_agree(gpu_lib, oracle_mod):
    """The block cyclic reduction and the dense Cholesky give the oracle's
    correction; the banded path is the one taken for this layout."""
    case = cases.small_case(precision="fp64", n_steps=40, pitch_deg=20.0)
    dense = cases.small_case(precision="fp64", n_steps=40, pitch_deg=20.0)
    dense.params.flags = _abi.LBM_FLAG_DENSE_SOLVE
    a = Lbm.from_case(case, gpu_lib)
    b = Lbm.from_case(dense, gpu_lib)
    o = oracle_mod.Oracle.from_case(case)
    ra, rb, ro = a.run(30), b.run(30), o.run(30)
    _, _, res_a, w_a = a.solver_info()
    _, _, res_b, _ = b.solver_info()
    assert w_a <= 16 and res_a < 1e-12 and res_b < 1e-12
    assert np.abs(a.populations() - o.populations()).max() < 1e-11
    assert np.abs(b.populations() - o.populations()).max() < 1e-11
    assert rel_series(ra[:, 1:4], ro[:, 1:4]) < 1e-8
    assert rel_series(rb[:, 1:4], ro[:, 1:4]) < 1e-8


def test_large_case_short_run_properties(gpu_lib):
    """4096x2048, 1024 markers: a few steps stay finite, the marker system is
    solved to FP64 accuracy on the banded path, mass drifts only by boundary flux."""
    case = cases.heave_pitch_case(n_steps=40, precision="fp32")
    s = Lbm.from_case(case, gpu_lib)
    rows = s.run(12)
    assert np.all(np.isfinite(rows))
    _, _, res, w = s.solver_info()
    assert w <= 16 and res < 1e-10
    rho, u, v = s.fields()
    assert np.all(np.isfinite(u)) and abs(rho.mean() - 1.0) < 1e-3


def _period_means(rows, start, period):
    """Per-period means of the force columns 1..2 (C_D, C_L of wing 1) over
    whole periods from `start` on."""
    n = (rows.shape[0] - start) // period
    return np.array([rows[start + p * period:start + (p + 1) * period, 1:3].mean(axis=0) for p in range(n)])


def test_fp32_parity_plunge_400x200_two_periods_after_step_1000(gpu_lib, oracle_mod):
    """The second parity bar on the 400x200 plunge case: after the first 1000
    steps, the per-period mean C_D within 0.5% of |mean C_D| of the oracle,
    and the per-period mean C_L within 0.5% of the oracle's RMS C_L (its mean
    is close to 0), over two whole periods (2 x 2667 steps)."""
    period = 2667   # 1 / (f* dt) = 1 / (0.6 * 6.25e-4) = 2666.7 steps
    nsteps = 1000 + 2 * period
    case = cases.plunge_case(precision="fp32", n_steps=nsteps + 8)
    g = Lbm.from_case(case, gpu_lib)
    o = oracle_mod.Oracle.from_case(case)
    rg = g.run(nsteps)
    ro = o.run(nsteps)
    assert rg.shape == ro.shape == (nsteps, g.row_len)
    mg, mo = _period_means(rg, 1000, period), _period_means(ro, 1000, period)
    assert mg.shape == (2, 2)
    rms_cl = np.sqrt(np.mean(ro[1000:, 2] ** 2))
    err_cd = np.abs(mg[:, 0] - mo[:, 0]) / np.abs(mo[:, 0])
    err_cl = np.abs(mg[:, 1] - mo[:, 1]) / rms_cl
    assert err_cd.max() < 5e-3, err_cd
    assert err_cl.max() < 5e-3, err_cl


def test_fp64_parity_plunge_400x200_first_1000_steps(gpu_lib, oracle_mod):
    """FP64 storage (the GPU FP64 oracle of the precision study) against the
    CPU oracle over the first 1000 steps of the 400x200 plunge case, the size
    the study runs at: populations within 1e-10 absolute (rounding of two
    different summation orders, accumulated over 1000 steps), fields likewise,
    per-step force coefficients within 1e-8 relative."""
    case = cases.plunge_case(precision="fp64", n_steps=1010)
    g, o, rg, ro = run_both(case, 1000, gpu_lib, oracle_mod, use_run=True)
    assert np.abs(g.populations() - o.populations()).max() < 1e-10
    for a, b in zip(g.fields(), o.fields()):
        assert np.abs(a - b).max() < 1e-10
    assert rel_series(rg[:, 1:4], ro[:, 1:4]) < 1e-8


def test_fp32_parity_heave_pitch_4096x2048_first_24_steps(gpu_lib, oracle_mod):
    """The benchmarked case (4096x2048, 1024 markers, heave + pitch, FP32
    storage) against the oracle over its first 24 steps: populations
    (max|df|/max|f|), velocity field (||du||/||u||) and per-step C_D/C_L/C_M
    within 1e-5 relative, the FP32 tolerance."""
    case = cases.heave_pitch_case(n_steps=40, precision="fp32")
    g, o, rg, ro = run_both(case, 24, gpu_lib, oracle_mod, use_run=True)
    assert rel_series(rg[:, 1:4], ro[:, 1:4]) < 1e-5
    np.testing.assert_array_equal(rg[:, 0], ro[:, 0])
    fg = g.populations()
    fo = o.populations()
    assert np.abs(fg - fo).max() / np.abs(fo).max() < 1e-5
    del fg, fo
    _, ug, vg = g.fields()
    _, uo, vo = o.fields()
    vel = np.sqrt(np.sum((ug - uo) ** 2 + (vg - vo) ** 2) / np.sum(uo ** 2 + vo ** 2))
    assert vel < 1e-5
    g.close()
    o.close()


def test_library_kernels_are_sm100a(gpu_lib):
    """The loaded kernels are sm_100a code (cudaFuncAttributes::binaryVersion)
    and the device is a B200-class part."""
    import ctypes as C
    ver, sms = C.c_int(), C.c_int()
    assert gpu_lib.lbm_device_check(C.byref(ver), C.byref(sms)) == 0
    assert ver.value == 100
    assert sms.value >= 132
