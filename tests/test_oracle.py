"""Property tests that pin the CPU oracle (no GPU). The reference ships no
tests or golden vectors, so these properties are what the oracle is checked
against before it checks the CUDA path."""
import math
import os

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import cases


def test_mrt_matrix_inverse(oracle_mod):
    m, mi = oracle_mod.mrt_matrices()
    assert np.abs(m @ mi - np.eye(9)).max() < 1e-15
    # rows of M are orthogonal: M^-1 = M^T diag(1/|row|^2)
    exact = m.T / (m * m).sum(axis=1)
    assert np.abs(mi - exact).max() < 1e-16


def test_lattice_order_and_single_precision_weights(oracle_mod):
    e, w = oracle_mod.lattice()
    assert e.tolist() == [[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]]
    assert w[0] == float(np.float32(4.0) / np.float32(9.0))
    assert w[1] == float(np.float32(1.0) / np.float32(9.0))
    assert w[5] == float(np.float32(1.0) / np.float32(36.0))
    assert w[0] != 4.0 / 9.0   # the REAL*4 quotient, not the FP64 one


@pytest.mark.parametrize("smooth,support", [(0, 2.0), (1, 2.5)])
def test_delta_kernel_partition_of_unity_and_symmetry(oracle_mod, smooth, support):
    rng = np.random.default_rng(1)
    for r0 in rng.uniform(0.0, 1.0, 50):
        vals = [oracle_mod.delta(r0 + i, smooth) for i in range(-4, 5)]
        assert abs(sum(vals) - 1.0) < 1e-14
        first = sum((r0 + i) * v for i, v in zip(range(-4, 5), vals))
        assert abs(first) < 1e-14
    for r in rng.uniform(0.0, 3.0, 50):
        assert oracle_mod.delta(r, smooth) == oracle_mod.delta(-r, smooth)
    assert oracle_mod.delta(support + 1e-9, smooth) == 0.0
    assert oracle_mod.delta(support + 0.3, smooth) == 0.0


def test_peskin_kernel_values(oracle_mod):
    # phi(0) = 1/2, phi(1) = 1/4, phi(0.5) = (3-1+sqrt(2))/8
    assert abs(oracle_mod.delta(0.0, 0) - 0.5) < 1e-16
    assert abs(oracle_mod.delta(1.0, 0) - 0.25) < 1e-16
    assert abs(oracle_mod.delta(0.5, 0) - (2.0 + math.sqrt(2.0)) / 8.0) < 1e-16


def test_motion_lookup_rows_and_interpolation(oracle_mod):
    t = np.array([0.0, 0.1, 0.2, 0.4])
    table = np.stack([t, 10 * t, t * t], axis=1)
    np.testing.assert_array_equal(oracle_mod.motion_lookup(table, 0.1), table[1])
    r = oracle_mod.motion_lookup(table, 0.3)
    assert abs(r[1] - 3.0) < 1e-12 and abs(r[2] - 0.1) < 1e-12   # linear between rows
    np.testing.assert_array_equal(oracle_mod.motion_lookup(table, -1.0), [-1.0, table[0, 1], table[0, 2]])
    np.testing.assert_array_equal(oracle_mod.motion_lookup(table, 9.0), [9.0, table[3, 1], table[3, 2]])


def _small(oracle_mod, **kw):
    c = cases.small_case(**kw)
    return c, oracle_mod.Oracle.from_case(c)


def test_motion_table_rejects_decreasing_time(oracle_mod):
    c = cases.small_case()
    o = oracle_mod.Oracle(c.params)
    bad = c.table.copy()
    bad[5, 0] = bad[3, 0]
    with pytest.raises(oracle_mod.OracleError):
        o.set_motion_table(bad)
    with pytest.raises(oracle_mod.OracleError):
        o.set_motion_table(c.table[:, :5])


def test_streaming_is_a_pull_permutation(oracle_mod):
    c, o = _small(oracle_mod)
    f_prev = o.populations().copy()
    o.evolution()
    f0 = o.streamed()
    e, _ = oracle_mod.lattice()
    for k in range(9):
        ex, ey = e[k]
        src = f_prev[k, 1 - ey:c.params.ny - 1 - ey, 1 - ex:c.params.nx - 1 - ex]
        np.testing.assert_array_equal(f0[k, 1:-1, 1:-1], src)


def test_collision_conserves_mass_and_momentum_off_body(oracle_mod):
    c, o = _small(oracle_mod)
    o.evolution()
    f0, f = o.streamed(), o.populations()
    gx, gy = o.gforce()
    e, _ = oracle_mod.lattice()
    free = (gx == 0) & (gy == 0)
    free[0, :] = free[-1, :] = False
    free[:, 0] = free[:, -1] = False
    assert free.sum() > 0.9 * free.size * 0.8
    for comp in (np.ones(9), e[:, 0], e[:, 1]):
        a = np.tensordot(comp, f0, axes=(0, 0))[free]
        b = np.tensordot(comp, f, axes=(0, 0))[free]
        assert np.abs(a - b).max() < 5e-15


def test_ib_interpolated_velocity_equals_body_velocity(oracle_mod):
    """Defining property of the implicit scheme: after the correction the
    delta-interpolated velocity at each marker is the marker velocity."""
    c, o = _small(oracle_mod, pitch_deg=10.0)
    for _ in range(3):
        row = o.evolution()
    p = c.params
    rho, u, v = o.fields()
    xm, ym, res = o.markers()
    assert res < 1e-12
    wing_row = row
    sa, sau, saac, sb, sbv, sbac, angle, omega, omgac = wing_row[7:16]
    x0, y0 = c.contours[0]
    xbar = 0.5 * (x0[1:] + x0[:-1])
    ybar = 0.5 * (y0[1:] + y0[:-1])
    ub = p.uu * (-omega * math.sin(angle) * xbar + omega * math.cos(angle) * ybar + sau)
    vb = p.uu * (-omega * math.cos(angle) * xbar - omega * math.sin(angle) * ybar + sbv)
    for k in range(len(xm)):
        ic = (xm[k] - p.ox) / p.scale
        jc = (ym[k] - p.oy) / p.scale
        su = sv = 0.0
        for i in range(int(ic) - 3, int(ic) + 4):
            for j in range(int(jc) - 3, int(jc) + 4):
                wgt = oracle_mod.delta(i - ic, p.delta_kernel) * oracle_mod.delta(j - jc, p.delta_kernel)
                su += wgt * u[j, i]
                sv += wgt * v[j, i]
        assert abs(su - ub[k]) < 1e-11 * p.uu * 100
        assert abs(sv - vb[k]) < 1e-11 * p.uu * 100


def test_force_row_is_normalised_sum_of_force_density(oracle_mod):
    c, o = _small(oracle_mod)
    for _ in range(4):
        row = o.evolution()
    p = c.params
    gx, gy = o.gforce()
    chord = 1.0 / p.scale
    cx = 2.0 * (-gx.sum()) / (p.uu * p.uu * chord)
    cy = 2.0 * (-gy.sum()) / (p.uu * p.uu * chord)
    assert abs(cx - row[1]) < 1e-9 * max(1.0, abs(cx))
    assert abs(cy - row[2]) < 1e-9 * max(1.0, abs(cy))
    # moment about the moving pivot (boundary_condition.f90:1672-1674)
    jj, ii = np.nonzero((gx != 0) | (gy != 0))
    sa, sb = row[7], row[10]
    x0 = (p.ox + p.scale * ii - (p.xc + sa)) / p.scale
    y0 = (p.oy + p.scale * jj - (p.yc + sb)) / p.scale
    mom = np.sum(-x0 * gy[jj, ii] + y0 * gx[jj, ii])
    cm = -2.0 * mom / (p.uu * p.uu * chord * chord)
    assert abs(cm - row[3]) < 1e-9 * max(1.0, abs(cm))
    # totals equal the single wing
    np.testing.assert_allclose(row[4:7], row[1:4], rtol=0, atol=1e-12)


def test_erranalysis_matches_definition(oracle_mod):
    c, o = _small(oracle_mod)
    o.evolution()
    _, u1, v1 = [a.copy() for a in o.fields()]
    o.evolution()
    _, u2, v2 = o.fields()
    s = (slice(1, -1), slice(1, -1))
    t1 = np.sum((u2[s] - u1[s]) ** 2 + (v2[s] - v1[s]) ** 2)
    t2 = np.sum(u2[s] ** 2 + v2[s] ** 2)
    assert abs(o.erranalysis() - math.sqrt(t1) / (math.sqrt(t2) + 1e-30)) < 1e-14


def test_top_bottom_rows_and_stale_edge_f0(oracle_mod):
    c, o = _small(oracle_mod)
    f_init = o.populations().copy()
    for _ in range(3):
        o.evolution()
    rho, u, v = o.fields()
    for row, nbr in ((0, 1), (-1, -2)):
        assert np.all(u[row] == 0.0) and np.all(v[row] == 0.0)
        np.testing.assert_array_equal(rho[row], rho[nbr])
    f0 = o.streamed()
    # streaming never rewrites the edge f0 (solution.f90:440-447)
    np.testing.assert_array_equal(f0[:, 0, :], f_init[:, 0, :])
    np.testing.assert_array_equal(f0[:, :, -1], f_init[:, :, -1])


def test_range_error_when_body_reaches_edge(oracle_mod):
    c = cases.small_case(pivot=(8, 33))
    o = oracle_mod.Oracle.from_case(c)
    with pytest.raises(oracle_mod.OracleError, match="-7"):
        o.evolution()


def test_run_stops_at_motion_end(oracle_mod):
    c = cases.small_case(n_steps=5)
    o = oracle_mod.Oracle.from_case(c)
    rows = o.run(10)
    assert rows.shape[0] == 5
    assert o.evolution() is None


def test_two_wings_and_smooth_kernel_step(oracle_mod):
    c, o = _small(oracle_mod, nx=128, wings=2, delta=1)
    rows = o.run(5)
    assert rows.shape == (5, 1 + 6 + 3 + 18)
    assert np.all(np.isfinite(rows))
    np.testing.assert_allclose(rows[:, 7], rows[:, 1] + rows[:, 4], rtol=1e-13, atol=1e-13)


def test_no_body_runs(oracle_mod):
    c = cases.small_case(wings=0)
    o = oracle_mod.Oracle.from_case(c)
    rows = o.run(3)
    assert rows.shape == (3, 4)
    assert np.all(rows[:, 1:] == 0.0)


def test_geometry_generator_reproduces_reference_boundary_file():
    """naca0012(204) is the layout of the reference's own boundary.dat
    (tests/golden/reference_boundary.dat is that file, byte for byte: the
    205-point closed NACA 0012 contour in chords, (2f14.8))."""
    ref = os.path.join(os.path.dirname(__file__), "golden", "reference_boundary.dat")
    d = np.loadtxt(ref)
    assert d.shape == (205, 2)
    x, y = cases.naca0012(204)
    assert np.abs(x - d[:, 0]).max() < 1.5e-8
    assert np.abs(y - d[:, 1]).max() < 1.5e-8


def _reference_constants():
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_constants.json")) as fh:
        return json.load(fh)


def test_oracle_model_constants_equal_the_reference_source(oracle_mod):
    """M, the lattice order and the weights as the reference's source writes
    them (tests/golden/make_reference_constants.py extracted them)."""
    ref = _reference_constants()
    m, _ = oracle_mod.mrt_matrices()
    np.testing.assert_array_equal(m, np.array(ref["matm"]))
    e, w = oracle_mod.lattice()
    assert e.tolist() == ref["e"]
    for k, lit in enumerate(ref["w_literal"]):
        # a default-REAL quotient (no d0 exponent): evaluated in single precision
        num, den = (float(x) for x in lit.split("/"))
        assert "d" not in lit.lower()
        assert w[k] == float(np.float32(num) / np.float32(den))


def test_default_rates_equal_the_reference_source():
    """lbm_default_params carries the reference's s(1..7); s(8), s(9) are
    1/tau_f there and <= 0 here, meaning 'from the viscosity'."""
    import ctypes as C
    from fortran_loadfile_mitiwing_b200 import LbmParams, load_library
    ref = _reference_constants()
    p = LbmParams()
    assert load_library().lbm_default_params(C.byref(p)) == 0
    for k in range(7):
        assert p.s[k] == float(ref["s_literal"][k].lower().replace("d", "e"))
    assert all("tau_f" in ref["s_literal"][k] for k in (7, 8)) and p.s[7] <= 0 and p.s[8] <= 0


def _fortran_to_python(expr):
    import re
    expr = re.sub(r"(\d+\.\d*)[dD]([+-]?\d+)", r"\1e\2", expr)
    for a, b in ((".lt.", " < "), (".le.", " <= "), (".gt.", " > "), (".ge.", " >= "), (".and.", " and "),
                 (".or.", " or ")):
        expr = expr.replace(a, b).replace(a.upper(), b)
    return expr


@pytest.mark.parametrize("smooth", [0, 1])
def test_oracle_delta_kernels_equal_the_reference_source(oracle_mod, smooth):
    """The oracle's one-axis kernels against the reference's branch formulas,
    evaluated as written (tests/golden/reference_constants.json), over a grid
    of distances that includes every branch boundary."""
    ref = _reference_constants()
    env = {"abs": abs, "sqrt": math.sqrt, "asin": math.asin,
           "pai": float(_fortran_to_python(ref["pai_literal"]))}
    branches = [(None if c == "else" else _fortran_to_python(c), _fortran_to_python(e))
                for c, e in ref["kernel_branches"][str(smooth)]]
    rs = sorted(set(np.round(np.linspace(0.0, 3.0, 601), 12).tolist() + [0.5, 1.0, 1.5, 2.0, 2.5]))
    for r in rs:
        env["disr"] = r
        want = next(eval(e, env) for c, e in branches if c is None or eval(c, env))
        got = oracle_mod.delta(r, smooth)
        assert abs(got - want) <= 1e-15 * max(1.0, abs(want)), (smooth, r, got, want)


def test_oracle_initial_state_is_the_reference_equilibrium(oracle_mod):
    """init's populations (solution.f90:33-59) are D2Q9feq(1, UU + du, dv) as
    the reference source writes it, with its single-precision weights."""
    from fortran_loadfile_mitiwing_b200 import cases
    ref = _reference_constants()
    case = cases.small_case(precision="fp64", n_steps=10)
    o = oracle_mod.Oracle.from_case(case)
    f = o.populations()
    p = case.params
    ny, nx = f.shape[1:]
    du, dv = case.du.reshape(ny, nx), case.dv.reshape(ny, nx)
    e = ref["e"]
    w = [float(np.float32(float(a)) / np.float32(float(b))) for a, b in (x.split("/") for x in ref["w_literal"])]
    code = {k: compile(_fortran_to_python(v), k, "eval") for k, v in ref["feq"].items()}
    for j, i in ((0, 0), (5, 7), (ny // 2, nx // 2), (ny - 1, nx - 1), (13, 41)):
        # Fortran's 1-based e(k,c) and w(k)
        env = {"rh": 1.0, "u1": p.uu + du[j, i], "v1": 0.0 + dv[j, i],
               "e": lambda a, c: e[a - 1][c - 1], "w": lambda a: w[a - 1]}
        for k in range(9):
            env["k"] = k + 1
            env["eu"] = eval(code["eu"], env)
            env["utwo"] = eval(code["utwo"], env)
            want = eval(code["D2Q9feq"], env)
            assert abs(f[k, j, i] - want) <= 2e-16, (k, j, i, f[k, j, i], want)


def test_oracle_collision_is_the_reference_colission(oracle_mod):
    """One node of colission as the reference source writes it (equilibrium
    moments temp(k), forcing fp(k), relaxation; solution.f90:592-635),
    evaluated as written with sequential matrix-vector sums, against the
    oracle's collision, at random node states with and without force."""
    from fortran_loadfile_mitiwing_b200 import cases
    import pyoracle
    ref = _reference_constants()["collision"]
    case = cases.small_case(precision="fp64", n_steps=10)
    o = oracle_mod.Oracle.from_case(case)
    m, minv = oracle_mod.mrt_matrices()
    s_rates = [float(x) for x in o.params.s]
    if s_rates[7] <= 0:   # 1/tau from the viscosity, as the library fills them
        nu = o.params.uu / (o.params.re * o.params.scale)
        s_rates[7] = s_rates[8] = 1.0 / (3.0 * nu + 0.5)
    temp_c = [compile(_fortran_to_python(e.replace("mesh%s(", "s(")), "temp", "eval") for e in ref["temp"]]
    fp_c = [compile(_fortran_to_python(e.replace("mesh%s(", "s(")), "fp", "eval") for e in ref["fp"]]

    def matmulvoc(a, b):   # boundary_condition.f90:1738-1755: sums in column order
        out = []
        for i in range(9):
            acc = 0.0
            for j in range(9):
                acc = acc + a[i][j] * b[j]
            out.append(acc)
        return out

    rng = np.random.default_rng(11)
    e_, w_ = oracle_mod.lattice()
    for trial in range(20):
        rt = 1.0 + rng.uniform(-0.02, 0.02)
        ut, vt = rng.uniform(-0.08, 0.08, 2)
        gfx, gfy = (0.0, 0.0) if trial % 2 == 0 else rng.uniform(-1e-3, 1e-3, 2)
        f = w_ * rt * (1.0 + 3.0 * (e_ @ [ut, vt])) + rng.uniform(-1e-3, 1e-3, 9)
        got = pyoracle.collide_node(o, f, rt, ut, vt, gfx, gfy)
        env = {"rt": rt, "ut": ut, "vt": vt, "gfx": gfx, "gfy": gfy, "s": lambda k: s_rates[k - 1]}
        temp1 = matmulvoc(m, f)
        temp = [eval(c, env) for c in temp_c]
        fp = [eval(c, env) for c in fp_c]
        temp = [temp1[k] + (temp[k] - temp1[k]) * s_rates[k] + fp[k] for k in range(9)]
        want = matmulvoc(minv, temp)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-16)
    assert ref["relax"].replace(" ", "") == "temp(k)=temp1(k)+(temp(k)-temp1(k))*mesh%s(k)+fp(k)"
