"""Output and restart files through a handle on the GPU: a checkpoint
restores the state exactly (the steps after a restart are bit-for-bit those
of the run that never stopped, in FP32 and FP16 storage), the loader falls
back to the copy when the file is damaged and refuses another grid, and
F<n>.dat carries the handle's fields and the airfoil contour of the last
step. The reference's own restart file (saveflowfield layout) restarts a
handle bit for bit, carries the oracle's state into a handle within FP64
parity, falls back to the copy, and refuses free-flight state."""
import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Lbm, LbmError, cases, io_formats

pytestmark = pytest.mark.gpu

SPEC = dict(nx=96, ny=64, chord=24, pivot=(33, 33), markers=40, heave=0.25, pitch_deg=10.0, st=0.3, seed=7)


def make(precision, lib, **kw):
    return Lbm.from_case(cases.small_case(precision=precision, n_steps=200, **{**SPEC, **kw}), lib)


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_restart_continues_bit_for_bit(gpu_lib, tmp_path, precision):
    path = str(tmp_path / "saved_flow_feild.dat")
    with make(precision, gpu_lib) as a:
        a.run(13)
        a.save_checkpoint(path)
        rows_a = a.run(21)
        pops_a, res_a, n_a = a.populations(), a.erranalysis(), a.step_index
    assert (tmp_path / "saved_flow_feild_copy.dat").exists()
    with make(precision, gpu_lib) as b:
        b.load_checkpoint(path)
        assert b.step_index == 14
        rows_b = b.run(21)
        np.testing.assert_array_equal(rows_b, rows_a)
        np.testing.assert_array_equal(b.populations(), pops_a)
        assert b.erranalysis() == res_a and b.step_index == n_a


def test_damaged_checkpoint_falls_back_to_the_copy(gpu_lib, tmp_path):
    path = tmp_path / "ck.dat"
    with make("fp32", gpu_lib) as a:
        a.run(9)
        a.save_checkpoint(str(path))
        ref = a.run(6)
    raw = bytearray(path.read_bytes())
    raw[len(raw) // 2] ^= 0xFF
    path.write_bytes(bytes(raw))
    with make("fp32", gpu_lib) as b:
        b.load_checkpoint(str(path))
        np.testing.assert_array_equal(b.run(6), ref)
    copy = tmp_path / "ck_copy.dat"
    copy.write_bytes(copy.read_bytes()[:1000])
    with make("fp32", gpu_lib) as c:
        with pytest.raises(LbmError):
            c.load_checkpoint(str(path))
    with make("fp32", gpu_lib) as d, make("fp32", gpu_lib, nx=128, pivot=(40, 33)) as e:
        d.save_checkpoint(str(tmp_path / "other.dat"))
        with pytest.raises(LbmError):
            e.load_checkpoint(str(tmp_path / "other.dat"))


def test_tecplot_of_a_handle(gpu_lib, tmp_path):
    with make("fp32", gpu_lib) as s:
        s.run(10)
        path = s.write_tecplot(directory=str(tmp_path))
        assert path.endswith("F10.dat")
        rho, u, v = s.fields()
        xb2, yb2, _ = s.markers()
        p = s.params
    lines = open(path).read().split("\n")
    ny, nx = rho.shape
    onx, ony = (nx - 1) // 2 + 1, (ny - 1) // 2 + 1
    data = np.array([[float(l[k:k + 16]) for k in range(0, 128, 16)] for l in lines[2:2 + onx * ony]])
    assert data.shape == (onx * ony, 8)
    np.testing.assert_allclose(data[:, 2], (u[::2, ::2] / p.uu).reshape(-1), rtol=1e-7, atol=1e-12)
    np.testing.assert_allclose(data[:, 4], (rho[::2, ::2] / 3.0).reshape(-1), rtol=1e-7)
    np.testing.assert_allclose(data[:, 0], (p.ox + p.scale * np.arange(0, nx, 2))[None, :].repeat(ony, 0).reshape(-1),
                               rtol=1e-7, atol=1e-12)
    rest = lines[2 + onx * ony:]
    npts = p.points_per_wing
    pts = np.array([[float(l[k:k + 14]) for k in range(0, 28, 14)] for l in rest[1:1 + npts]])
    mid = 0.5 * (pts[1:] + pts[:-1])
    np.testing.assert_allclose(mid[:, 0], xb2, atol=2e-8)
    np.testing.assert_allclose(mid[:, 1], yb2, atol=2e-8)


def edges_of(f):
    """edge_f0 layout from populations (9, ny, nx): left, right, bottom, top."""
    return np.concatenate([f[:, :, 0].T, f[:, :, -1].T, f[:, 0, :].T, f[:, -1, :].T])


@pytest.mark.parametrize("precision", ["fp32", "fp16", "fp64"])
def test_reference_restart_file_continues_bit_for_bit(gpu_lib, tmp_path, precision):
    path = tmp_path / "saved_flow_feild.dat"
    with make("fp64", gpu_lib) as z:
        init_edges = edges_of(z.populations())     # f0 on the edges = the initial f there
    with make(precision, gpu_lib) as a:
        a.run(13)
        a.save_flow_field(str(path))
        _, u_a, v_a = a.fields()
        f_a = a.populations()
        rows_a = a.run(21)
        pops_a, n_a = a.populations(), a.step_index
    assert (tmp_path / "saved_flow_feild_copy.dat").read_bytes() == path.read_bytes()
    r = io_formats.read_flow_field_file(path, SPEC["nx"], SPEC["ny"], 1)
    assert r["cycle"] == 13 and r["movenum"] == 0 and not r["body_state"].any()
    for got, want in ((r["u"], u_a), (r["v"], v_a), (r["f"], f_a)):
        np.testing.assert_array_equal(got, want)
    # the file's edge f0 is init's feq; the FP64 handle's populations hold it
    # as a deviation from the weights plus the weights (a last-bit rounding)
    np.testing.assert_allclose(r["edge_f0"], init_edges, rtol=0, atol=1e-15)
    with make(precision, gpu_lib) as b:
        cyc, body, mv = b.read_flow_field(str(path))
        assert (cyc, mv, b.step_index) == (13, 0, 14) and body.shape == (11, 1)
        rho_b, u_b, v_b = b.fields()
        assert (rho_b == 1.0).all()
        np.testing.assert_array_equal(u_b, u_a)
        np.testing.assert_array_equal(v_b, v_a)
        rows_b = b.run(21)
        assert b.step_index == n_a
        if precision != "fp64":
            np.testing.assert_array_equal(rows_b, rows_a)
            np.testing.assert_array_equal(b.populations(), pops_a)
        else:
            # FP64 storage keeps f - w; the file's f = (f - w) + w drops the
            # deviation's bits below f's last bit, so the restart continues
            # within rounding instead of bit for bit
            assert np.abs(b.populations() - pops_a).max() < 1e-14
            np.testing.assert_allclose(rows_b, rows_a, rtol=1e-10, atol=1e-12)


def test_oracle_state_in_the_reference_file_restarts_a_handle(gpu_lib, oracle_mod, tmp_path):
    """The oracle (the reference's step restated in FP64) stands in for a
    reference run: its state after 17 steps, written in the reference's
    layout, restarts an FP64 handle, whose next 23 steps stay within FP64
    parity of the oracle's."""
    case = cases.small_case(precision="fp64", n_steps=200, pitch_deg=10.0)
    o = oracle_mod.Oracle.from_case(case)
    edges = edges_of(o.populations())
    o.run(17)
    _, u, v = o.fields()
    path = tmp_path / "saved_flow_feild.dat"
    io_formats.write_flow_field_file(path, 17, u, v, o.populations(), edges, body_state=np.zeros((11, 1)))
    with Lbm.from_case(case, gpu_lib) as g:
        assert g.read_flow_field(str(path))[0] == 17 and g.step_index == 18
        rg, ro = g.run(23), o.run(23)
        np.testing.assert_array_equal(rg[:, 0], ro[:, 0])
        assert np.abs(g.populations() - o.populations()).max() < 1e-11
        floor = np.sqrt(np.mean(ro[:, 1:7] ** 2, axis=0, keepdims=True))
        assert np.max(np.abs(rg[:, 1:7] - ro[:, 1:7]) / np.maximum(np.abs(ro[:, 1:7]), floor)) < 1e-8


def test_reference_restart_fallback_and_refusals(gpu_lib, tmp_path):
    path = tmp_path / "saved_flow_feild.dat"
    with make("fp32", gpu_lib) as a:
        a.run(9)
        a.save_flow_field(str(path))
        ref = a.run(6)
    path.write_bytes(path.read_bytes()[:4096])          # short primary: the copy is read
    with make("fp32", gpu_lib) as b:
        assert b.read_flow_field(str(path))[0] == 9
        np.testing.assert_array_equal(b.run(6), ref)
    r = io_formats.read_flow_field_file(tmp_path / "saved_flow_feild_copy.dat", SPEC["nx"], SPEC["ny"], 1)
    moved = tmp_path / "moved.dat"
    io_formats.write_flow_field_file(moved, 9, r["u"], r["v"], r["f"], r["edge_f0"], body_state=np.zeros((11, 1)),
                                     movenum=1)
    with make("fp32", gpu_lib) as c:
        with pytest.raises(LbmError, match="LBM_ERR_STATE"):     # free flight shifted the mesh
            c.read_flow_field(str(moved))
        assert c.step_index == 1
    two = tmp_path / "two_wings.dat"
    io_formats.write_flow_field_file(two, 9, r["u"], r["v"], r["f"], r["edge_f0"], body_state=np.zeros((11, 2)))
    with make("fp32", gpu_lib) as d:
        with pytest.raises(LbmError, match="wing count"):
            d.read_flow_field(str(two))


def test_checkpoint_carries_the_edge_populations(gpu_lib, tmp_path):
    """The library's checkpoint keeps the FP64 edge f0, so a handle restored
    from it (here one initialised with another perturbation) writes the same
    reference-layout restart file as the handle that saved it."""
    ck, p1, p2 = (str(tmp_path / n) for n in ("ck.dat", "a.dat", "b.dat"))
    with make("fp32", gpu_lib) as a:
        a.run(13)
        a.save_checkpoint(ck)
        a.save_flow_field(p1)
    with make("fp32", gpu_lib, seed=8) as b:
        b.load_checkpoint(ck)
        b.save_flow_field(p2)
    assert open(p1, "rb").read() == open(p2, "rb").read()
