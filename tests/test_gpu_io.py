"""Output and restart files through a handle on the GPU: a checkpoint
restores the state exactly (the steps after a restart are bit-for-bit those
of the run that never stopped, in FP32 and FP16 storage), the loader falls
back to the copy when the file is damaged and refuses another grid, and
F<n>.dat carries the handle's fields and the airfoil contour of the last
step."""
import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Lbm, LbmError, cases

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
