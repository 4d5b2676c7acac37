"""Output files on the CPU: the library's F<n>.dat writer against a
restatement of the reference's output routine (solution.f90:165-235) in
Python, byte for byte on the data lines, and the airfoil_motion.dat rows
(solution.f90:379-390). The handle-based writer and the checkpoint are GPU
tests (test_gpu_io.py)."""
import math

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import io_formats


def fortran_e(x, w=16, d=8):
    """Ew.d: 0.d1..dd E+xx (E dropped for a 3-digit exponent), right-justified."""
    if x == 0.0:
        s = ("-" if math.copysign(1.0, x) < 0 else "") + "0." + "0" * d + "E+00"
    else:
        m, e = f"{abs(x):.{d - 1}e}".split("e")
        digits = m.replace(".", "")
        ex = int(e) + 1
        body = f"0.{digits}" + (f"E{'-' if ex < 0 else '+'}{abs(ex):02d}" if abs(ex) <= 99
                                else f"{'-' if ex < 0 else '+'}{abs(ex):03d}")
        s = ("-" if x < 0 else "") + body
    return "*" * w if len(s) > w else s.rjust(w)


def reference_field_lines(rho, u, v, ox, oy, scale, uu, sx, sy):
    """solution.f90:175-210, 0-based indices."""
    ny, nx = rho.shape
    out = []
    for j in range(0, ny, sy):
        for i in range(0, nx, sx):
            if i == nx - 1:
                dvx = (1.5 * v[j, i] - 2.0 * v[j, i - 1] + 0.5 * v[j, i - 2]) / (uu * scale)
            elif i == 0:
                dvx = (-1.5 * v[j, i] + 2.0 * v[j, i + 1] - 0.5 * v[j, i + 2]) / (uu * scale)
            else:
                dvx = (v[j, i + 1] - v[j, i - 1]) / (uu * 2.0 * scale)
            if j == ny - 1:
                duy = (1.5 * u[j, i] - 2.0 * u[j - 1, i] + 0.5 * u[j - 2, i]) / (uu * scale)
            elif j == 0:
                duy = (-1.5 * u[j, i] + 2.0 * u[j + 1, i] - 0.5 * u[j + 2, i]) / (uu * scale)
            else:
                duy = (u[j + 1, i] - u[j - 1, i]) / (uu * 2.0 * scale)
            vals = [ox + i * scale, oy + j * scale, u[j, i] / uu, v[j, i] / uu, rho[j, i] / 3.0, dvx - duy, 0.0, 0.0]
            out.append("".join(fortran_e(x) for x in vals))
    return out


def test_fortran_e_editing():
    assert fortran_e(12.345678) == "  0.12345678E+02"
    assert fortran_e(-0.00012345678) == " -0.12345678E-03"
    assert fortran_e(9.9999999999) == "  0.10000000E+02"
    assert fortran_e(1.5e100) == "  0.15000000+101"


@pytest.mark.parametrize("stride", [(2, 2), (1, 3)])
def test_tecplot_matches_the_reference_layout(tmp_path, stride):
    rng = np.random.default_rng(3)
    ny, nx = 9, 12
    rho = 1.0 + 0.01 * rng.standard_normal((ny, nx))
    u = 0.05 + 0.01 * rng.standard_normal((ny, nx))
    v = 0.01 * rng.standard_normal((ny, nx))
    u[2, 3] = 0.0
    rho[0, 0] = 4.5e100          # a 3-digit exponent: E dropped
    rho[0, 2] = -0.0             # signed zero
    ox, oy, scale, uu = -1.25, -0.5, 0.125, 0.05
    th = np.linspace(0.0, 2 * np.pi, 7)
    xb1, yb1 = 0.3 * np.cos(th), 0.1 * np.sin(th)
    p = tmp_path / "F42.dat"
    io_formats.write_tecplot_fields(str(p), rho, u, v, ox, oy, scale, uu, 42 * uu * scale, stride, xb1, yb1, 1)
    lines = p.read_text().split("\n")
    assert lines[0].startswith('VARIABLES = "X" "Y" "U" "V" "Presure" "Vorticity" "body" "dvordt"')
    onx, ony = (nx - 1) // stride[0] + 1, (ny - 1) // stride[1] + 1
    hd = lines[1].replace(",", " ").split()
    assert hd[:3] == ["ZONE", 'T="Flow', 'feild"'] and int(hd[4]) == onx and int(hd[6]) == ony
    assert hd[7] == "SOLUTIONTIME=" and abs(float(hd[8]) - 42 * uu * scale) < 1e-15
    ref = reference_field_lines(rho, u, v, ox, oy, scale, uu, *stride)
    assert lines[2:2 + onx * ony] == ref
    rest = lines[2 + onx * ony:]
    assert "ZONETYPE=FETRIANGLE" in rest[0] and " 8 " in rest[0].replace(",", " ").replace("=", " ")
    pts = [[float(s[k:k + 14]) for k in range(0, 112, 14)] for s in rest[1:9]]
    assert np.allclose([q[0] for q in pts[:7]], np.round(xb1, 8)) and all(q[2] == 255.0 for q in pts)
    assert np.allclose(pts[7][:2], [0.5 * (xb1[0] + xb1[3]), 0.5 * (yb1[0] + yb1[3])], atol=1e-8)
    tris = rest[9:15]
    assert tris[0] == "  001  002  008" and tris[-1] == "  006  007  008"


def test_airfoil_motion_rows(tmp_path):
    p = tmp_path / "airfoil_motion.dat"
    io_formats.write_airfoil_motion(str(p), [0.0, 0.000625], 2)
    lines = p.read_text().splitlines()
    assert lines[1] == "     0.00062500" + "     0.00000000" * 6


@pytest.mark.parametrize("nx,ny", [(5, 3), (3, 4)])
def test_gforce_file_follows_the_write_statements(tmp_path, nx, ny):
    """g<n>.dat (output_gforce, solution.f90:240-267) against its WRITE
    statements restated: the (a) header, the zone line, then (25e25.17) of
    ox+(i-1)scale, oy+(j-1)scale, gforce(i,j,1:2) for i = 1..Ny outer and
    j = 1..Nx inner as the loop is written; positions outside the (Nx,Ny)
    array (j > Ny when Nx > Ny) hold 0, as does every node without arrays."""
    rng = np.random.default_rng(11)
    gx, gy = rng.standard_normal((ny, nx)), rng.standard_normal((ny, nx)) * 1e-7
    ox, oy, scale = -1.25, -0.5, 0.01
    path = tmp_path / "g7.dat"
    io_formats.write_gforce(path, 7, nx, ny, ox, oy, scale, gx, gy)
    lines = open(path).read().split("\n")
    assert lines[0] == 'VARIABLES = "X" "Y" "gforcex" "gforcey" '
    # list-directed items: integers in 12 columns (the spacing is the
    # compiler's; the values and their order are the reference's)
    assert lines[1] == f' zone,t="{7:12d}",i={nx:12d},j={ny:12d}'
    assert lines[1].replace(" ", "") == f'zone,t="7",i={nx},j={ny}'
    want = []
    fx_all, fy_all = gx.reshape(-1), gy.reshape(-1)   # gforce(i,j) at (i-1) + (j-1) nx
    for i in range(ny):
        for j in range(nx):
            inside = i < nx and j < ny
            fx = fx_all[j * nx + i] if inside else 0.0
            fy = fy_all[j * nx + i] if inside else 0.0
            want.append("".join(fortran_e(v, 25, 17) for v in (ox + i * scale, oy + j * scale, fx, fy)))
    assert lines[2:2 + nx * ny] == want
    assert lines[2 + nx * ny:] == [""]
    zero = tmp_path / "g8.dat"
    io_formats.write_gforce(zero, 8, nx, ny, ox, oy, scale)
    body = open(zero).read().split("\n")[2:2 + nx * ny]
    assert all(ln[50:] == fortran_e(0.0, 25, 17) * 2 for ln in body)
