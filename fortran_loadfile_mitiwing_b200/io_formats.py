"""Writers and readers of the reference's text formats.

  boundary.dat        (2f14.8) per point          airfoil.f90:229
  motion_params.dat   list-directed rows           mode.f90:88-123
  force.dat           (1000f15.8) per step         solution.f90:376
  airfoil_motion.dat  (1000f15.8) per step         solution.f90:379-390
  F<n>.dat            Tecplot ASCII                solution.f90:129-238 (written by
                      the library: lbm_write_tecplot, Lbm.write_tecplot; from host
                      arrays: write_tecplot_fields)
"""
import ctypes as C
import os

import numpy as np

from . import _abi


def fortran_f(x, w, d):
    """Fortran Fw.d edit descriptor: right-justified, '*' fill on overflow."""
    s = f"{x:{w}.{d}f}"
    return "*" * w if len(s) > w else s


def write_boundary(path, x, y):
    with open(path, "w") as fh:
        for a, b in zip(x, y):
            fh.write(fortran_f(a, 14, 8) + fortran_f(b, 14, 8) + "\n")


def write_motion(path, table):
    with open(path, "w") as fh:
        for row in np.asarray(table):
            fh.write(" ".join(f"{v:.17g}" for v in row) + "\n")


def format_force_row(row):
    """One force.dat record, format (1000f15.8)."""
    return "".join(fortran_f(v, 15, 8) for v in row)


def write_force_rows(path, rows, append=False):
    with open(path, "a" if append else "w") as fh:
        for r in rows:
            fh.write(format_force_row(r) + "\n")


def parse_boundary(path, npts, lib=None):
    """Reads one boundary file with the library's own (2f14.8) parser."""
    lib = lib or _abi.load_library()
    x, y = np.zeros(npts), np.zeros(npts)
    rc = lib.lbm_parse_boundary_file(os.fsencode(path), npts, _abi.dptr(x), _abi.dptr(y))
    if rc != 0:
        raise IOError(f"lbm_parse_boundary_file({path}) = {rc}")
    return x, y


def parse_motion(path, cols, lib=None):
    """Reads a motion_params.dat with the library's own parser; (rows, cols)."""
    lib = lib or _abi.load_library()
    n = C.c_int(0)
    rc = lib.lbm_parse_motion_file(os.fsencode(path), cols, None, 0, C.byref(n))
    if rc != 0:
        raise IOError(f"lbm_parse_motion_file({path}) = {rc}")
    flat = np.zeros(n.value * cols)
    rc = lib.lbm_parse_motion_file(os.fsencode(path), cols, _abi.dptr(flat), n.value, C.byref(n))
    if rc != 0:
        raise IOError(f"lbm_parse_motion_file({path}) = {rc}")
    return flat.reshape(cols, n.value).T.copy()


def airfoil_motion_row(time, wing_count):
    """One airfoil_motion.dat record (solution.f90:379-390): time, then per
    wing 0, body_extra_v/UU and body_extra_s*scale, which are 0 for the
    prescribed motion this library solves (no body dynamics)."""
    return np.concatenate([[time], np.zeros(3 * wing_count)])


def write_airfoil_motion(path, times, wing_count, append=False):
    """airfoil_motion.dat rows for the steps at `times`, format (1000f15.8)."""
    with open(path, "a" if append else "w") as fh:
        for t in times:
            fh.write(format_force_row(airfoil_motion_row(t, wing_count)) + "\n")


def write_tecplot_fields(path, rho, u, v, ox, oy, scale, uu, solution_time, stride=(2, 2), xb1=None, yb1=None,
                         wing_count=0, lib=None):
    """F<n>.dat from host fields (ny, nx) through lbm_write_tecplot_fields."""
    lib = lib or _abi.load_library()
    ny, nx = np.shape(rho)
    a = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (rho, u, v)]
    ppw = 0
    if wing_count:
        xb1 = np.ascontiguousarray(xb1, dtype=np.float64)
        yb1 = np.ascontiguousarray(yb1, dtype=np.float64)
        ppw = xb1.size // wing_count
    rc = lib.lbm_write_tecplot_fields(os.fsencode(path), nx, ny, ox, oy, scale, uu, solution_time, int(stride[0]),
                                      int(stride[1]), _abi.dptr(a[0]), _abi.dptr(a[1]), _abi.dptr(a[2]), wing_count,
                                      ppw, _abi.dptr(xb1) if wing_count else None,
                                      _abi.dptr(yb1) if wing_count else None)
    if rc != 0:
        raise IOError(f"lbm_write_tecplot_fields({path}) = {rc}")
