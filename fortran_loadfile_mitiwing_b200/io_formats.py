"""Writers and readers of the reference's text formats.

  boundary.dat        (2f14.8) per point          airfoil.f90:229
  motion_params.dat   list-directed rows           mode.f90:88-123
  force.dat           (1000f15.8) per step         solution.f90:376
  airfoil_motion.dat  (1000f15.8) per step         solution.f90:379-390
  F<n>.dat            Tecplot ASCII                solution.f90:129-238 (written by
                      the library: lbm_write_tecplot, Lbm.write_tecplot; from host
                      arrays: write_tecplot_fields)
  g<n>.dat            (25e25.17) per loop position solution.f90:240-267 (write_gforce)
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


def write_gforce(path, cycle, nx, ny, ox, oy, scale, gforce_x=None, gforce_y=None, lib=None):
    """g<n>.dat of output_gforce through lbm_write_gforce: gforce_x, gforce_y
    host arrays (ny, nx) or None for zeros, the live path's value."""
    lib = lib or _abi.load_library()
    a = [None if g is None else np.ascontiguousarray(g, dtype=np.float64).reshape(-1) for g in (gforce_x, gforce_y)]
    for g in a:
        if g is not None and g.size != nx * ny:
            raise ValueError("gforce arrays must hold nx*ny values")
    rc = lib.lbm_write_gforce(os.fsencode(path), int(cycle), int(nx), int(ny), float(ox), float(oy), float(scale),
                              _abi.dptr(a[0]) if a[0] is not None else None,
                              _abi.dptr(a[1]) if a[1] is not None else None)
    if rc != 0:
        raise IOError(f"lbm_write_gforce({path}) = {rc}")


def edge_count(nx, ny):
    """Nodes of the edge f0 array: left column, right column, bottom row, top row."""
    return 2 * ny + 2 * nx


def write_flow_field_file(path, cycle, u, v, f, edge_f0, body_state=None, movenum=0, lib=None):
    """One restart file in the reference's saveflowfield layout from host
    arrays (lbm_write_flow_field_file): u, v (ny, nx), f (9, ny, nx),
    edge_f0 (2 ny + 2 nx, 9), body_state (11, wing_count) or None."""
    lib = lib or _abi.load_library()
    ny, nx = np.shape(u)
    a = [np.ascontiguousarray(x, dtype=np.float64).reshape(-1) for x in (u, v, f, edge_f0)]
    if a[2].size != 9 * nx * ny or a[3].size != 9 * edge_count(nx, ny):
        raise ValueError("f must hold 9 nx ny values and edge_f0 9 (2 nx + 2 ny)")
    bs = None if body_state is None else np.ascontiguousarray(body_state, dtype=np.float64).reshape(-1)
    wing_count = 0 if bs is None else bs.size // 11
    rc = lib.lbm_write_flow_field_file(os.fsencode(path), nx, ny, int(cycle), wing_count, _abi.dptr(bs),
                                       int(movenum), *(_abi.dptr(x) for x in a))
    if rc != 0:
        raise IOError(f"lbm_write_flow_field_file({path}) = {rc}")


def read_flow_field_file(path, nx, ny, wing_count, lib=None):
    """Reads one restart file of the reference's layout
    (lbm_read_flow_field_file): dict of cycle, body_state (11, wing_count),
    movenum, u, v (ny, nx), f (9, ny, nx), edge_f0 (2 ny + 2 nx, 9)."""
    lib = lib or _abi.load_library()
    cyc, mv = C.c_int(0), C.c_int(0)
    bs = np.zeros(11 * wing_count)
    u, v = np.zeros(nx * ny), np.zeros(nx * ny)
    f, ef = np.zeros(9 * nx * ny), np.zeros(9 * edge_count(nx, ny))
    rc = lib.lbm_read_flow_field_file(os.fsencode(path), nx, ny, wing_count, C.byref(cyc), _abi.dptr(bs),
                                      C.byref(mv), _abi.dptr(u), _abi.dptr(v), _abi.dptr(f), _abi.dptr(ef))
    if rc != 0:
        raise IOError(f"lbm_read_flow_field_file({path}) = {_abi.STATUS_NAMES.get(rc, rc)}")
    return dict(cycle=cyc.value, body_state=bs.reshape(11, wing_count), movenum=mv.value,
                u=u.reshape(ny, nx), v=v.reshape(ny, nx), f=f.reshape(9, ny, nx),
                edge_f0=ef.reshape(edge_count(nx, ny), 9))
