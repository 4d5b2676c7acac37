"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (liblbmoracle.so).

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
checker; the product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblbmoracle.so")

_D = C.POINTER(C.c_double)
_lib = None


def _dptr(a):
    return None if a is None else a.ctypes.data_as(_D)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    from fortran_loadfile_mitiwing_b200._abi import LbmParams
    lib = C.CDLL(LIB)
    P = C.c_void_p
    sig = {
        "ora_create": (P, [C.POINTER(LbmParams)]),
        "ora_destroy": (None, [P]),
        "ora_set_boundary": (C.c_int, [P, C.c_int, _D, _D, C.c_int]),
        "ora_set_motion_table": (C.c_int, [P, _D, C.c_int, C.c_int]),
        "ora_init": (C.c_int, [P, _D, _D]),
        "ora_step": (C.c_int, [P, _D]),
        "ora_force_row_length": (C.c_int, [P]),
        "ora_erranalysis": (C.c_int, [P, _D]),
        "ora_get_fields": (None, [P, _D, _D, _D]),
        "ora_get_f": (None, [P, _D]),
        "ora_set_f": (None, [P, _D]),
        "ora_get_f0": (None, [P, _D]),
        "ora_get_gforce": (None, [P, _D, _D]),
        "ora_get_markers": (C.c_int, [P, _D, _D, _D]),
        "ora_support_count": (C.c_int, [P]),
        "ora_step_index": (C.c_int, [P]),
        "ora_last_error": (C.c_char_p, [P]),
        "ora_mrt_matrices": (None, [_D, _D]),
        "ora_lattice": (None, [C.POINTER(C.c_int), _D]),
        "ora_delta": (C.c_double, [C.c_double, C.c_int]),
        "ora_collide_node": (None, [P, _D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _D]),
        "ora_motion_row": (C.c_int, [P, C.c_int, _D]),
        "ora_motion_lookup": (C.c_int, [_D, C.c_int, C.c_int, C.c_double, _D]),
        "ora_set_threads": (None, [C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def collide_node(oracle, f, rho, u, v, gfx=0.0, gfy=0.0):
    """One node of the collision (solution.f90:592-635) with the oracle's
    rates: post-collision f from f (9), rho, u, v and the force density."""
    import numpy as np
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros(9)
    oracle.lib.ora_collide_node(oracle.h, _dptr(f), rho, u, v, gfx, gfy, _dptr(out))
    return out


class OracleError(RuntimeError):
    pass


class Oracle:
    """FP64 CPU restatement of the reference step with the same calls as
    fortran_loadfile_mitiwing_b200.Lbm."""

    def __init__(self, params):
        self.lib = load()
        self.params = params
        self.h = self.lib.ora_create(C.byref(params))
        if not self.h:
            raise OracleError("ora_create rejected the parameters")
        self.nx, self.ny = params.nx, params.ny
        self.row_len = self.lib.ora_force_row_length(self.h)

    def _ck(self, rc, ok=(0,)):
        if rc not in ok:
            raise OracleError(f"{rc}: {self.lib.ora_last_error(self.h).decode()}")
        return rc

    def close(self):
        if self.h:
            self.lib.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_boundary(self, wing, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._ck(self.lib.ora_set_boundary(self.h, wing, _dptr(x), _dptr(y), len(x)))

    def set_motion_table(self, table):
        t = np.asfortranarray(table, dtype=np.float64)
        flat = np.ascontiguousarray(t.reshape(-1, order="F"))
        self._ck(self.lib.ora_set_motion_table(self.h, _dptr(flat), t.shape[0], t.shape[1]))

    def init(self, du=None, dv=None):
        du = None if du is None else np.ascontiguousarray(du, dtype=np.float64)
        dv = None if dv is None else np.ascontiguousarray(dv, dtype=np.float64)
        self._ck(self.lib.ora_init(self.h, _dptr(du), _dptr(dv)))

    @classmethod
    def from_case(cls, case):
        o = cls(case.params)
        for w, (x, y) in enumerate(case.contours, start=1):
            o.set_boundary(w, x, y)
        o.set_motion_table(case.table)
        o.init(case.du, case.dv)
        return o

    def evolution(self):
        row = np.zeros(self.row_len)
        rc = self._ck(self.lib.ora_step(self.h, _dptr(row)), ok=(0, 1))
        return None if rc == 1 else row

    def run(self, nsteps):
        rows = []
        for _ in range(nsteps):
            r = self.evolution()
            if r is None:
                break
            rows.append(r)
        return np.array(rows).reshape(len(rows), self.row_len)

    def fields(self):
        n = self.nx * self.ny
        rho, u, v = np.zeros(n), np.zeros(n), np.zeros(n)
        self.lib.ora_get_fields(self.h, _dptr(rho), _dptr(u), _dptr(v))
        return tuple(a.reshape(self.ny, self.nx) for a in (rho, u, v))

    def populations(self):
        f = np.zeros(9 * self.nx * self.ny)
        self.lib.ora_get_f(self.h, _dptr(f))
        return f.reshape(9, self.ny, self.nx)

    def set_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        self.lib.ora_set_f(self.h, _dptr(f))

    def streamed(self):
        f0 = np.zeros(9 * self.nx * self.ny)
        self.lib.ora_get_f0(self.h, _dptr(f0))
        return f0.reshape(9, self.ny, self.nx)

    def gforce(self):
        n = self.nx * self.ny
        gx, gy = np.zeros(n), np.zeros(n)
        self.lib.ora_get_gforce(self.h, _dptr(gx), _dptr(gy))
        return gx.reshape(self.ny, self.nx), gy.reshape(self.ny, self.nx)

    def erranalysis(self):
        e = C.c_double()
        self._ck(self.lib.ora_erranalysis(self.h, C.byref(e)))
        return e.value

    def markers(self):
        n = self.params.wing_count * (self.params.points_per_wing - 1)
        x, y, r = np.zeros(n), np.zeros(n), C.c_double()
        self.lib.ora_get_markers(self.h, _dptr(x), _dptr(y), C.byref(r))
        return x, y, r.value

    def support_count(self):
        return self.lib.ora_support_count(self.h)


def mrt_matrices():
    lib = load()
    m, mi = np.zeros(81), np.zeros(81)
    lib.ora_mrt_matrices(_dptr(m), _dptr(mi))
    return m.reshape(9, 9), mi.reshape(9, 9)


def lattice():
    lib = load()
    e = (C.c_int * 18)()
    w = np.zeros(9)
    lib.ora_lattice(e, _dptr(w))
    return np.array(list(e)).reshape(9, 2), w


def delta(r, smooth):
    return load().ora_delta(float(r), int(smooth))


def motion_lookup(table, t):
    lib = load()
    tf = np.asfortranarray(table, dtype=np.float64)
    flat = np.ascontiguousarray(tf.reshape(-1, order="F"))
    row = np.zeros(tf.shape[1])
    lib.ora_motion_lookup(_dptr(flat), tf.shape[0], tf.shape[1], float(t), _dptr(row))
    return row


def set_threads(n):
    load().ora_set_threads(int(n))
