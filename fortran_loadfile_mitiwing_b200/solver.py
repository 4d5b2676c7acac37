"""Python host side of the B200 time step, mirroring the reference's
subroutine interface (ini_mesh, read_boundary, load_motion_table, init,
evolution, erranalysis, output/saveflowfield) over the C ABI of
include/lbm_b200.h. All compute runs in liblbmb200.so; this module only moves
host arrays across the boundary."""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import dptr


class LbmError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Lbm:
    """One case on the GPU (lbm_create ... lbm_destroy)."""

    def __init__(self, params, lib=None):
        self.lib = lib or _abi.load_library()
        self.params = params
        h = C.c_void_p()
        rc = self.lib.lbm_create(C.byref(params), C.byref(h))
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_last_error(None).decode())
        self.h = h
        self.nx, self.ny = params.nx, params.ny
        self.row_len = self.lib.lbm_force_row_length(self.h)

    # -- error handling --------------------------------------------------
    def _ck(self, rc, ok=(0,)):
        if rc not in ok:
            raise LbmError(rc, self.lib.lbm_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.lbm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up (ini_mesh / read_boundary / load_motion_table / init) ----
    def set_boundary(self, wing, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        self._ck(self.lib.lbm_set_boundary(self.h, wing, dptr(x), dptr(y), len(x)))

    def read_boundary(self, directory=""):
        self._ck(self.lib.lbm_read_boundary(self.h, os.fsencode(directory)))

    def set_motion_table(self, table):
        t = np.asfortranarray(table, dtype=np.float64)
        rows, cols = t.shape
        flat = np.ascontiguousarray(t.reshape(-1, order="F"))
        self._ck(self.lib.lbm_set_motion_table(self.h, dptr(flat), rows, cols))

    def load_motion_table(self, path="motion_params.dat"):
        self._ck(self.lib.lbm_load_motion_table(self.h, os.fsencode(path)))

    def init(self, du=None, dv=None):
        du = None if du is None else np.ascontiguousarray(du, dtype=np.float64)
        dv = None if dv is None else np.ascontiguousarray(dv, dtype=np.float64)
        self._ck(self.lib.lbm_init(self.h, dptr(du), dptr(dv)))

    @classmethod
    def from_case(cls, case, lib=None):
        s = cls(case.params, lib)
        for w, (x, y) in enumerate(case.contours, start=1):
            s.set_boundary(w, x, y)
        s.set_motion_table(case.table)
        s.init(case.du, case.dv)
        return s

    # -- the time step (evolution) ----------------------------------------
    def evolution(self):
        """One step; returns its force.dat row, or None past motion_end_time."""
        row = np.zeros(self.row_len)
        rc = self._ck(self.lib.lbm_step(self.h, dptr(row)), ok=(0, 1))
        return None if rc == 1 else row

    def run(self, nsteps, keep_rows=True):
        rows = np.zeros((max(nsteps, 1), self.row_len)) if keep_rows else None
        done = C.c_int(0)
        self._ck(self.lib.lbm_run(self.h, nsteps, dptr(rows), C.byref(done)), ok=(0, 1))
        return rows[: done.value] if keep_rows else done.value

    # -- observation --------------------------------------------------------
    def fields(self):
        """(rho, u, v) as (ny, nx) arrays (row j, column i)."""
        n = self.nx * self.ny
        rho, u, v = np.zeros(n), np.zeros(n), np.zeros(n)
        self._ck(self.lib.lbm_get_fields(self.h, dptr(rho), dptr(u), dptr(v)))
        return tuple(a.reshape(self.ny, self.nx) for a in (rho, u, v))

    def populations(self):
        """f as (9, ny, nx)."""
        f = np.zeros(9 * self.nx * self.ny)
        self._ck(self.lib.lbm_get_populations(self.h, dptr(f)))
        return f.reshape(9, self.ny, self.nx)

    # -- output and restart files ----------------------------------------
    def write_tecplot(self, path=None, cycle=None, stride=(2, 2), directory="."):
        """F<n>.dat of the state after the last step (lbm_write_tecplot);
        cycle defaults to the reference's n of that step. Returns the path."""
        cycle = self.step_index - 1 if cycle is None else int(cycle)
        path = path or os.path.join(directory, f"F{cycle}.dat")
        self._ck(self.lib.lbm_write_tecplot(self.h, os.fsencode(path), cycle, int(stride[0]), int(stride[1])))
        return path

    def save_checkpoint(self, path="saved_flow_feild.dat"):
        """Writes the state to `path` and its _copy (lbm_save_checkpoint)."""
        self._ck(self.lib.lbm_save_checkpoint(self.h, os.fsencode(path)))

    def load_checkpoint(self, path="saved_flow_feild.dat"):
        """Restores the state from `path`, else its _copy (lbm_load_checkpoint)."""
        self._ck(self.lib.lbm_load_checkpoint(self.h, os.fsencode(path)))

    def save_flow_field(self, path="saved_flow_feild.dat", body_state=None, movenum=0):
        """Writes the reference's own restart file (saveflowfield layout) to
        `path` and its _copy (lbm_save_flow_field)."""
        bs = None if body_state is None else np.ascontiguousarray(body_state, dtype=np.float64).reshape(-1)
        if bs is not None and bs.size != 11 * self.params.wing_count:
            raise ValueError("body_state holds 11 arrays of wing_count values")
        self._ck(self.lib.lbm_save_flow_field(self.h, os.fsencode(path), dptr(bs), int(movenum)))

    def read_flow_field(self, path="saved_flow_feild.dat"):
        """Restarts from the reference's restart file `path`, else its _copy
        (lbm_read_flow_field). Returns (cycle1, body_state (11, wing_count),
        movenum); the next step is cycle1 + 1."""
        cyc, mv = C.c_int(0), C.c_int(0)
        bs = np.zeros(11 * self.params.wing_count)
        self._ck(self.lib.lbm_read_flow_field(self.h, os.fsencode(path), C.byref(cyc), dptr(bs), C.byref(mv)))
        return cyc.value, bs.reshape(11, self.params.wing_count), mv.value

    def set_populations(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        self._ck(self.lib.lbm_set_populations(self.h, dptr(f)))

    def erranalysis(self):
        e = C.c_double()
        self._ck(self.lib.lbm_residual(self.h, C.byref(e)))
        return e.value

    def mass(self):
        """Global mass sum of f over the lattice after the last step (lbm_mass,
        FP64 on the device)."""
        m = C.c_double()
        self._ck(self.lib.lbm_mass(self.h, C.byref(m)))
        return m.value

    def markers(self):
        """(xb2, yb2, solve residual) of the last step."""
        x, y, r, _ = self.solver_info()
        return x, y, r

    def solver_info(self):
        """(xb2, yb2, solve residual, half-bandwidth of the marker system)."""
        n = self.params.wing_count * (self.params.points_per_wing - 1)
        x, y, r, w = np.zeros(n), np.zeros(n), C.c_double(), C.c_int()
        self._ck(self.lib.lbm_get_markers(self.h, dptr(x), dptr(y), C.byref(r), C.byref(w)))
        return x, y, r.value, w.value

    @property
    def step_index(self):
        return self.lib.lbm_step_index(self.h)

    def device_bytes(self):
        """Device memory the case holds now (lbm_device_bytes)."""
        v = C.c_longlong()
        self._ck(self.lib.lbm_device_bytes(self.h, C.byref(v)))
        return v.value


class Batch:
    """Several initialised cases stepped together on one GPU
    (lbm_batch_create ... lbm_batch_destroy): one lattice launch for all of
    them driven by a case table, one launch per immersed-boundary stage. The
    cases stay usable as `Lbm` objects; each one's results are those of
    running it alone."""

    def __init__(self, cases=(), lib=None):
        self.cases = list(cases)
        self.lib = lib or (self.cases[0].lib if self.cases else _abi.load_library())
        arr = (C.c_void_p * max(len(self.cases), 1))(*[c.h.value for c in self.cases])
        b = C.c_void_p()
        rc = self.lib.lbm_batch_create(arr, len(self.cases), C.byref(b))
        if rc != 0:
            msgs = "; ".join(c.lib.lbm_last_error(c.h).decode() for c in self.cases)
            raise LbmError(rc, msgs)
        self.b = b
        self.rows = 0
        self.occupancy = 0

    def __len__(self):
        return len(self.cases)

    def add(self, case):
        """The case joins the batch (at whatever step it is)."""
        rc = self.lib.lbm_batch_add(self.b, case.h)
        if rc != 0:
            raise LbmError(rc, case.lib.lbm_last_error(case.h).decode())
        self.cases.append(case)

    def remove(self, case):
        """The case leaves the batch; the others keep their order."""
        rc = self.lib.lbm_batch_remove(self.b, case.h)
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())
        self.cases.remove(case)

    def close(self):
        if getattr(self, "b", None):
            self.lib.lbm_batch_destroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_rows(self, rows_per_cta):
        rc = self.lib.lbm_batch_set_rows(self.b, int(rows_per_cta))
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())
        self.rows = int(rows_per_cta)

    def set_occupancy(self, ctas_per_sm):
        """At most `ctas_per_sm` lattice CTAs per SM (0: as many as fit)."""
        rc = self.lib.lbm_batch_set_occupancy(self.b, int(ctas_per_sm))
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())
        self.occupancy = int(ctas_per_sm)

    def set_graphs(self, enable):
        """Steady steps as replayed CUDA graphs of 16 steps (True, the
        default) or every launch issued from the host (False); the results
        are the same bit for bit."""
        rc = self.lib.lbm_batch_set_graphs(self.b, 1 if enable else 0)
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())

    def graph_stats(self):
        """(steps run as graph segments, graph launches, graphs
        instantiated) over the batch's life."""
        v = [C.c_longlong() for _ in range(3)]
        rc = self.lib.lbm_batch_graph_stats(self.b, *[C.byref(x) for x in v])
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())
        return tuple(x.value for x in v)

    def run(self, nsteps, keep_rows=True, errors="raise"):
        """Steps every case up to `nsteps` times; returns each case's force
        rows (trimmed to the steps it ran) or the step counts. A failed case
        (a diverged flow, say) stops the run: errors="raise" raises LbmError;
        errors="return" returns (rows or counts, statuses), statuses[c] None
        for a case that is fine, else (code, message)."""
        n = len(self.cases)
        bufs = [np.zeros((max(nsteps, 1), c.row_len)) for c in self.cases] if keep_rows else None
        ptrs = (_abi._D * n)(*[dptr(x) for x in bufs]) if keep_rows else None
        done = (C.c_int * n)()
        rc = self.lib.lbm_batch_run(self.b, int(nsteps), ptrs, done)
        if rc not in (0, 1) and errors == "raise":
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())
        out = [bufs[c][: done[c]] for c in range(n)] if keep_rows else list(done)
        if errors == "raise":
            return out
        status = []
        for c, case in enumerate(self.cases):
            st = self.lib.lbm_batch_case_status(self.b, c)
            status.append(None if st == 0 else (st, case.lib.lbm_last_error(case.h).decode()))
        if rc not in (0, 1) and all(x is None for x in status):
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())   # not a case's own failure
        return out, status

    def device_time(self):
        """(device milliseconds, steps) of the last run (lbm_batch_get_timing)."""
        ms, n = C.c_double(), C.c_int()
        rc = self.lib.lbm_batch_get_timing(self.b, C.byref(ms), C.byref(n))
        if rc != 0:
            raise LbmError(rc, self.lib.lbm_batch_last_error(self.b).decode())
        return ms.value, n.value

    def autotune(self, steps_per_trial=20, candidates=(4, 8, 16), rounds=2, occupancy=(0, 3)):
        """Picks the lattice kernel's tile shape (rows per CTA: `candidates`)
        and occupancy (lattice CTAs per SM: `occupancy`, 0 for as many as
        fit) for this batch by timing `steps_per_trial` real steps with each
        pair on the device (CUDA events around the steps of each trial,
        `rounds` trials per pair in alternating order, the best kept); the
        steps advance the cases and the results do not depend on the choice.
        Returns {(rows, ctas_per_sm): seconds per step} and keeps the
        fastest. The strip width, the ring depth and the registers per
        thread are compile-time choices of the kernel, measured on the
        single case."""
        timing = {}
        order = [(r, o) for r in candidates for o in occupancy]
        for k in range(rounds):
            for r, o in (order if k % 2 == 0 else order[::-1]):
                self.set_rows(r)
                self.set_occupancy(o)
                self.run(steps_per_trial, keep_rows=False)
                ms, n = self.device_time()
                if n > 0:
                    t = ms / 1e3 / n
                    timing[(r, o)] = min(timing.get((r, o), t), t)
        if timing:
            r, o = min(timing, key=timing.get)
            self.set_rows(r)
            self.set_occupancy(o)
        return timing
