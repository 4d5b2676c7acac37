"""Serving loop: flapping-wing solves that arrive over time, stepped in one
continuously changing batch on one GPU.

A request is a case (grid, kinematics, Reynolds number, number of steps). The
server keeps each admitted case's populations and marker state on the device
for its whole solve. Between ticks it admits waiting requests in arrival order
while the HBM budget holds them: a case is charged its estimated device bytes
until it exists and its measured bytes (lbm_device_bytes) after. Cases are
prepared (lbm_create, boundary, motion table, lbm_init) on a worker thread
while the batch steps, and join the batch at the next tick. A tick runs
`tick_steps` steps of every case in the batch (lbm_batch_run); a case whose
motion table ends stops inside the tick, leaves the batch, and its force rows
are returned and its memory released. Each case's result is bit-for-bit the
result of solving it alone: the batch only packs the cases' launches together.

`serve_stream()` drives the server with Poisson arrivals in real time and
reports the time from arrival to result (p50, p99) and cases per hour; the
FP32 one-at-a-time baseline is the same arrivals served first come, first
served by solving each case alone, with service times measured per case. Run
as `python -m fortran_loadfile_mitiwing_b200.serve [--rates 2 8 32]`; prints
one JSON object. Needs a GPU.
"""
import argparse
import collections
import concurrent.futures
import json
import math
import sys
import time

import numpy as np

from .solver import Batch, Lbm

# sizes of the device structures a case holds (csrc/lbm_common.cuh, lbm_internal.h, ib_kernels.cu)
_MARKER_BYTES = 152        # struct Marker
_PATCHINFO_BYTES = 16      # struct PatchInfo
_NSLOT_MAX = 16            # LBM_NSLOT_MAX
_FPAD = 64                 # LBM_FPAD elements before and after the population planes
_RING = 2048               # force rows kept on the device
_MAXW = 8                  # LBM_MAXW
_NPART = 3 * _MAXW + 3     # per-tile partials of the correction
_TILE_INTS = 257           # per-tile list: count + 256 markers
_BS, _GW = 16, 48          # block size and factor row width of the marker solve
_FBATCH = 4                # steps per factorization batch (LBM_IB_BATCH)
_MASS_BLOCKS = 296         # CTAs of the mass check (kf_kernel.cu)


def _elem_bytes(precision):
    return {0: 4, 1: 8, 2: 2, 3: 2}[precision]


def patch_extent(case):
    """Largest per-step marker patch (width, height) in lattice units: the
    union over wings of the discs of radius R/scale + 4 about each pivot,
    maximised over the steps of the motion table."""
    p = case.params
    if not case.contours:
        return 0, 0
    dt = p.scale * p.uu
    t = case.table[:, 0]
    n = int((t[-1] + 1e-12) / dt) + 1
    times = np.arange(n) * dt
    xlo = np.full(n, np.inf)
    xhi = np.full(n, -np.inf)
    ylo = np.full(n, np.inf)
    yhi = np.full(n, -np.inf)
    for w, (x, y) in enumerate(case.contours):
        r = float(np.max(np.hypot(x, y))) / p.scale + 4.0
        cx = (np.interp(times, t, case.table[:, 1 + 9 * w + 3]) + p.xc - p.ox) / p.scale
        cy = (np.interp(times, t, case.table[:, 1 + 9 * w + 6]) + p.yc - p.oy) / p.scale
        xlo = np.minimum(xlo, cx - r)
        xhi = np.maximum(xhi, cx + r)
        ylo = np.minimum(ylo, cy - r)
        yhi = np.maximum(yhi, cy + r)
    return (min(int(np.max(np.ceil(xhi - xlo))) + 2, p.nx), min(int(np.max(np.ceil(yhi - ylo))) + 2, p.ny))


def estimate_device_bytes(case):
    """Device bytes a case holds while it is stepped: lattice buffers, fields
    and edge values (lbm_create), step table and contour, and the
    immersed-boundary scratch of 2 x 4 step slots (first step)."""
    p = case.params
    nx, ny = p.nx, p.ny
    elem = _elem_bytes(p.precision)
    cs = 8 if p.precision == 1 else 4
    pitch = (nx + 63) // 64 * 64
    nwing = len(case.contours)
    npts = nwing * p.points_per_wing
    ns = max(1, nwing * (p.points_per_wing - 1)) if nwing else 1
    row_len = 1 + 3 * nwing + 3 + 9 * nwing
    total = 2 * elem * (9 * pitch * ny + 2 * _FPAD)          # populations, two buffers
    total += 2 * 3 * cs * nx * ny                              # fields, two slots
    total += cs * (6 * ny + 36)                                # edge values
    total += 4 + 4 + _NSLOT_MAX * _PATCHINFO_BYTES + 8 * 2 * 296 + 2 * 16 + 8 * row_len * _RING
    total += 8 * (_MASS_BLOCKS + 1) + 4                        # mass check: partials and sum, counter
    if nwing:
        dt = p.scale * p.uu
        msteps = int((case.table[-1, 0] + 1e-12) / dt) + 1
        total += 8 * msteps * case.table.shape[1]              # step table
        total += 2 * 8 * npts + 8 * ns                         # contour and arc lengths
        S, K = 2 * _FBATCH, _FBATCH
        nb = (ns + _BS - 1) // _BS
        pw, ph = patch_extent(case)
        nblk = max(1, (pw + 15) // 16) * max(1, (ph + 15) // 16)
        # right-hand sides, solution and tile partials: one set per step parity
        total += S * _MARKER_BYTES * ns + 2 * 2 * 8 * 2 * ns + S * 8 * ns * ns
        total += 2 * K * 8 * nb * _BS * _BS + S * 8 * nb * _BS * _GW + S * 2 * 4 + S * 4
        total += 2 * 8 * max(_NPART * nblk, 2 * ((ns + 7) // 8))
        total += S * 4 * _TILE_INTS * nblk + S * 4 + S * 4 * nblk
        total += S * 4 * ns + S * 8 * ns + 8 + K * 4
    return int(total)


class Request:
    """A solve: `make()` returns the case (cases.Case), built when the case
    is prepared; `estimate` its device bytes (from `make()` if None);
    `arrival` in the server clock's seconds."""

    def __init__(self, rid, make, arrival=0.0, estimate=None):
        self.rid = rid
        self.make = make
        self.arrival = arrival
        self.estimate = estimate


class Result:
    """A finished solve: its force rows (one per step, as lbm_run gives them)
    and its times on the server clock; `error` (code, message) when the case
    failed (its rows then stop at the failing check)."""

    def __init__(self, rid, rows, arrival, admitted, started, finished, handle=None, error=None):
        self.rid = rid
        self.error = error
        self.rows = rows
        self.arrival = arrival
        self.admitted = admitted
        self.started = started
        self.finished = finished
        self.handle = handle
        self.steps = rows.shape[0]

    @property
    def latency(self):
        return self.finished - self.arrival


class Admission:
    """First-come first-served admission against a byte budget and a case
    limit: the head of the queue waits until it fits (a later, smaller
    request does not pass it, so no request starves)."""

    def __init__(self, budget_bytes, max_cases=256):
        self.budget = int(budget_bytes)
        self.max_cases = max_cases
        self.charged = {}
        self.queue = collections.deque()

    @property
    def used(self):
        return sum(self.charged.values())

    def submit(self, rid, nbytes):
        if nbytes > self.budget:
            raise ValueError(f"request {rid}: {nbytes} bytes exceed the budget of {self.budget}")
        self.queue.append((rid, int(nbytes)))

    def admit(self):
        """Requests admitted now, in arrival order."""
        out = []
        while self.queue and len(self.charged) < self.max_cases:
            rid, nbytes = self.queue[0]
            if self.used + nbytes > self.budget:
                break
            self.queue.popleft()
            self.charged[rid] = nbytes
            out.append(rid)
        return out

    def recharge(self, rid, nbytes):
        self.charged[rid] = int(nbytes)

    def withdraw(self, rid):
        """Takes a waiting request out of the queue; True if it was there."""
        for k, (r, _) in enumerate(self.queue):
            if r == rid:
                del self.queue[k]
                return True
        return False

    def release(self, rid):
        self.charged.pop(rid, None)


class _Done:
    """A finished future (the server without a worker thread)."""

    def __init__(self, value):
        self.value = value

    def done(self):
        return True

    def result(self):
        return self.value


class Server:
    """Continuous batching of solves on one GPU (see the module docstring).

    budget_bytes: device memory the cases may hold together; tick_steps: steps
    between admissions; keep_handles: results carry the finished case's handle
    (open; the caller closes it) instead of closing it; workers: threads that
    prepare admitted cases (0: prepared in `tick`; 2 measured best: the
    preparation of cases arriving together keeps pace with the batch)."""

    def __init__(self, budget_bytes, tick_steps=100, lib=None, max_cases=256, keep_handles=False,
                 clock=time.perf_counter, workers=2):
        self.adm = Admission(budget_bytes, max_cases)
        self.tick_steps = tick_steps
        self.lib = lib
        self.keep_handles = keep_handles
        self.clock = clock
        self.batch = None
        self.requests = {}
        self.live = {}          # rid -> [case handle, row chunks, admitted, started, last step]
        self.preparing = {}     # rid -> (future, admitted)
        self.pool = concurrent.futures.ThreadPoolExecutor(max_workers=workers) if workers else None
        self.done = []
        self.peak_used = 0
        self.peak_cases = 0
        self.ticks = 0

    def close(self):
        if self.pool:
            self.pool.shutdown(wait=True)
            self.pool = None
        for fut, _ in self.preparing.values():
            fut.result()[0].close()
        self.preparing.clear()
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        for st in self.live.values():
            st[0].close()
        self.live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, req):
        if req.estimate is None:
            req.estimate = estimate_device_bytes(req.make())
        self.requests[req.rid] = req
        self.adm.submit(req.rid, req.estimate)

    def _prepare(self, req):
        case = req.make()
        h = Lbm.from_case(case, self.lib)
        dt = case.params.scale * case.params.uu
        return h, int(math.floor((case.table[-1, 0] + 1e-12) / dt)) + 1   # last step the motion covers

    def idle(self):
        return not self.live and not self.preparing and not self.adm.queue

    def cancel(self, rid):
        """Cancels a request wherever it is: waiting (it leaves the queue),
        being prepared (its case is closed when ready) or running (it leaves
        the batch between ticks). Its memory is released and a Result with
        error (LBM_ERR_STATE, "cancelled") and the rows computed so far is
        returned, or None for an unknown or finished request."""
        req = self.requests.get(rid)
        if req is None:
            return None
        t = self.clock()
        if self.adm.withdraw(rid):
            self.requests.pop(rid)
            res = Result(rid, np.zeros((0, 0)), req.arrival, None, None, t, None, (-2, "cancelled"))
        elif rid in self.preparing:
            fut, admitted = self.preparing.pop(rid)
            fut.result()[0].close()
            self.adm.release(rid)
            self.requests.pop(rid)
            res = Result(rid, np.zeros((0, 0)), req.arrival, admitted, None, t, None, (-2, "cancelled"))
        elif rid in self.live:
            h, chunks, admitted, started, _ = self.live.pop(rid)
            self.batch.remove(h)
            self.adm.release(rid)
            self.requests.pop(rid)
            rows_all = np.concatenate(chunks) if chunks else np.zeros((0, h.row_len))
            h.close()
            res = Result(rid, rows_all, req.arrival, admitted, started, t, None, (-2, "cancelled"))
        else:
            return None
        self.done.append(res)
        return res

    def tick(self, wait_for_ready=False):
        """Admits what fits, joins the prepared cases, steps the batch once;
        returns the results that finished. wait_for_ready: with nothing in
        the batch, wait for a case being prepared instead of returning."""
        now = self.clock()
        for rid in self.adm.admit():
            req = self.requests[rid]
            fut = self.pool.submit(self._prepare, req) if self.pool else _Done(self._prepare(req))
            self.preparing[rid] = (fut, now)
        if wait_for_ready and not self.live and self.preparing:
            concurrent.futures.wait([f for f, _ in self.preparing.values() if isinstance(f, concurrent.futures.Future)],
                                    return_when=concurrent.futures.FIRST_COMPLETED)
        for rid in [r for r, (f, _) in self.preparing.items() if f.done()]:
            fut, admitted = self.preparing.pop(rid)
            h, last = fut.result()
            if self.batch is None:
                self.batch = Batch([], lib=h.lib)
            self.batch.add(h)
            self.adm.recharge(rid, h.device_bytes())
            self.live[rid] = [h, [], admitted, self.clock(), last]
        self.peak_used = max(self.peak_used, self.adm.used)
        self.peak_cases = max(self.peak_cases, len(self.live))
        if not self.live:
            return []
        rows, status = self.batch.run(self.tick_steps, errors="return")
        self.ticks += 1
        t = self.clock()
        by_handle = {id(st[0]): rid for rid, st in self.live.items()}
        finished = {}
        for h, r, err in zip(list(self.batch.cases), rows, status):
            rid = by_handle[id(h)]
            st = self.live[rid]
            if r.shape[0]:
                st[1].append(r)
            if err is not None or h.step_index > st[4]:   # failed, or the case's motion table ended
                finished[rid] = err
        out = []
        for rid, err in finished.items():
            h, chunks, admitted, started, _ = self.live.pop(rid)
            self.batch.remove(h)
            self.adm.release(rid)
            rows_all = np.concatenate(chunks) if chunks else np.zeros((0, h.row_len))
            req = self.requests.pop(rid)
            out.append(Result(rid, rows_all, req.arrival, admitted, started, t, h if self.keep_handles else None, err))
            if not self.keep_handles:
                h.close()
        self.done.extend(out)
        return out


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else float("nan")


def poisson_arrivals(rate, n, seed=0):
    """Arrival times (s) of a Poisson stream of `rate` requests/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def serve_stream(specs, rate, periods=3.0, budget_bytes=150e9, precision="fp16", tick_steps=100, seed=1, lib=None,
                 keep_rows=(), workers=2):
    """Serves `specs` (sweep.sweep_specs items, `periods` flapping periods
    each) arriving as a Poisson stream of `rate` requests/s in real time;
    returns the results (force rows kept for the request ids in keep_rows,
    else only the first and last row) and a summary."""
    from . import sweep
    arrivals = poisson_arrivals(rate, len(specs), seed)
    reqs = []
    for i, sp in enumerate(specs):
        n = int(math.ceil(periods * sp["period_steps"]))
        est = estimate_device_bytes(sweep.case_of(sp, n, precision, amp=0.0))
        reqs.append(Request(i, lambda sp=sp, n=n: sweep.case_of(sp, n, precision), float(arrivals[i]), est))
    srv = Server(budget_bytes, tick_steps=tick_steps, lib=lib, workers=workers)
    try:
        t0 = srv.clock()
        for r in reqs:
            r.arrival += t0
        nxt = 0
        while nxt < len(reqs) or not srv.idle():
            now = srv.clock()
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                srv.submit(reqs[nxt])
                nxt += 1
            if srv.idle():
                time.sleep(max(0.0, reqs[nxt].arrival - srv.clock()))
                continue
            for r in srv.tick(wait_for_ready=True):
                if r.rid not in keep_rows and r.rows.shape[0] > 2:
                    r.rows = r.rows[[0, -1]]
        res = sorted(srv.done, key=lambda r: r.rid)
    finally:
        srv.close()
    lat = [r.latency for r in res]
    span = max(r.finished for r in res) - t0
    lups = sum(sp["nx"] * sp["ny"] * int(math.ceil(periods * sp["period_steps"])) for sp in specs)
    return res, {"rate_per_s": rate, "requests": len(res), "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
                 "mean_s": float(np.mean(lat)), "makespan_s": span, "cases_per_hour": len(res) * 3600.0 / span,
                 "mlups": lups / span / 1e6, "peak_cases": srv.peak_cases, "peak_bytes": srv.peak_used,
                 "ticks": srv.ticks}


COL_CD, COL_CL = 1, 2   # force-row columns of a one-wing case: time, C_x (drag), C_y (lift), ...


def period_errors(rows, ref, period_steps, periods):
    """Per flapping period, |mean(rows) - mean(ref)| of C_D relative to
    |mean(ref)| of C_D, and of C_L relative to the RMS of `ref`'s C_L over
    that period (C_L of a symmetric section in symmetric motion has a mean
    near zero). Returns the largest of each."""
    out = {"cd": 0.0, "cl": 0.0}
    for k in range(int(periods)):
        a, b = int(round(k * period_steps)), int(round((k + 1) * period_steps))
        for name, col in (("cd", COL_CD), ("cl", COL_CL)):
            r = ref[a:b, col]
            scale = abs(float(np.mean(r))) if name == "cd" else math.sqrt(float(np.mean(r ** 2)))
            out[name] = max(out[name], abs(float(np.mean(rows[a:b, col]) - np.mean(r))) / scale)
    return out


def fp64_reference_rows(specs, periods=3.0, lib=None):
    """Force rows of `specs` stored in FP64, run together as one batch to the
    end of their motion."""
    from . import sweep
    hs = [Lbm.from_case(sweep.case_of(sp, int(math.ceil(periods * sp["period_steps"])), "fp64"), lib)
          for sp in specs]
    try:
        with Batch(hs) as b:
            return b.run(max(int(math.ceil(periods * sp["period_steps"])) for sp in specs) + 2)
    finally:
        for h in hs:
            h.close()


def fifo_one_at_a_time(arrivals, service):
    """Finish times of a single first-come first-served server."""
    t, out = -math.inf, []
    for a, s in zip(arrivals, service):
        t = max(t, a) + s
        out.append(t)
    return out


def alone_service_times(specs, periods=3.0, precision="fp32", sample_steps=300, warmup=20, lib=None):
    """Seconds to solve each case alone (lbm_run): preparation (create,
    boundary, motion, init) measured in full, and the steps timed over a
    sample of `sample_steps` after `warmup` and scaled to the case's steps."""
    from . import sweep
    out = []
    for sp in specs:
        n = int(math.ceil(periods * sp["period_steps"]))
        case = sweep.case_of(sp, n, precision)
        t0 = time.perf_counter()
        s = Lbm.from_case(case, lib)
        prep = time.perf_counter() - t0
        s.run(warmup, keep_rows=False)
        t0 = time.perf_counter()
        s.run(sample_steps, keep_rows=False)
        per_step = (time.perf_counter() - t0) / sample_steps
        s.close()
        out.append(prep + per_step * n)
    return out


def main():
    from . import sweep
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--rates", type=float, nargs="+", default=[2.0, 8.0, 32.0])
    ap.add_argument("--requests", type=int, default=64)
    ap.add_argument("--periods", type=float, default=3.0)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--tick-steps", type=int, default=100)
    ap.add_argument("--precision", default="fp16")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--workers", type=int, default=2, help="threads preparing admitted cases")
    ap.add_argument("--check", type=int, default=8,
                    help="requests of the first stream whose coefficients are checked against FP64 storage")
    args = ap.parse_args()
    specs = sweep.sweep_specs(args.requests, args.seed)
    out = {"requests": args.requests, "periods": args.periods, "budget_gb": args.budget_gb,
           "precision": args.precision, "tick_steps": args.tick_steps, "workers": args.workers,
           "case_distribution": "sweep_specs(seed): Nx in [512, 2048], Ny = Nx/2, chord = Ny/4",
           "served": [], "fp32_one_at_a_time": []}
    service = alone_service_times(specs, args.periods)
    out["fp32_alone_service_s_total"] = float(sum(service))
    for k, rate in enumerate(args.rates):
        keep = set(range(args.check)) if k == 0 else set()
        res, summ = serve_stream(specs, rate, args.periods, args.budget_gb * 1e9, args.precision, args.tick_steps,
                                 seed=args.seed + k, keep_rows=keep, workers=args.workers)
        if keep:
            ref = fp64_reference_rows(specs[:args.check], args.periods)
            errs = [period_errors(res[i].rows, ref[i], specs[i]["period_steps"], args.periods) for i in sorted(keep)]
            out["coefficients_vs_fp64"] = {
                "requests": len(keep), "periods": int(args.periods),
                "max_period_mean_err_cd": max(e["cd"] for e in errs),
                "max_period_mean_err_cl": max(e["cl"] for e in errs),
                "note": "per period |mean - mean_fp64| / |mean_fp64| for C_D, / rms_fp64 for C_L; served rows vs "
                        "the same cases in FP64 storage"}
        arr = poisson_arrivals(rate, len(specs), args.seed + k)
        fin = fifo_one_at_a_time(arr, service)
        lat = [f - a for f, a in zip(fin, arr)]
        base = {"rate_per_s": rate, "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
                "makespan_s": float(max(fin)), "cases_per_hour": len(specs) * 3600.0 / float(max(fin))}
        summ["vs_fp32_one_at_a_time"] = summ["cases_per_hour"] / base["cases_per_hour"]
        out["served"].append(summ)
        out["fp32_one_at_a_time"].append(base)
        print(json.dumps(summ), flush=True, file=sys.stderr)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
