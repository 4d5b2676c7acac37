"""Host logic of the serving loop: first-come first-served admission against
a byte budget, the one-at-a-time queue model, arrivals, the device-memory
estimate's arithmetic (its agreement with what a case holds is a GPU test),
and the server's join/finish bookkeeping over a stand-in for the device, and
the batch autotuner's choice over a stand-in for the library."""
import math

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import cases, sweep
from fortran_loadfile_mitiwing_b200.serve import (Admission, estimate_device_bytes, fifo_one_at_a_time,
                                                  patch_extent, poisson_arrivals)


def test_admission_is_fifo_within_budget():
    a = Admission(100)
    for rid, nb in enumerate([40, 50, 30, 5]):
        a.submit(rid, nb)
    assert a.admit() == [0, 1]          # 40 + 50; 30 does not fit, and 5 does not pass it
    assert a.used == 90
    a.recharge(1, 20)                   # measured below the estimate
    assert a.admit() == [2, 3]
    a.release(0)
    a.release(2)
    assert a.used == 25 and not a.queue
    with pytest.raises(ValueError):
        a.submit(9, 101)


def test_admission_case_limit():
    a = Admission(10 ** 9, max_cases=2)
    for rid in range(4):
        a.submit(rid, 1)
    assert a.admit() == [0, 1]
    assert a.admit() == []
    a.release(1)
    assert a.admit() == [2]


def test_fifo_queue_model():
    assert fifo_one_at_a_time([0.0, 0.5, 5.0], [2.0, 1.0, 1.0]) == [2.0, 3.0, 6.0]


def test_poisson_arrivals_rate():
    t = poisson_arrivals(8.0, 20000, seed=3)
    assert np.all(np.diff(t) > 0)
    assert abs(t[-1] / 20000 - 1.0 / 8.0) < 0.005
    np.testing.assert_array_equal(t, poisson_arrivals(8.0, 20000, seed=3))


def test_patch_extent_of_a_plunge():
    """A pure plunge: each step's patch is the disc about the pivot (width and
    height 2r + 2), not the band it sweeps."""
    case = cases.plunge_case(n_steps=3000, amp=0.0)
    w, h = patch_extent(case)
    p = case.params
    x, y = case.contours[0]
    r = float(np.max(np.hypot(x, y))) / p.scale + 4.0
    assert w == math.ceil(2 * r) + 2
    assert abs(h - (math.ceil(2 * r) + 2)) <= 1


def test_estimate_grows_with_the_lattice_and_the_storage():
    for sp in sweep.sweep_specs(8, seed=5):
        e16 = estimate_device_bytes(sweep.case_of(sp, 400, "fp16", amp=0.0))
        e32 = estimate_device_bytes(sweep.case_of(sp, 400, "fp32", amp=0.0))
        nn = sp["nx"] * sp["ny"]
        assert 2 * 9 * 2 * nn < e16 < e32
        # only the population storage differs: 2 buffers x 9 planes x 2 more bytes
        assert e32 - e16 == 2 * 2 * (9 * ((sp["nx"] + 63) // 64 * 64) * sp["ny"] + 2 * 64)


class _FakeCase:
    """Stands in for a solve on the device: steps until its motion ends."""

    closed = []

    def __init__(self, spec):
        self.n = 1
        self.last = spec["last"]
        self.row_len = 2
        self.lib = None
        self.rid = spec["rid"]
        self.bytes = spec["bytes"]
        self.fail_at = spec.get("fail_at")

    @classmethod
    def from_case(cls, case, lib=None):
        return cls(case)

    @property
    def step_index(self):
        return self.n

    def device_bytes(self):
        return self.bytes

    def close(self):
        _FakeCase.closed.append(self.rid)


class _FakeBatch:
    def __init__(self, cases=(), lib=None):
        self.cases = list(cases)

    def add(self, h):
        self.cases.append(h)

    def remove(self, h):
        self.cases.remove(h)

    def run(self, n, errors="raise"):
        out, status = [], []
        for h in self.cases:
            k = max(0, min(n, h.last - h.n + 1))
            fail = h.fail_at is not None and h.n <= h.fail_at < h.n + k
            if fail:
                k = h.fail_at - h.n + 1
            out.append(np.array([[h.rid, h.n + i] for i in range(k)], dtype=float).reshape(k, 2))
            h.n += k
            status.append((-6, "diverged") if fail else None)
        return (out, status) if errors == "return" else out

    def close(self):
        pass


@pytest.mark.parametrize("workers", [0, 1])
def test_server_joins_and_finishes_cases(monkeypatch, workers):
    from fortran_loadfile_mitiwing_b200 import serve

    class _Params:
        scale, uu = 1.0, 1.0

    class _Spec(dict):
        pass

    def make(rid, last, nbytes):
        c = _Spec(rid=rid, last=last, bytes=nbytes)
        c.params = _Params()
        c.table = np.array([[float(last - 1)]])   # motion end time: the last step is `last`
        return lambda: c

    monkeypatch.setattr(serve, "Lbm", _FakeCase)
    monkeypatch.setattr(serve, "Batch", _FakeBatch)
    _FakeCase.closed = []
    lasts = [10, 25, 7, 16]
    with serve.Server(budget_bytes=100, tick_steps=4, workers=workers) as srv:
        for rid, last in enumerate(lasts):
            srv.submit(serve.Request(rid, make(rid, last, 40), estimate=45))
        while not srv.idle():
            srv.tick(wait_for_ready=True)
            assert srv.adm.used <= 100 and len(srv.live) <= 2
        res = {r.rid: r for r in srv.done}
    assert sorted(res) == [0, 1, 2, 3]
    for rid, last in enumerate(lasts):
        np.testing.assert_array_equal(res[rid].rows[:, 1], np.arange(1, last + 1))
        assert res[rid].steps == last
    assert sorted(_FakeCase.closed) == [0, 1, 2, 3]
    assert srv.peak_cases == 2


def test_period_errors():
    from fortran_loadfile_mitiwing_b200.serve import period_errors
    t = np.arange(300)
    ref = np.zeros((300, 3))
    ref[:, 1] = 2.0 + np.sin(2 * np.pi * t / 100.0)
    ref[:, 2] = np.cos(2 * np.pi * t / 100.0)
    got = ref.copy()
    got[100:200, 1] += 0.01          # period 2: C_D mean off by 0.01
    got[200:300, 2] += 0.005         # period 3: C_L mean off by 0.005
    e = period_errors(got, ref, 100.0, 3)
    mean_cd = abs(float(np.mean(ref[100:200, 1])))              # C_D: relative to |mean|
    rms_cl = math.sqrt(float(np.mean(ref[200:300, 2] ** 2)))    # C_L: relative to its RMS
    assert abs(e["cd"] - 0.01 / mean_cd) < 1e-12
    assert abs(e["cl"] - 0.005 / rms_cl) < 1e-12


def test_server_returns_a_failed_case_and_serves_the_rest(monkeypatch):
    from fortran_loadfile_mitiwing_b200 import serve

    class _Params:
        scale, uu = 1.0, 1.0

    class _Spec(dict):
        pass

    def make(rid, last, fail_at=None):
        c = _Spec(rid=rid, last=last, bytes=10, fail_at=fail_at)
        c.params = _Params()
        c.table = np.array([[float(last - 1)]])
        return lambda: c

    monkeypatch.setattr(serve, "Lbm", _FakeCase)
    monkeypatch.setattr(serve, "Batch", _FakeBatch)
    _FakeCase.closed = []
    with serve.Server(budget_bytes=100, tick_steps=5, workers=0) as srv:
        srv.submit(serve.Request(0, make(0, 30), estimate=10))
        srv.submit(serve.Request(1, make(1, 30, fail_at=12), estimate=10))
        srv.submit(serve.Request(2, make(2, 20), estimate=10))
        while not srv.idle():
            srv.tick(wait_for_ready=True)
        res = {r.rid: r for r in srv.done}
    assert res[1].error == (-6, "diverged") and res[1].steps == 12
    assert res[0].error is None and res[0].steps == 30
    assert res[2].error is None and res[2].steps == 20
    assert sorted(_FakeCase.closed) == [0, 1, 2]


def test_cancel_waiting_preparing_and_running(monkeypatch):
    from fortran_loadfile_mitiwing_b200 import serve

    class _Params:
        scale, uu = 1.0, 1.0

    class _Spec(dict):
        pass

    def make(rid, last):
        c = _Spec(rid=rid, last=last, bytes=40)
        c.params = _Params()
        c.table = np.array([[float(last - 1)]])
        return lambda: c

    monkeypatch.setattr(serve, "Lbm", _FakeCase)
    monkeypatch.setattr(serve, "Batch", _FakeBatch)
    _FakeCase.closed = []
    with serve.Server(budget_bytes=100, tick_steps=4, workers=0) as srv:
        for rid, last in enumerate([30, 30, 30, 30]):
            srv.submit(serve.Request(rid, make(rid, last), estimate=45))
        srv.tick(wait_for_ready=True)          # 0 and 1 run; 2 and 3 wait
        r3 = srv.cancel(3)                     # waiting
        assert r3.error == (-2, "cancelled") and 3 not in [q for q, _ in srv.adm.queue]
        r1 = srv.cancel(1)                     # running: leaves the batch with its rows so far
        assert r1.error == (-2, "cancelled") and r1.steps == 4 and 1 not in srv.live
        assert srv.cancel(1) is None and srv.cancel(99) is None
        while not srv.idle():
            srv.tick(wait_for_ready=True)
        res = {r.rid: r for r in srv.done}
    assert res[0].error is None and res[0].steps == 30
    assert res[2].error is None and res[2].steps == 30
    assert sorted(_FakeCase.closed) == [0, 1, 2]


def test_batch_autotune_keeps_the_fastest_pair():
    """Batch.autotune times every (rows per CTA, CTAs per SM) pair on the
    device in alternating order over its rounds, keeps each pair's best
    trial and leaves the batch on the fastest pair; a stand-in replaces the
    library calls (the GPU test checks the results do not depend on it)."""
    from fortran_loadfile_mitiwing_b200.solver import Batch
    b = Batch.__new__(Batch)
    b.rows, b.occupancy, b.b = 0, 0, None
    cost = {(4, 0): 1.3, (4, 3): 1.4, (8, 0): 1.0, (8, 3): 0.9, (16, 0): 1.1, (16, 3): 1.2}
    trials = []

    def set_rows(r):
        b.rows = r

    def set_occupancy(o):
        b.occupancy = o

    def run(n, keep_rows=True):
        trials.append((b.rows, b.occupancy))
        b._n = n

    def device_time():
        # a slower first trial of each pair: the best of the rounds is kept
        first = trials.count((b.rows, b.occupancy)) == 1
        return cost[(b.rows, b.occupancy)] * b._n * (1.5 if first else 1.0), b._n

    b.set_rows, b.set_occupancy, b.run, b.device_time = set_rows, set_occupancy, run, device_time
    timing = b.autotune(steps_per_trial=5, candidates=(4, 8, 16), rounds=2, occupancy=(0, 3))
    assert set(timing) == set(cost)
    assert trials[:6] == [(r, o) for r in (4, 8, 16) for o in (0, 3)]
    assert trials[6:] == trials[:6][::-1]                     # the second round in reverse order
    for pair, t in timing.items():
        assert t == pytest.approx(cost[pair] / 1e3)            # seconds per step, best trial
    assert (b.rows, b.occupancy) == (8, 3)
