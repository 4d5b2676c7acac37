"""Serving: requests admitted against a device-memory budget join a running
batch and leave it when their motion ends; each result is bit-for-bit the
result of solving the case alone. The device-memory estimate used for
admission covers what a case holds."""
import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Lbm, cases
from fortran_loadfile_mitiwing_b200.serve import Request, Server, estimate_device_bytes

pytestmark = pytest.mark.gpu

SPECS = [
    dict(nx=96, ny=64, chord=24, pivot=(33, 33), markers=40, heave=0.25, pitch_deg=10.0, st=0.3, seed=7),
    dict(nx=160, ny=96, chord=32, pivot=(50, 49), markers=64, heave=0.2, pitch_deg=20.0, st=0.25, seed=11),
    dict(nx=128, ny=64, chord=20, pivot=(40, 33), markers=36, heave=0.3, pitch_deg=0.0, st=0.35, seed=13),
]


def make(i, n_steps, precision="fp32"):
    return lambda: cases.small_case(precision=precision, n_steps=n_steps, **SPECS[i % len(SPECS)])


@pytest.mark.parametrize("precision", ["fp32", "fp16", "fp64"])
def test_estimate_covers_device_bytes(gpu_lib, precision):
    for i in range(len(SPECS)):
        case = make(i, 60, precision)()
        est = estimate_device_bytes(case)
        with Lbm.from_case(case, gpu_lib) as s:
            s.run(1, keep_rows=False)
            got = s.device_bytes()
        assert got <= est <= got * 1.02, (precision, i, est, got)


@pytest.mark.parametrize("workers,tick", [(0, 7), (1, 7), (1, 40)])
def test_served_results_equal_alone(gpu_lib, workers, tick):
    """Ticks of 7 steps run every step from the host; ticks of 40 replay
    graph segments of 16 steps between their first and last steps."""
    lens = [30, 52, 41, 23, 35] if tick < 20 else [60, 90, 75, 44, 66]
    reqs = [Request(i, make(i, n)) for i, n in enumerate(lens)]
    ests = [estimate_device_bytes(r.make()) for r in reqs]
    budget = sorted(ests)[-1] + sorted(ests)[-2]          # room for two cases at most
    with Server(budget, tick_steps=tick, lib=gpu_lib, keep_handles=True, workers=workers) as srv:
        for r in reqs:
            srv.submit(r)
        while not srv.idle():
            srv.tick(wait_for_ready=True)
        if tick >= 20:
            assert srv.batch.graph_stats()[0] > 0         # steps run as graph segments
        res = sorted(srv.done, key=lambda r: r.rid)
        assert [r.rid for r in res] == list(range(len(lens)))
        assert 1 <= srv.peak_cases <= 2 and srv.peak_used <= budget
        assert len({r.started for r in res}) > 1          # cases joined a running batch
        for r, n in zip(res, lens):
            with Lbm.from_case(make(r.rid, n)(), gpu_lib) as a:
                ref = a.run(200)
                assert r.steps == ref.shape[0]
                np.testing.assert_array_equal(r.rows, ref, err_msg=f"request {r.rid} force rows")
                np.testing.assert_array_equal(r.handle.populations(), a.populations(),
                                              err_msg=f"request {r.rid} populations")
            r.handle.close()


def test_cancelled_request_leaves_the_others_exact(gpu_lib):
    lens = [30, 40, 26]
    reqs = [Request(i, make(i, n)) for i, n in enumerate(lens)]
    with Server(10 ** 10, tick_steps=6, lib=gpu_lib, keep_handles=True, workers=0) as srv:
        for r in reqs:
            srv.submit(r)
        srv.tick(wait_for_ready=True)
        srv.tick(wait_for_ready=True)
        cancelled = srv.cancel(1)                 # running: leaves the batch after 12 steps
        assert cancelled.error[1] == "cancelled" and cancelled.steps == 12
        while not srv.idle():
            srv.tick(wait_for_ready=True)
        res = {r.rid: r for r in srv.done}
        for rid in (0, 2):
            with Lbm.from_case(make(rid, lens[rid])(), gpu_lib) as a:
                np.testing.assert_array_equal(res[rid].rows, a.run(200))
                np.testing.assert_array_equal(res[rid].handle.populations(), a.populations())
            res[rid].handle.close()
        with Lbm.from_case(make(1, lens[1])(), gpu_lib) as a:
            np.testing.assert_array_equal(cancelled.rows, a.run(12))
