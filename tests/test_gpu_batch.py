"""Batches: several cases of different grid sizes and kinematics stepped
together (one lattice launch driven by a case table, one launch per
immersed-boundary stage) give each case exactly the results of running it
alone: force rows and populations bit-for-bit."""
import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Batch, Lbm, cases

pytestmark = pytest.mark.gpu

SPECS = [
    dict(nx=96, ny=64, chord=24, pivot=(33, 33), markers=40, heave=0.25, pitch_deg=10.0, st=0.3, seed=7),
    dict(nx=160, ny=96, chord=32, pivot=(50, 49), markers=64, heave=0.2, pitch_deg=20.0, st=0.25, seed=11),
    dict(nx=128, ny=64, chord=20, pivot=(40, 33), markers=36, heave=0.3, pitch_deg=0.0, st=0.35, seed=13),
]


def build(precision, n_steps, specs=SPECS, lib=None):
    return [Lbm.from_case(cases.small_case(precision=precision, n_steps=n_steps, **sp), lib) for sp in specs]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_equals_each_case_alone(gpu_lib, precision):
    steps = 37   # several factorization batches of 4 steps, and a partial one
    together = build(precision, steps + 20, lib=gpu_lib)
    alone = build(precision, steps + 20, lib=gpu_lib)
    with Batch(together) as b:
        rows_b = b.run(steps)
    for c, (t, a) in enumerate(zip(together, alone)):
        rows_a = a.run(steps)
        np.testing.assert_array_equal(rows_b[c], rows_a, err_msg=f"case {c} force rows")
        np.testing.assert_array_equal(t.populations(), a.populations(), err_msg=f"case {c} populations")


def test_batch_cases_stop_at_their_motion_end(gpu_lib):
    lens = [30, 50, 40]
    together = [Lbm.from_case(cases.small_case(precision="fp32", n_steps=n, **sp), gpu_lib) for n, sp in zip(lens, SPECS)]
    with Batch(together) as b:
        done = b.run(100, keep_rows=False)
    # a case runs while (n - 1) dt <= motion end; the table covers n_steps rows
    alone = [Lbm.from_case(cases.small_case(precision="fp32", n_steps=n, **sp), gpu_lib) for n, sp in zip(lens, SPECS)]
    for c, a in enumerate(alone):
        rows_a = a.run(100)
        assert done[c] == rows_a.shape[0], (c, done[c], rows_a.shape[0])
        np.testing.assert_array_equal(together[c].populations(), a.populations())


def test_autotuned_batch_still_equals_alone(gpu_lib):
    together = build("fp32", 120, lib=gpu_lib)
    alone = build("fp32", 120, lib=gpu_lib)
    with Batch(together) as b:
        # rows per CTA x lattice CTAs per SM, 2 rounds of 5 steps: 60 steps
        timing = b.autotune(steps_per_trial=5, candidates=(4, 8, 16), rounds=2, occupancy=(0, 2))
        assert set(timing) == {(r, o) for r in (4, 8, 16) for o in (0, 2)}
        assert (b.rows, b.occupancy) in timing
        assert all(0 < t < 1.0 for t in timing.values())
        b.run(10, keep_rows=False)
        ms, n = b.device_time()      # device time of the last run's steps
        assert n == 10 and ms > 0
    for t, a in zip(together, alone):
        a.run(70)
        np.testing.assert_array_equal(t.populations(), a.populations())


def test_cases_join_and_leave_at_different_steps(gpu_lib):
    """Cases stepped alone before joining, joining a running batch (an empty
    one included), leaving it and stepped alone afterwards each end bit-for-bit
    where the same number of steps alone ends."""
    mixed = build("fp32", 120, lib=gpu_lib)
    alone = build("fp32", 120, lib=gpu_lib)
    rows = [[] for _ in mixed]

    def take(b, n):
        for case, r in zip(b.cases, b.run(n)):
            rows[mixed.index(case)].append(r)

    rows[0].append(mixed[0].run(6))      # mid-way through a factorization batch of 4 steps
    rows[2].append(mixed[2].run(13))
    with Batch([], lib=gpu_lib) as b:
        b.add(mixed[0])
        b.add(mixed[1])
        take(b, 9)
        b.add(mixed[2])                  # joins at step 14 beside cases at 16 and 10
        take(b, 10)
        b.remove(mixed[0])
        take(b, 5)
        rows[0].append(mixed[0].run(7))  # alone in between
        b.add(mixed[0])
        take(b, 11)
        assert len(b) == 3
    for c, (m, a) in enumerate(zip(mixed, alone)):
        got = np.concatenate(rows[c])
        ref = a.run(got.shape[0])
        assert m.step_index == a.step_index
        np.testing.assert_array_equal(got, ref, err_msg=f"case {c} force rows")
        np.testing.assert_array_equal(m.populations(), a.populations(), err_msg=f"case {c} populations")


def test_rows_of_a_case_ending_alone_in_a_run(gpu_lib):
    """The only case of a run ends before the run's step count: its last rows
    still reach the host."""
    t = Lbm.from_case(cases.small_case(precision="fp32", n_steps=23, **SPECS[0]), gpu_lib)
    a = Lbm.from_case(cases.small_case(precision="fp32", n_steps=23, **SPECS[0]), gpu_lib)
    with Batch([t]) as b:
        r1 = b.run(21)[0]
        r2 = b.run(7)[0]
    ref = a.run(100)
    assert r1.shape[0] + r2.shape[0] == ref.shape[0]
    np.testing.assert_array_equal(np.concatenate([r1, r2]), ref)


def test_batch_refuses_mixed_precision(gpu_lib):
    from fortran_loadfile_mitiwing_b200 import LbmError
    a = build("fp32", 20, specs=SPECS[:1], lib=gpu_lib)[0]
    d = build("fp64", 20, specs=SPECS[1:2], lib=gpu_lib)[0]
    with Batch([a]) as b:
        with pytest.raises(LbmError):
            b.add(d)
        with pytest.raises(LbmError):
            b.add(a)                     # already in the batch
        assert len(b) == 1 and b.lib.lbm_batch_count(b.b) == 1


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_odd_row_chunks_equal_alone(gpu_lib, precision):
    """The lattice update pairs rows of a chunk for the paired FP32
    instructions; with 5 or 7 rows per CTA every chunk ends with an unpaired
    row, and a case with an odd number of interior rows ends the lattice with
    one: each node's arithmetic is the same in either half of a pair, so the
    results stay bit-for-bit those of the case alone (8 rows per CTA)."""
    specs = SPECS[:2] + [dict(nx=100, ny=61, chord=20, pivot=(35, 31), markers=36, heave=0.2, pitch_deg=15.0,
                              st=0.3, seed=17)]
    for rows in (5, 7):
        together = build(precision, 40, specs=specs, lib=gpu_lib)
        alone = build(precision, 40, specs=specs, lib=gpu_lib)
        with Batch(together) as b:
            b.set_rows(rows)
            rows_b = b.run(21)
        for c, (t, a) in enumerate(zip(together, alone)):
            np.testing.assert_array_equal(rows_b[c], a.run(21), err_msg=f"rows {rows} case {c}")
            np.testing.assert_array_equal(t.populations(), a.populations(), err_msg=f"rows {rows} case {c}")


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_graph_segments_equal_stream_code(gpu_lib, precision):
    """Steady steps replayed as CUDA graphs give the steps the host issues one
    by one, bit for bit: two runs (the second starting mid-way through a
    factorization batch and through the force ring's rows), with a case
    joining in between at another phase of its factorization batches; the
    graphs of repeated segments are reused, not captured again."""
    graphed = build(precision, 160, lib=gpu_lib)
    plain = build(precision, 160, lib=gpu_lib)
    late_g = Lbm.from_case(cases.small_case(precision=precision, n_steps=160, **SPECS[0]), gpu_lib)
    late_p = Lbm.from_case(cases.small_case(precision=precision, n_steps=160, **SPECS[0]), gpu_lib)
    late_g.run(3)
    late_p.run(3)
    rows = {}
    for key, cs, late, graphs in (("g", graphed, late_g, True), ("p", plain, late_p, False)):
        with Batch(cs) as b:
            b.set_graphs(graphs)
            r1 = b.run(54)
            b.add(late)
            r2 = b.run(61)
            rows[key] = (r1, r2)
            stats = b.graph_stats()
        if graphs:
            # 3 segments in the first run, 3 in the second; both argument
            # buffers alternate, so at most 2 structures per run
            assert stats[0] == 16 * 6 and stats[1] == 6 and 1 <= stats[2] <= 5, stats
        else:
            assert stats == (0, 0, 0), stats
    for c in range(len(SPECS)):
        np.testing.assert_array_equal(rows["g"][0][c], rows["p"][0][c], err_msg=f"run 1 case {c}")
        np.testing.assert_array_equal(rows["g"][1][c], rows["p"][1][c], err_msg=f"run 2 case {c}")
        np.testing.assert_array_equal(graphed[c].populations(), plain[c].populations(), err_msg=f"case {c}")
    np.testing.assert_array_equal(rows["g"][1][3], rows["p"][1][3], err_msg="joined case")
    np.testing.assert_array_equal(late_g.populations(), late_p.populations())
    # and the graphed batch equals each case alone
    alone = build(precision, 160, lib=gpu_lib)
    for c, a in enumerate(alone):
        np.testing.assert_array_equal(np.concatenate(rows["g"][0][c:c + 1] + rows["g"][1][c:c + 1]), a.run(115),
                                      err_msg=f"alone case {c}")
        np.testing.assert_array_equal(graphed[c].populations(), a.populations())
