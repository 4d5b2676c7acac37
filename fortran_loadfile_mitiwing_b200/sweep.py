"""Batched sweep throughput: many flapping-wing cases of different grid sizes
and kinematics on one GPU, stepped one at a time (each case alone through
lbm_run) and stepped together (a Batch: one lattice launch over a case
table, one launch per immersed-boundary stage), in FP32 and FP16 storage.

Cases (seeded): Nx uniform in [512, 2048] (multiples of 64), Ny = Nx/2,
chord = Ny/4, Re in [100, 2000], heave amplitude in [0.1c, 0.75c], pitch
amplitude in [0, 45] deg, phase in [0, 180] deg, St in [0.15, 0.45]; NACA
0012 with 2 markers per lattice unit of chord, pivot at the quarter chord on
node (2c+1, Ny/2+1), seeded 1e-4 initial perturbation. U0 = 0.05, lowered
per case where the body moves fast so that the fluid speed near it stays
below 0.1 lattice units (`lattice_speed`): with U0 = 0.05 throughout, the
fastest pitching cases reach 0.15-0.27 lattice units per step (Mach 0.3-0.5)
and the lattice-Boltzmann flow diverges within a few hundred steps, in any
storage precision.

Each form runs a fixed sample of steps per case after a warm-up; the report
gives the aggregate lattice updates per second and the cases per hour that
rate gives for 5 flapping periods of every case (a case's period is
c / (f U0) steps, f = St / (2 heave)). Run as
`python -m fortran_loadfile_mitiwing_b200.sweep [--cases N] [--steps S]
[--forms alone_fp32,batch_fp32,batch_fp16] [--no-tune]`, or with `--floor`
for the per-step floor of batches of tiny cases; prints one JSON object.
Needs a GPU.
"""
import argparse
import json
import math
import time

import numpy as np

from . import cases as cs
from .solver import Batch, Lbm

U0 = 0.05


def lattice_speed(spec, uu=U0):
    """Bound on the fluid speed near the body in lattice units: free stream
    plus the body surface speed, U0 (1 + pi St (1 + 0.75 theta0 / h)), the
    heave speed 2 pi f h plus the pitch speed 2 pi f theta0 at the trailing
    edge (0.75 chord behind the pivot), f = St / (2 h)."""
    th = math.radians(spec["pitch_deg"])
    return uu * (1.0 + math.pi * spec["st"] * (1.0 + 0.75 * th / spec["heave"]))


def sweep_specs(n=64, seed=2026, nx_lo=512, nx_hi=2048, u_lat=0.1):
    """Seeded cases; U0 = min(0.05, the U0 that keeps `lattice_speed` at
    u_lat), so that fast pitching and heaving keep the lattice Mach number
    below about u_lat / c_s (c_s = 1/sqrt 3). u_lat=None keeps U0 = 0.05."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        nx = int(rng.integers(nx_lo // 64, nx_hi // 64 + 1)) * 64
        ny = nx // 2
        chord = ny // 4
        spec = dict(nx=nx, ny=ny, chord=chord, pivot=(2 * chord + 1, ny // 2 + 1), markers=2 * chord,
                    re=float(rng.uniform(100.0, 2000.0)), heave=float(rng.uniform(0.1, 0.75)),
                    pitch_deg=float(rng.uniform(0.0, 45.0)), phase_deg=float(rng.uniform(0.0, 180.0)),
                    st=float(rng.uniform(0.15, 0.45)), seed=seed + c)
        uu = U0 if u_lat is None else min(U0, u_lat * U0 / lattice_speed(spec))
        spec["uu"] = uu
        spec["period_steps"] = chord / (spec["st"] / (2.0 * spec["heave"]) * uu)
        out.append(spec)
    return out


def case_of(spec, n_steps, precision, amp=1.0e-4):
    """The case of a sweep spec (amp=0: without the perturbation arrays)."""
    kw = {k: spec[k] for k in ("nx", "ny", "chord", "pivot", "markers", "re", "heave", "pitch_deg", "phase_deg",
                               "st", "seed")}
    return cs.heave_pitch_case(n_steps=n_steps, precision=precision, uu=spec.get("uu", U0), amp=amp, **kw)


def make(spec, n_steps, precision, lib=None):
    return Lbm.from_case(case_of(spec, n_steps, precision), lib)


def cases_per_hour(specs, lups_per_s, periods=5):
    work = sum(s["nx"] * s["ny"] * periods * s["period_steps"] for s in specs)
    return len(specs) * 3600.0 * lups_per_s / work


def run_alone(specs, steps, warmup, precision, lib=None):
    total, lups = 0.0, 0
    for sp in specs:
        s = make(sp, steps + warmup + 8, precision, lib)
        s.run(warmup, keep_rows=False)
        t0 = time.perf_counter()
        s.run(steps, keep_rows=False)
        total += time.perf_counter() - t0
        lups += sp["nx"] * sp["ny"] * steps
        s.close()
    return lups / total, total


def run_batch(specs, steps, warmup, precision, lib=None, tune=True):
    hs = [make(sp, steps + warmup + 64, precision, lib) for sp in specs]
    b = Batch(hs)
    timing = b.autotune(steps_per_trial=max(2, warmup // 3), candidates=(4, 8, 16)) if tune else {}
    timing = {f"rows {r}, ctas/SM {o or 'max'}": t for (r, o), t in timing.items()}
    choice = {"rows_per_cta": b.rows, "ctas_per_sm": b.occupancy}
    b.run(warmup, keep_rows=False)
    t0 = time.perf_counter()
    done = b.run(steps, keep_rows=False)
    el = time.perf_counter() - t0
    assert all(d == steps for d in done), done
    lups = sum(sp["nx"] * sp["ny"] * steps for sp in specs)
    b.close()
    for h in hs:
        h.close()
    return lups / el, el, timing, choice


def launch_floor(counts=(1, 8, 64), steps=192, warmup=24, lib=None):
    """Time per step of batches of tiny cases (128x64 lattices, 40 markers,
    where the GPU has almost nothing to do): the floor that issuing the
    launches sets, with the steady steps replayed as CUDA graphs and with
    every launch issued from the host, and one case stepped alone (lbm_run)
    for comparison. Wall clock around one run of `steps` steps after a
    warm-up run, in microseconds per step; the device time of the same run
    (lbm_batch_get_timing) beside it."""
    out = {}
    n_steps = 2 * (steps + warmup) + 64
    one = Lbm.from_case(cs.small_case(nx=128, ny=64, n_steps=n_steps), lib)
    one.run(warmup, keep_rows=False)
    t0 = time.perf_counter()
    one.run(steps, keep_rows=False)
    out["alone_us"] = (time.perf_counter() - t0) / steps * 1e6
    one.close()
    for n in counts:
        hs = [Lbm.from_case(cs.small_case(nx=128, ny=64, n_steps=n_steps, seed=7 + c), lib) for c in range(n)]
        row = {}
        with Batch(hs) as b:
            for graphs in (True, False):
                b.set_graphs(graphs)
                b.run(warmup, keep_rows=False)
                t0 = time.perf_counter()
                b.run(steps, keep_rows=False)
                el = time.perf_counter() - t0
                ms, k = b.device_time()
                key = "graphs" if graphs else "stream"
                row[key + "_us"] = el / steps * 1e6
                row[key + "_device_us"] = ms * 1e3 / max(k, 1)
        for h in hs:
            h.close()
        out[str(n)] = row
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=12)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--floor", action="store_true", help="only the per-step floor of batches of tiny cases")
    ap.add_argument("--forms", default="alone_fp32,batch_fp32,batch_fp16",
                    help="comma-separated subset of alone_fp32, batch_fp32, batch_fp16")
    ap.add_argument("--no-tune", action="store_true", help="batches keep the cases' own rows per CTA")
    args = ap.parse_args()
    if args.floor:
        print(json.dumps(launch_floor()))
        return
    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    specs = sweep_specs(args.cases, args.seed)
    res = {"cases": args.cases, "steps_per_case": args.steps, "seed": args.seed,
           "grid_nodes_total": sum(s["nx"] * s["ny"] for s in specs)}
    if "alone_fp32" in forms:
        r, t = run_alone(specs, args.steps, args.warmup, "fp32")
        res["alone_fp32"] = {"mlups": r / 1e6, "seconds": t, "cases_per_hour_5_periods": cases_per_hour(specs, r)}
    for prec in ("fp32", "fp16"):
        if "batch_" + prec not in forms:
            continue
        r, t, timing, choice = run_batch(specs, args.steps, args.warmup, prec, tune=not args.no_tune)
        res["batch_" + prec] = {"mlups": r / 1e6, "seconds": t, "cases_per_hour_5_periods": cases_per_hour(specs, r),
                                "autotuned": choice, "autotune_s_per_step": timing}
    if "alone_fp32" in res:
        base = res["alone_fp32"]["cases_per_hour_5_periods"]
        for k in ("batch_fp32", "batch_fp16"):
            if k in res:
                res[k]["vs_alone_fp32"] = res[k]["cases_per_hour_5_periods"] / base
    print(json.dumps(res))


if __name__ == "__main__":
    main()
