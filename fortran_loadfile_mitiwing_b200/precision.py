"""Storage-precision study of the time step (the FP16/BF16 deviation storage
against an FP64 run of the same case on the GPU).

Populations are stored as deviations f_i - w_i from the lattice weights; with
FP16 or BF16 storage the collision and IB arithmetic stay FP32 (the lattice
kernels' compute type) and the marker system and force sums stay FP64. The
study runs one case in each storage precision and compares it with the FP64
run over whole flapping periods:

  - the relative L2 error of the velocity field, ||u_p - u_64|| / ||u_64||
    over (u, v), at the ends of chosen periods;
  - per period, the error of the mean of C_D relative to |mean C_D| of the
    FP64 period, the error of the mean of C_L relative to the FP64 period's
    RMS of C_L (C_L of a symmetric plunge has a mean near zero, so a
    mean-relative error would divide by ~0), and the RMS of each
    coefficient's difference relative to the FP64 period's RMS of it.

Run as `python -m fortran_loadfile_mitiwing_b200.precision [--periods N]`; it
prints one JSON object. Needs a GPU.
"""
import argparse
import json
import math

import numpy as np

from . import cases
from .solver import Lbm

# force-row columns of a one-wing case: time, C_x (drag), C_y (lift), C_m, ...
COL_CD, COL_CL = 1, 2


def steps_per_period(case):
    """Steps of one flapping period of a `cases.plunge_case` (its motion
    frequency St / (2 heave) in chord-per-U0 time units, dt = scale U0)."""
    freq = 0.3 / (2.0 * 0.25)
    return int(round(1.0 / (freq * case.params.scale * case.params.uu)))


def run_case(precision, n_steps, report_steps, lib=None):
    """Runs the plunge case in `precision` for `n_steps`; returns the force
    rows and the (u, v) fields at each step of `report_steps`."""
    case = cases.plunge_case(n_steps=n_steps + 8, precision=precision)
    s = Lbm.from_case(case, lib)
    rows, fields, done = [], {}, 0
    for target in sorted(report_steps):
        rows.append(s.run(target - done))
        done = target
        _, u, v = s.fields()
        fields[target] = (u.copy(), v.copy())
    if done < n_steps:
        rows.append(s.run(n_steps - done))
    s.close()
    return np.concatenate(rows), fields


def compare(rows_p, fields_p, rows_64, fields_64, period):
    out = {"velocity_l2": {}, "periods": []}
    for step, (u64, v64) in fields_64.items():
        up, vp = fields_p[step]
        num = math.sqrt(float(np.sum((up - u64) ** 2) + np.sum((vp - v64) ** 2)))
        den = math.sqrt(float(np.sum(u64 ** 2) + np.sum(v64 ** 2)))
        out["velocity_l2"][str(step // period)] = num / den
    n_per = rows_64.shape[0] // period
    for k in range(n_per):
        sl = slice(k * period, (k + 1) * period)
        rec = {"period": k + 1}
        for name, col in (("cd", COL_CD), ("cl", COL_CL)):
            ref, got = rows_64[sl, col], rows_p[sl, col]
            rms_ref = math.sqrt(float(np.mean(ref ** 2)))
            mean_ref = float(np.mean(ref))
            # C_D's per-period mean is far from zero: its error is relative to
            # |mean|; C_L's mean is close to zero (a symmetric section in
            # symmetric motion), so its error is relative to its RMS
            scale = abs(mean_ref) if name == "cd" else rms_ref
            rec[name + "_mean_ref"] = mean_ref
            rec[name + "_mean_err"] = abs(float(np.mean(got)) - mean_ref) / scale
            rec[name + "_rms_err"] = math.sqrt(float(np.mean((got - ref) ** 2))) / rms_ref
        out["periods"].append(rec)
    return out


def study(periods=10, report=(5, 10), precisions=("fp16", "bf16", "fp32"), lib=None):
    """The study over `periods` periods of the 400x200 plunge case; velocity
    errors at the ends of the periods in `report`."""
    period = steps_per_period(cases.plunge_case(n_steps=8))
    n = periods * period
    report_steps = [p * period for p in report if p <= periods]
    rows_64, fields_64 = run_case("fp64", n, report_steps, lib)
    res = {"case": "plunge 400x200, chord 80, Re 100, St 0.3, 160 markers", "steps_per_period": period,
           "periods": periods, "reference": "fp64 storage on the GPU"}
    for p in precisions:
        rows_p, fields_p = run_case(p, n, report_steps, lib)
        res[p] = compare(rows_p, fields_p, rows_64, fields_64, period)
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--periods", type=int, default=10)
    args = ap.parse_args()
    print(json.dumps(study(periods=args.periods)))


if __name__ == "__main__":
    main()
