"""Generates the golden fixtures of tests/test_golden.py with the CPU oracle.

The reference ships no golden vectors and cannot be compiled in this image, so
these fixtures anchor the oracle (and through it the CUDA path) against
regressions: a tiny heaving/pitching NACA 0012 case and a tandem two-wing
case with the smoothed kernel, FP64, populations/fields/force rows after a
fixed number of steps.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fortran_loadfile_mitiwing_b200 import cases  # noqa: E402


def golden_cases():
    return {
        "tiny_heave_pitch": (cases.small_case(nx=48, ny=32, chord=12, pivot=(17, 17), markers=16, n_steps=40,
                                              pitch_deg=15.0, precision="fp64", seed=11), 30),
        "tandem_smooth": (cases.small_case(nx=72, ny=32, chord=8, pivot=(17, 17), markers=12, n_steps=30,
                                           wings=2, delta=1, precision="fp64", seed=12), 20),
    }


def main():
    import pyoracle
    for name, (case, nsteps) in golden_cases().items():
        o = pyoracle.Oracle.from_case(case)
        rows = o.run(nsteps)
        rho, u, v = o.fields()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), f=o.populations(), rho=rho, u=u, v=v,
                            rows=rows, steps=nsteps)
        print(name, rows.shape, float(np.abs(rows[:, 1:4]).max()))


if __name__ == "__main__":
    main()
