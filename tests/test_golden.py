"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py):
the oracle must reproduce them (CPU), and the CUDA path in FP64 storage must
match them (GPU)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_golden import golden_cases  # noqa: E402

CASES = golden_cases()


def load(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_golden(oracle_mod, name):
    case, nsteps = CASES[name]
    g = load(name)
    o = oracle_mod.Oracle.from_case(case)
    rows = o.run(nsteps)
    np.testing.assert_allclose(o.populations(), g["f"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(rows, g["rows"], rtol=1e-11, atol=1e-11)
    for key, arr in zip(("rho", "u", "v"), o.fields()):
        np.testing.assert_allclose(arr, g[key], rtol=0, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_cuda_fp64_matches_golden(gpu_lib, name):
    from fortran_loadfile_mitiwing_b200 import Lbm
    case, nsteps = CASES[name]
    g = load(name)
    s = Lbm.from_case(case, gpu_lib)
    rows = s.run(nsteps)
    assert np.abs(s.populations() - g["f"]).max() < 1e-11
    rel = np.abs(rows[:, 1:] - g["rows"][:, 1:]).max() / np.abs(g["rows"][:, 1:]).max()
    assert rel < 1e-9
    for key, arr in zip(("rho", "u", "v"), s.fields()):
        assert np.abs(arr - g[key]).max() < 1e-11
