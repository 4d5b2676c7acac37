"""The global mass check on the GPU (lbm_mass, and the check lbm_run and
lbm_batch_run make): an FP64 sum over every node and direction of the
populations, in a fixed order.

Tolerances: FP64 storage against the oracle's populations summed on the host,
1e-12 relative (both sum the same FP64 values, in different orders); the same
state gives the same mass bit for bit, alone or in a batch.
"""
import ctypes as C

import numpy as np
import pytest

from fortran_loadfile_mitiwing_b200 import Batch, Lbm, LbmError, cases
from fortran_loadfile_mitiwing_b200 import _abi

pytestmark = pytest.mark.gpu


def test_mass_matches_the_oracle_in_fp64(gpu_lib, oracle_mod):
    case = cases.small_case(precision="fp64", n_steps=100)
    g = Lbm.from_case(case, gpu_lib)
    o = oracle_mod.Oracle.from_case(case)
    m0 = g.mass()
    assert abs(m0 - o.populations().sum()) <= 1e-12 * abs(m0)
    g.run(50)
    o.run(50)
    mo = o.populations().sum()
    m = g.mass()
    assert abs(m - mo) <= 1e-12 * abs(mo), (m, mo)
    assert m == g.mass()   # the same state, the same sum


def test_nonfinite_population_stops_the_run(gpu_lib):
    """A NaN placed far from the body (where no immersed-boundary check reads
    the flow) is found by the mass check at the end of the run."""
    case = cases.small_case(precision="fp32", n_steps=100)
    g = Lbm.from_case(case, gpu_lib)
    g.run(5)
    f = g.populations().reshape(9, g.ny, g.nx)
    f[0, 10, 85] = np.nan
    g.set_populations(f)
    with pytest.raises(LbmError) as ei:
        g.run(3)
    assert ei.value.status == _abi.LBM_ERR_NONFINITE
    assert "mass" in str(ei.value)
    m = C.c_double()
    assert gpu_lib.lbm_mass(g.h, C.byref(m)) == _abi.LBM_ERR_NONFINITE
    assert not np.isfinite(m.value)


def test_batch_checks_mass_and_matches_alone(gpu_lib):
    """After a batch run each case's mass is the one of the same case run
    alone, bit for bit (the batch checked it at the end of the run)."""
    specs = [cases.small_case(precision="fp32", n_steps=60),
             cases.small_case(nx=128, ny=80, chord=30, pivot=(40, 40), precision="fp32", n_steps=60)]
    alone = []
    for c in specs:
        s = Lbm.from_case(c, gpu_lib)
        s.run(20)
        alone.append(s.mass())
        s.close()
    hs = [Lbm.from_case(c, gpu_lib) for c in specs]
    b = Batch(hs, gpu_lib)
    b.run(20)
    for h, m in zip(hs, alone):
        assert h.mass() == m
    b.close()
