"""Pinning the microchannel steady oracle.

The reference solves the steady state of a microchannel model only through
SuperLU (absent here), so the FP64 oracle of the BiCGStab solver is the
restated system G T = P solved by sparse LU.  It is pinned to the
reference's own model: the reference's slope function (slope_fn_grid,
temperature_grid.c:3130-3601, run from the reference build) vanishes at the
direct solution, i.e. it is the fixed point of the reference's transient."""
import numpy as np
import pytest

from hotspot_b200 import workloads as W
from oracle import ref as R
from oracle.restatement import OracleModel


@pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed", [41, 44])
def test_direct_microchannel_steady_is_reference_fixed_point(workdir, seed):
    sc = W.scenario_microchannel(workdir, seed=seed, grid=32, die=32 * 20e-6, blocks=8)
    r, o = R.RefModel(sc), OracleModel(sc)
    p = r.power_vector(sc.block_power[0])
    pg = r.power_grid(p.copy())
    T, _ = o.steady_direct(p)
    s_fix = np.max(np.abs(r.slope(T, pg)))
    t0 = np.full_like(T, o.init_temp)
    s_init = np.max(np.abs(r.slope(t0, pg)))
    r.close()
    assert s_fix <= 1e-9 * s_init, (s_fix, s_init)
