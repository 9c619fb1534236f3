"""Both GPU forms against the FP64 oracle over 1000 steps of a driven wake.

Single trajectories diverge chaotically within tens of plasma periods, so
the comparison after N steps is on the aggregates: total field energy,
particle kinetic energy, the alive count and the Gauss-law residual.  The
case is the wake physics at a size the oracle steps in seconds: 64 x 512
cells over 0.025 x 0.2 m, electrons and protons at 2 ppc and 1e17 m^-3,
1 eV electrons, a gamma = 5 bunch (r 2.5 mm, length 1 cm, 5e16 m^-3)
injected at z = 0 with the upstream TESTMODE sequence, absorbing layer,
relativistic Boris; the bunch stays inside the grid for the 1000 steps.

Tolerances (the measured values on a B200 in brackets):
  * FP64 plain form: field and kinetic energy within 1e-3 of the oracle's
    (5e-10, < 2e-10), alive count equal, Gauss relative residual <= 1e-9
    (4.9e-12, rounding level);
  * FP32 cell-local form: field and kinetic energy within 1e-3 of the
    oracle's (8.7e-7, 3.7e-6), alive count equal, Gauss relative residual
    <= 1e-5 (1.3e-8).
"""
import pytest

from helpers import diagnostics_np, oracle_from_workload
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

STEPS = 1000


def test_driven_wake_1000_steps_against_the_oracle():
    wl = W.wake_config(n_grid_r=65, n_grid_z=513, r_size=0.025, z_size=0.2, ppc=2,
                       beam_radius=2.5e-3, beam_length=0.01, steps=STEPS)
    orc = oracle_from_workload(wl)
    orc.run(STEPS)
    do = diagnostics_np(orc, 3)
    assert do["field_energy"] > 0 and do["alive"] > 2 * wl.species[0].n
    assert do["gauss_residual"] <= 1e-9 * do["gauss_norm"]
    for precision, gauss_tol in (("fp64", 1e-9), ("fp32", 1e-5)):
        gpu = api.from_workload(wl, precision=precision)
        gpu.mark_initial_charge()
        gpu.step(STEPS)
        gpu.sync()
        dg = gpu.diagnostics()
        gpu.close()
        print("%s: field energy %.9e (oracle %.9e), kinetic %.9e (%.9e), gauss %.2e" % (
            precision, dg["field_energy"], do["field_energy"], dg["kinetic_energy"],
            do["kinetic_energy"], dg["gauss_residual"] / dg["gauss_norm"]))
        assert abs(dg["field_energy"] - do["field_energy"]) <= 1e-3 * do["field_energy"], precision
        assert abs(dg["kinetic_energy"] - do["kinetic_energy"]) <= 1e-3 * do["kinetic_energy"], \
            precision
        assert dg["alive"] == do["alive"], precision
        assert dg["gauss_residual"] <= gauss_tol * dg["gauss_norm"], precision
