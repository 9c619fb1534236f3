"""The CPU side of `bench.py --workload diag`: the upstream diagnostics
(oracle/_ref) timed on two seeded plasma samples and extrapolated along a
straight line in the particle count; the Poisson solve timed on its grid."""
import pytest

import bench
from oracle import refsim
from pdp3_b200 import workloads as W


@pytest.mark.skipif(not refsim.available("boris"), reason="oracle/_ref not built")
def test_diag_cpu_times_extrapolate_from_two_samples():
    wl = W.small_config(n_grid_r=33, n_grid_z=129, r_size=0.02, z_size=0.16, ppc=16)
    out = bench.diag_cpu_times(wl, (0.25, 0.5), 1)
    n_el = wl.species[0].n
    for name in ("charge_density", "temperature_electrons", "density_electrons"):
        s = out[name]["samples"]
        assert len(s) == 2 and s[0]["particles"] < s[1]["particles"]
        full = sum(x.n for x in wl.species) if name == "charge_density" else n_el
        assert s[1]["particles"] < full
        # never below the larger sample's own time
        assert out[name]["ms_extrapolated"] >= s[1]["ms"] > 0


@pytest.mark.skipif(not refsim.available("boris"), reason="oracle/_ref not built")
def test_diag_cpu_poisson_runs_on_its_grid():
    nr, nz = bench.DIAG_POISSON_GRID
    assert ((2 * nz + 2) & (2 * nz + 1)) == 0  # the radix-2 transform's size
    assert bench.diag_cpu_poisson(1) > 0
