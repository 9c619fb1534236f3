"""The large-case machinery on a small grid: plasma generated on the GPU
(pdp3g_add_species_device), a density ramp carried by the weights, the Vay
pusher with a bunch, and periodic re-sorting by cell.

* the generated particles sit inside their cells, in cell order, with the
  weights n(z_cell) V_cell / ppc summing to the ramp's total;
* 30 steps of the FP32 form with a re-sort every 10 steps match the FP64
  form stepped without re-sorting: total field energy within 1e-3, Gauss
  residual of both forms at or below 1e-5 relative.
"""
import math

import numpy as np
import pytest

from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_large(ppc=8, sort_interval=10):
    return W.large_config(n_grid_r=65, n_grid_z=257, r_size=0.1 / 8, z_size=0.8 / 16, ppc=ppc,
                          beam_radius=2e-3, beam_length=4e-3, sort_interval=sort_interval)


def test_device_plasma_layout_and_weights():
    wl = small_large()
    sim = api.from_workload(wl, precision="fp64")
    dp = wl.device_plasma
    dr, dz = wl.dr, wl.dz
    nrc, nzc = wl.n_grid_r - 1, wl.n_grid_z - 1
    e = sim.species(0)
    i = np.ceil(e["r"] / dr).astype(np.int64) - 1
    k = np.ceil(e["z"] / dz).astype(np.int64) - 1
    p = np.arange(e["r"].size)
    assert np.array_equal(i, p // (nzc * dp.ppc))
    assert np.array_equal(k, (p // dp.ppc) % nzc)
    # total weight: sum over cells of n(z_c) V_c (domain [dr/2, R-dr/2] x [dz/2, Z-dz/2])
    r_e = np.concatenate(([dr / 2], dr * np.arange(1, nrc), [wl.r_size - dr / 2]))
    z_e = np.concatenate(([dz / 2], dz * np.arange(1, nzc), [wl.z_size - dz / 2]))
    zc = 0.5 * (z_e[1:] + z_e[:-1])
    n_z = dp.n_max * np.minimum(zc / dp.z_ramp, 1.0)
    ring = math.pi * (r_e[1:] ** 2 - r_e[:-1] ** 2)
    total = float(np.sum(ring[:, None] * (n_z * np.diff(z_e))[None, :]))
    assert abs(e["w"].sum() - total) <= 1e-12 * total
    ion = sim.species(1)
    assert np.array_equal(ion["r"], e["r"]) and np.array_equal(ion["w"], e["w"])
    assert np.all(ion["vr"] == 0)
    sd = np.std(e["vz"])
    assert abs(sd / math.sqrt(dp.t_ev * W.EL_CHARGE / W.EL_MASS) - 1) < 0.02
    sim.close()


def test_large_case_fp32_resorted_against_fp64():
    wl = small_large()
    g32 = api.from_workload(wl, precision="fp32")
    g64 = api.from_workload(wl, precision="fp64", sort_interval=0)
    g32.set_timing(True)
    for g in (g32, g64):
        g.mark_initial_charge()
        g.step(30)
        g.sync()
    assert g32.timing()["ms_sort"] > 0  # steps 0, 10 and 20 re-sorted
    d32, d64 = g32.diagnostics(), g64.diagnostics()
    assert abs(d32["field_energy"] - d64["field_energy"]) <= 1e-3 * d64["field_energy"]
    assert d32["gauss_residual"] <= 1e-5 * d32["gauss_norm"]
    assert d64["gauss_residual"] <= 1e-5 * d64["gauss_norm"]
    g32.close()
    g64.close()
