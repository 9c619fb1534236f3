"""GPU checks of the FP32 cell-local form against the FP64 oracle and the
FP64 GPU form.

Stated tolerances (FP32 state and arithmetic, FP64 grid accumulation):
  * one step from seeded fields: particle positions within 1e-5 cell of the
    oracle's, momenta within 1e-5 of the largest, J within 1e-4 of max|J|
    (FP32 rounding of offsets, momenta and per-particle deposits);
  * Gauss law: relative residual <= 1e-5 after 100 steps (no absorbing
    layer), the deposition being charge-conserving up to FP32 rounding;
  * wake case (driven bunch) over 300 steps: total field energy within 1e-3
    of the FP64 GPU form, kinetic energy within 1e-3.
"""
import numpy as np
import pytest

from helpers import GRIDS, oracle_from_workload, rel_inf, seed_fields
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_grid_z", [33, 41])
def test_fp32_one_step_small_vs_oracle(n_grid_z):
    """32 cells per radial row (the cell index splits by a shift) and 40
    (by a division)."""
    wl = W.small_config(beam=True, steps=1, n_grid_z=n_grid_z, z_size=0.04 * (n_grid_z - 1) / 32)
    orc = oracle_from_workload(wl)
    gpu = api.from_workload(wl, precision="fp32")
    seed_fields([orc, gpu], (wl.n_grid_r, wl.n_grid_z), seed=3)
    # the bunch is injected at the start of the step: run it once to get live bunch particles
    orc.step()
    gpu.step()
    gpu.sync()
    for c in ("J_r", "J_phi", "J_z"):
        assert rel_inf(gpu.field(c), orc.field(c)) <= 1e-4, c
    for c in ("E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z"):
        assert rel_inf(gpu.field(c), orc.field(c)) <= 1e-4, c
    for sid in range(3):
        a, b = gpu.species(sid), orc.species(sid)
        assert np.array_equal(a["alive"], b["alive"])
        m = b["alive"].astype(bool)
        if not m.any():
            continue
        assert np.abs(a["r"][m] - b["r"][m]).max() <= 1e-5 * wl.dr
        assert np.abs(a["z"][m] - b["z"][m]).max() <= 1e-5 * wl.dz
        for k in ("vr", "vphi", "vz"):
            scale = max(float(np.abs(b[k][m]).max()), 1.0)
            assert np.abs(a[k][m] - b[k][m]).max() <= 1e-5 * scale, (sid, k)


@pytest.mark.parametrize("pusher", ["vay", "boris_classic"])
def test_fp32_one_step_other_pushers(pusher):
    wl = W.small_config(beam=False, steps=1, pusher=pusher)
    orc = oracle_from_workload(wl)
    gpu = api.from_workload(wl, precision="fp32")
    seed_fields([orc, gpu], (wl.n_grid_r, wl.n_grid_z), seed=5)
    orc.step()
    gpu.step()
    gpu.sync()
    for c in ("J_r", "J_phi", "J_z"):
        assert rel_inf(gpu.field(c), orc.field(c)) <= 1e-4, c
    a, b = gpu.species(0), orc.species(0)
    assert np.abs(a["r"] - b["r"]).max() <= 1e-5 * wl.dr
    scale = float(np.abs(b["vz"]).max())
    assert np.abs(a["vz"] - b["vz"]).max() <= 1e-5 * scale


def test_fp32_gauss_law_holds():
    wl = W.thermal_config(steps=100, ppc=4)
    wl.pml = None
    gpu = api.from_workload(wl, precision="fp32")
    gpu.mark_initial_charge()
    gpu.step(100)
    gpu.sync()
    d = gpu.diagnostics()
    assert d["gauss_norm"] > 0
    assert d["gauss_residual"] <= 1e-5 * d["gauss_norm"], d


def test_fp32_tracks_fp64_on_driven_wake():
    wl = W.wake_config(n_grid_r=65, n_grid_z=513, r_size=0.025, z_size=0.2, ppc=4,
                       beam_radius=2.5e-3, beam_length=0.01)
    g64 = api.from_workload(wl, precision="fp64")
    g32 = api.from_workload(wl, precision="fp32")
    for g in (g64, g32):
        g.mark_initial_charge()
        g.step(300)
        g.sync()
    d64, d32 = g64.diagnostics(), g32.diagnostics()
    assert d64["field_energy"] > 0
    assert abs(d32["field_energy"] - d64["field_energy"]) <= 1e-3 * d64["field_energy"], (d32, d64)
    assert abs(d32["kinetic_energy"] - d64["kinetic_energy"]) <= 1e-3 * d64["kinetic_energy"]
    assert d32["alive"] == d64["alive"]
