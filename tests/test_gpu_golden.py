"""The GPU step against the upstream's own golden smoke frames
(test/functional/true_data, frame 4 = 21 steps of the smoke template:
255 x 2047 nodes, 2 x 1e5 upstream-initialised plasma particles, a
1e6-slot bunch; fixture tests/golden/smoke_frame4.npz).  The particles are
initialised by the upstream code itself (oracle/_ref, TESTMODE sequences),
then stepped on the GPU through the C ABI.

* FP64 plain form: every E, H, J component and the bunch charge density at
  the golden files' 6 significant digits (the oracle's pin).
* FP32 cell-local form: the same frames within 1e-3 of each component's
  largest magnitude.
"""
import numpy as np
import pytest

from helpers import GOLDEN, SMOKE, golden_match, recover_weights
from oracle import refsim
from pdp3_b200 import api

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refsim.available("boris"),
                                 reason="oracle/_ref not built (needs the upstream sources)")]

FIELDS = ["E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "J_r", "J_phi", "J_z"]


def smoke_sim(precision):
    ref = refsim.RefSim(SMOKE["r_size"], SMOKE["z_size"], SMOKE["n_grid_r"], SMOKE["n_grid_z"],
                        SMOKE["dt"], end_time=SMOKE["end_time"], pusher="boris")
    sim = api.Simulation(SMOKE["r_size"], SMOKE["z_size"], SMOKE["n_grid_r"], SMOKE["n_grid_z"],
                         SMOKE["dt"], pusher="boris", precision=precision)
    for idx, (name, c, m, n, nl, nrt, t) in enumerate(SMOKE["species"]):
        ref.add_species_upstream_init(name, c, m, n, nl, nrt, t)
        s = ref.species(idx)
        w = recover_weights(s["q"], s["m"], c * 1.6e-19, m * 9.1e-31)
        assert not np.isnan(w).any()
        sim.add_species(c, m, s["r"], s["z"], s["vr"], s["vphi"], s["vz"], w)
    b = SMOKE["beam"]
    sim.add_bunch(b["charge_e"], b["mass_me"], b["number_macro"],
                  b["bunch_length"] / b["velocity"], b["radius"], b["density"], b["velocity"],
                  0, b["bunches_distance"] / b["velocity"])
    return sim


def test_fp64_gpu_reproduces_golden_smoke_frames():
    g = np.load(GOLDEN)
    sim = smoke_sim("fp64")
    sim.step(21)
    sim.sync()
    for comp in FIELDS:
        r0, z0, r1, z1 = g[comp + "__box"]
        ok = golden_match(sim.field(comp)[r0:r1, z0:z1], g[comp])
        assert ok.all(), (comp, int((~ok).sum()))
    r0, z0, r1, z1 = g["rho_beam__box"]
    ok = golden_match(sim.charge_density(1 << 2)[r0:r1, z0:z1], g["rho_beam"])
    assert ok.all()
    sim.close()


def test_fp32_gpu_tracks_golden_smoke_frames():
    g = np.load(GOLDEN)
    sim = smoke_sim("fp32")
    sim.step(21)
    sim.sync()
    for comp in FIELDS:
        r0, z0, r1, z1 = g[comp + "__box"]
        got, want = sim.field(comp)[r0:r1, z0:z1], g[comp].astype(np.float64)
        scale = np.abs(want).max()
        assert scale > 0, comp
        assert np.abs(got - want).max() <= 1e-3 * scale, (comp, np.abs(got - want).max() / scale)
    sim.close()
