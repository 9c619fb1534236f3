"""The upstream's initial plasma state generated on the device
(pdp3g_add_species_upstream: Particles + load_cylindrical_spatial_distribution
+ velocity_distribution with TESTMODE sequences) against the upstream code
itself (oracle/_ref, ref_add_species_upstream_init).

* Positions and weights bit for bit: flat and ramped densities, a left plasma
  boundary of 0 as init_particles passes it.
* Velocities within 1e-12 of the largest speed: the Maxwell-Juttner branch
  (T >= 0.1, rejection sampling), the classical branch (0 < T < 0.1) and a
  cold species (T = 0, all velocities zero).
* The whole upstream smoke run from its parameters alone: both plasma
  species generated on the device, the bunch injected on the device, 21
  steps; every golden frame at its 6 printed digits, through the C ABI and
  through the C++ class layer (pdp3g_loop with the species given by their
  densities and temperatures, probes on dump_data's schedule).
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN, SMOKE, golden_match
from oracle import refsim
from pdp3_b200 import api
from test_gpu_host_loop import LOOP

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refsim.available("boris"),
                                 reason="oracle/_ref not built (needs the upstream sources)")]

FIELDS = ["E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "J_r", "J_phi", "J_z"]
GEOM = (0.05, 0.2, 65, 257, 1e-12)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("case", [
    ("electrons, ramp, Maxwell-Juttner", -1.0, 1.0, 20000, 2e16, 2.05e16, 1.0),
    ("ions, flat, T = 0.1", 1.0, 1836.0, 20000, 1e16, 1e16, 0.1),
    ("electrons, ramp, classical", -1.0, 1.0, 5000, 1e16, 3e16, 0.05),
    ("cold ions", 1.0, 1836.0, 3000, 1e17, 1e17, 0.0),
])
def test_upstream_init_matches_reference(case, precision):
    name, c, m, n, nl, nrt, t = case
    ref = refsim.RefSim(*GEOM)
    ref.add_species_upstream_init("s", c, m, n, nl, nrt, t)
    want = ref.species(0)
    sim = api.Simulation(*GEOM, precision=precision)
    sid = sim.add_species_upstream(c, m, n, nl, nrt, t)
    got = sim.species(sid)
    if precision == "fp64":
        for k in ("r", "z"):
            assert np.array_equal(got[k], want[k]), (name, k)
        # charge_array = charge * n_per_macro, mass_array = mass * n_per_macro
        assert np.array_equal(c * 1.6e-19 * got["w"], want["q"]), name
        assert np.array_equal(m * 9.1e-31 * got["w"], want["m"]), name
        vtol = 1e-12
    else:
        # the cell-local form stores offsets, momenta and weights in FP32
        for k in ("r", "z"):
            assert np.abs(got[k] - want[k]).max() <= 1e-6 * np.abs(want[k]).max(), (name, k)
        w_ref = want["q"] / (c * 1.6e-19)
        assert np.abs(got["w"] - w_ref).max() <= 1e-6 * w_ref.max(), name
        vtol = 2e-7
    vmax = max(np.abs(want[k]).max() for k in ("vr", "vphi", "vz"))
    if t == 0:
        assert vmax == 0
        for k in ("vr", "vphi", "vz"):
            assert not got[k].any(), (name, k)
    else:
        assert vmax > 0
        for k in ("vr", "vphi", "vz"):
            err = np.abs(got[k] - want[k]).max() / vmax
            assert err <= vtol, (name, k, err)
    assert got["alive"].all()
    sim.close()
    ref.close()


def test_device_initialised_smoke_reproduces_golden_frames():
    g = np.load(GOLDEN)
    sim = api.Simulation(SMOKE["r_size"], SMOKE["z_size"], SMOKE["n_grid_r"], SMOKE["n_grid_z"],
                         SMOKE["dt"], pusher="boris")
    for (name, c, m, n, nl, nrt, t) in SMOKE["species"]:
        sim.add_species_upstream(c, m, n, nl, nrt, t)
    b = SMOKE["beam"]
    sim.add_bunch(b["charge_e"], b["mass_me"], b["number_macro"],
                  b["bunch_length"] / b["velocity"], b["radius"], b["density"], b["velocity"],
                  0, b["bunches_distance"] / b["velocity"])
    sim.step(21)
    sim.sync()
    for comp in FIELDS:
        r0, z0, r1, z1 = g[comp + "__box"]
        ok = golden_match(sim.field(comp)[r0:r1, z0:z1], g[comp])
        assert ok.all(), (comp, int((~ok).sum()))
    r0, z0, r1, z1 = g["rho_beam__box"]
    assert golden_match(sim.charge_density(1 << 2)[r0:r1, z0:z1], g["rho_beam"]).all()
    for idx, (name, *_rest) in enumerate(SMOKE["species"]):
        t = sim.temperature(idx)
        r0, z0, r1, z1 = g["T_%s__box" % name]
        got, gold = t[r0:r1, z0:z1], g["T_" + name]
        assert np.array_equal(np.isnan(got), np.isnan(gold)), name
        fin = ~np.isnan(gold)
        assert golden_match(got[fin], gold[fin]).all(), name
    sim.close()


def test_upstream_init_rejects_bad_arguments():
    sim = api.Simulation(*GEOM)
    with pytest.raises(api.Pdp3gError):
        sim.add_species_upstream(-1.0, 1.0, 0, 1e16, 1e16, 1.0)
    with pytest.raises(api.Pdp3gError):
        sim.add_species_upstream(-1.0, 1.0, 1 << 30, 1e16, 1e16, 1.0)
    with pytest.raises(api.Pdp3gError):
        sim.add_species_upstream(-1.0, 1.0, 100, 1e16, 1e16, -1.0)
    sim.close()


def test_cpp_loop_from_parameters_reproduces_golden_frames(tmp_path):
    if not os.path.exists(LOOP):
        pytest.fail("pdp3g_loop is not built (python -m pdp3_b200.build)")
    g = np.load(GOLDEN)
    case, out = tmp_path / "case", tmp_path / "out"
    case.mkdir()
    out.mkdir()
    b = SMOKE["beam"]
    kv = {"r_size": SMOKE["r_size"], "z_size": SMOKE["z_size"], "n_grid_r": SMOKE["n_grid_r"],
          "n_grid_z": SMOKE["n_grid_z"], "dt": SMOKE["dt"], "current_time": 0.0,
          "pusher": api.PUSHERS["boris"], "precision": 0,
          "n_species": len(SMOKE["species"]),
          "beam_charge": b["charge_e"], "beam_mass": b["mass_me"],
          "beam_number_macro": b["number_macro"], "beam_length": b["bunch_length"],
          "beam_radius": b["radius"], "beam_density": b["density"],
          "beam_velocity": b["velocity"], "beam_number_bunches": b["number_bunches"],
          "beam_distance": b["bunches_distance"]}
    names = []
    for i, (name, c, m, n, nl, nrt, t) in enumerate(SMOKE["species"]):
        names.append(name)
        kv.update({"species%d_charge" % i: c, "species%d_mass" % i: m, "species%d_n" % i: n,
                   "species%d_left_density" % i: nl, "species%d_right_density" % i: nrt,
                   "species%d_temperature" % i: t})
    (case / "case.txt").write_text("".join("%s %.17g\n" % kv_ for kv_ in kv.items()))
    (case / "names.txt").write_text("\n".join(names) + "\n")
    comps = FIELDS + ["rho_beam"]
    lines = []
    for c in comps:
        r0, z0, r1, z1 = g[c + "__box"]
        lines.append("0 %s %d %d %d %d 5" % (c, r0, z0, r1, z1))
    for n in names:
        r0, z0, r1, z1 = g["T_%s__box" % n]
        lines.append("0 T %d %d %d %d 5 %s" % (r0, z0, r1, z1, n))
    (case / "probes.txt").write_text("\n".join(lines) + "\n")
    res = subprocess.run([LOOP, str(case), "21", str(out)], capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stderr
    for c in comps + ["T/" + n for n in names]:
        key = c.replace("/", "_")
        r0, z0, r1, z1 = (int(x) for x in g[key + "__box"])
        path = out / "probes" / c / ("frame_%d:%d_%d:%d" % (r0, z0, r1, z1)) / "4.dat"
        vals = np.array(path.read_text().split(), dtype=np.float64).reshape(r1 - r0, z1 - z0)
        gold = g[key]
        assert np.array_equal(np.isnan(vals), np.isnan(gold)), c
        fin = ~np.isnan(gold)
        assert golden_match(vals[fin], gold[fin]).all(), c
