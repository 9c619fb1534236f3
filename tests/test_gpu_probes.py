"""Probe output (ProbePlain, src/probePlain.cpp; LoadInitParam::dump_data).

* pdp3g_probe_read: frame, col, row and dot regions of a component equal the
  same slices of the full grid; rho_beam equals the bunch's charge weighting.
* pdp3g_probe_particles: the slots of a species inside a cell region, in slot
  order, with the upstream's inclusive bounds and CELL_NUMBER, dead slots
  included (both precisions).
* pdp3g_temperature / pdp3g_density and the T / density probes:
  TemperatureClassic and ParticlesDensity of each species equal the oracle's
  restatements on the same particles (empty cells NaN at the same places; the
  sums' order differs only by the device atomics).
* The upstream run itself: the smoke template (upstream-initialised
  particles, 21 steps) driven by the C++ class layer (pdp3g_loop) with frame
  probes on dump_data's schedule writes <component>/frame_*/4.dat and
  T/<specie>/frame_*/4.dat files whose values are the golden frames at their
  6 printed digits.
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import GOLDEN, SMOKE, golden_match, recover_weights
from oracle.diagnostics import particles_density, temperature_classic
from pdp3_b200 import api
from pdp3_b200 import workloads as W
from test_gpu_host_loop import LOOP, write_case

pytestmark = pytest.mark.gpu

FIELDS = ["E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "J_r", "J_phi", "J_z"]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_probe_regions_and_particles(precision):
    wl = W.small_config(beam=True, steps=6)
    sim = api.from_workload(wl, precision=precision)
    sim.step(6)
    sim.sync()
    ez = sim.field("E_z")
    assert np.array_equal(sim.probe("E_z", "frame", 2, 3, 9, 20), ez[2:9, 3:20].ravel())
    assert np.array_equal(sim.probe("E_z", "col", 1, 7, 12), ez[1:12, 7])
    assert np.array_equal(sim.probe("E_z", "row", 4, 2, 0, 30), ez[4, 2:30])
    assert np.array_equal(sim.probe("E_z", "dot", 5, 6), ez[5:6, 6])
    rho_b = sim.charge_density(1 << 2)
    assert np.allclose(sim.probe("rho_beam", "frame", 0, 0, wl.n_grid_r, wl.n_grid_z),
                       rho_b.ravel(), rtol=1e-12, atol=1e-12 * np.abs(rho_b).max())
    for sid, box in ((0, (2, 3, 6, 12)), (2, (0, 0, 5, 8))):
        sp = sim.species(sid)
        i = np.ceil(sp["r"] / wl.dr).astype(np.int64) - 1
        k = np.ceil(sp["z"] / wl.dz).astype(np.int64) - 1
        r0, z0, r1, z1 = box
        sel = (i >= r0) & (i <= r1) & (k >= z0) & (k <= z1)
        got = sim.probe_particles(sid, r0, z0, r1, z1)
        assert sel.sum() > 0
        assert got["r"].size == sel.sum()
        for key in ("r", "z", "vr", "vphi", "vz"):
            assert np.array_equal(got[key], sp[key][sel]), (sid, key)
    sim.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_species_diagnostics_match_oracle(precision):
    wl = W.small_config(beam=True, steps=6)
    sim = api.from_workload(wl, precision=precision)
    sim.step(6)
    sim.sync()
    masses = [s.mass_me * 9.1e-31 for s in wl.species] + [wl.beam.mass_me * 9.1e-31]
    charges = [s.charge_e * 1.6e-19 for s in wl.species] + [wl.beam.charge_e * 1.6e-19]
    for sid in range(3):
        sp = sim.species(sid)
        ref, rnd = temperature_classic(sp["r"], sp["z"], sp["vr"], sp["vphi"], sp["vz"], wl.dr,
                                       wl.dz, wl.n_grid_r, wl.n_grid_z, masses[sid],
                                       charges[sid], rounding=True)
        got = sim.temperature(sid)
        t = got[:-1, :-1]
        assert np.array_equal(np.isnan(t), np.isnan(ref)), sid
        fin = ~np.isnan(ref)
        assert fin.sum() > 3, sid  # the bunch has entered a few cells
        # the device sums in atomic order: T within the order's rounding
        # bound (for the mono-energetic bunch T is that rounding alone)
        tol = 1e-12 * np.abs(ref[fin]).max() + rnd[fin]
        assert np.all(np.abs(t[fin] - ref[fin]) <= tol), sid
        if sid < 2:  # the thermal plasma: T far above its rounding
            assert np.median(rnd[fin] / np.abs(ref[fin])) < 1e-10
        # the probe recomputes the same grid and returns its region in write
        # order
        pr = sim.probe_species("T", sid, "frame", 1, 2, 7, 11)
        want = got[1:7, 2:11].ravel()
        assert np.array_equal(np.isnan(pr), np.isnan(want)), sid
        f = ~np.isnan(want)
        tol = 1e-12 * np.abs(ref[fin]).max() + 2 * rnd[1:7, 2:11].ravel()[f]
        assert np.all(np.abs(pr[f] - want[f]) <= tol), sid
        # ParticlesDensity: sums of positive terms, order rounding only
        dref = particles_density(sp["r"], sp["z"], masses[sid] * sp["w"], wl.dr, wl.dz,
                                 wl.n_grid_r, wl.n_grid_z)
        dens = sim.density(sid)
        assert (dref > 0).sum() > 3, sid
        assert np.abs(dens - dref).max() <= 1e-12 * dref.max(), sid
        pd = sim.probe_species("density", sid, "col", 0, 3, wl.n_grid_r, 0)
        assert np.abs(pd - dref[:, 3]).max() <= 1e-12 * dref.max(), sid
    sim.close()


def smoke_workload():
    from oracle import refsim
    ref = refsim.RefSim(SMOKE["r_size"], SMOKE["z_size"], SMOKE["n_grid_r"], SMOKE["n_grid_z"],
                        SMOKE["dt"], end_time=SMOKE["end_time"], pusher="boris")
    species = []
    for idx, (name, c, m, n, nl, nrt, t) in enumerate(SMOKE["species"]):
        ref.add_species_upstream_init(name, c, m, n, nl, nrt, t)
        s = ref.species(idx)
        w = recover_weights(s["q"], s["m"], c * 1.6e-19, m * 9.1e-31)
        species.append(W.SpeciesInit(name, c, m, s["r"], s["z"], s["vr"], s["vphi"], s["vz"], w))
    b = SMOKE["beam"]
    beam = W.BeamInit(b["charge_e"], b["mass_me"], b["number_macro"], b["bunch_length"],
                      b["radius"], b["density"], b["velocity"], b["number_bunches"],
                      b["bunches_distance"])
    return W.Workload("smoke", SMOKE["r_size"], SMOKE["z_size"], SMOKE["n_grid_r"],
                      SMOKE["n_grid_z"], SMOKE["dt"], 21, None, "boris", species, beam)


def test_cpp_loop_probes_reproduce_golden_smoke_frames(tmp_path):
    from oracle import refsim
    if not refsim.available("boris"):
        pytest.skip("oracle/_ref not built (needs the upstream sources)")
    if not os.path.exists(LOOP):
        pytest.fail("pdp3g_loop is not built (python -m pdp3_b200.build)")
    g = np.load(GOLDEN)
    wl = smoke_workload()
    case, out = str(tmp_path / "case"), str(tmp_path / "out")
    os.makedirs(out)
    write_case(wl, case)
    comps = FIELDS + ["rho_beam"]
    names = [sp[0] for sp in SMOKE["species"]]
    with open(os.path.join(case, "names.txt"), "w") as f:
        f.write("\n".join(names) + "\n")
    with open(os.path.join(case, "probes.txt"), "w") as f:
        for c in comps:
            r0, z0, r1, z1 = g[c + "__box"]
            f.write("0 %s %d %d %d %d 5\n" % (c, r0, z0, r1, z1))
        for n in names:
            r0, z0, r1, z1 = g["T_%s__box" % n]
            f.write("0 T %d %d %d %d 5 %s\n" % (r0, z0, r1, z1, n))
        f.write("0 density 100 100 150 150 5 Electrons\n")
    res = subprocess.run([LOOP, case, "21", out], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    for c in comps + ["T/" + n for n in names]:
        key = c.replace("/", "_")
        r0, z0, r1, z1 = (int(x) for x in g[key + "__box"])
        path = os.path.join(out, "probes", c, "frame_%d:%d_%d:%d" % (r0, z0, r1, z1), "4.dat")
        vals = np.array(open(path).read().split(), dtype=np.float64)
        assert vals.size == (r1 - r0) * (z1 - z0), c
        vals = vals.reshape(r1 - r0, z1 - z0)
        gold = g[key]
        assert np.array_equal(np.isnan(vals), np.isnan(gold)), c
        fin = ~np.isnan(gold)
        ok = golden_match(vals[fin], gold[fin])
        assert ok.all(), (c, int((~ok).sum()))
        # the five dumps so far (steps 1, 6, 11, 16, 21) each wrote one file
        assert sorted(os.listdir(os.path.dirname(path))) == ["%d.dat" % i for i in range(5)]
    # the density probe (no golden frame): the oracle's ParticlesDensity of
    # the electrons the loop wrote after step 21, the state of the last dump
    n = wl.species[0].n
    fin = {k: np.fromfile(os.path.join(out, "out0_%s.f64" % k), dtype=np.float64, count=n)
           for k in ("r", "z")}
    dref = particles_density(fin["r"], fin["z"], 9.1e-31 * wl.species[0].w, wl.dr, wl.dz,
                             wl.n_grid_r, wl.n_grid_z)[100:150, 100:150]
    path = os.path.join(out, "probes", "density", "Electrons", "frame_100:100_150:150", "4.dat")
    vals = np.array(open(path).read().split(), dtype=np.float64).reshape(50, 50)
    assert golden_match(vals, dref).all()
    assert (dref > 0).sum() > 1000
