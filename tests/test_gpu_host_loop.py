"""The C++ host layer with the upstream class interfaces (pdp3_b200/host):
pdp3g_loop runs LoadInitParam::run's call sequence (init_beam,
HField::calc_field, Current::reset_j, ParticlesList::step_v and
full_current_distribution, EField::calc_field, t += dt) through those
classes; its result must match the same workload stepped through the C ABI
directly and the oracle (FP64, 1e-12 of max|x| per grid)."""
import os
import subprocess

import numpy as np
import pytest

from helpers import GRIDS, oracle_from_workload, rel_inf
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LOOP = os.path.join(os.path.dirname(HERE), "pdp3_b200", "pdp3g_loop")


def write_case(wl, d, precision=0):
    os.makedirs(d, exist_ok=True)
    pml = wl.pml or [0.0] * 5
    kv = {"r_size": wl.r_size, "z_size": wl.z_size, "n_grid_r": wl.n_grid_r,
          "n_grid_z": wl.n_grid_z, "dt": wl.dt, "current_time": 0.0, "pml_l1": pml[0],
          "pml_l2": pml[1], "pml_l3": pml[2], "pml_sigma1": pml[3], "pml_sigma2": pml[4],
          "pusher": api.PUSHERS[wl.pusher], "precision": precision,
          "n_species": len(wl.species)}
    for i, s in enumerate(wl.species):
        kv["species%d_charge" % i] = s.charge_e
        kv["species%d_mass" % i] = s.mass_me
        kv["species%d_n" % i] = s.n
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            np.ascontiguousarray(getattr(s, name), dtype=np.float64).tofile(
                os.path.join(d, "species%d_%s.f64" % (i, name)))
    if wl.beam is not None:
        b = wl.beam
        kv.update({"beam_charge": b.charge_e, "beam_mass": b.mass_me,
                   "beam_number_macro": b.number_macro, "beam_length": b.bunch_length,
                   "beam_radius": b.radius, "beam_density": b.density,
                   "beam_velocity": b.velocity, "beam_number_bunches": b.number_bunches,
                   "beam_distance": b.bunches_distance})
    with open(os.path.join(d, "case.txt"), "w") as f:
        for k, v in kv.items():
            f.write("%s %.17g\n" % (k, v))


def test_cpp_class_loop_matches_c_abi_and_oracle(tmp_path):
    if not os.path.exists(LOOP):
        pytest.fail("pdp3g_loop is not built (python -m pdp3_b200.build)")
    wl = W.small_config(beam=True, steps=12)
    case, out = str(tmp_path / "case"), str(tmp_path / "out")
    os.makedirs(out)
    write_case(wl, case)
    res = subprocess.run([LOOP, case, "12", out], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    sim = api.from_workload(wl)
    sim.step(12)
    sim.sync()
    orc = oracle_from_workload(wl)
    for _ in range(12):
        orc.step()
    n = wl.n_grid_r * wl.n_grid_z
    for c in ("E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "J_r", "J_phi", "J_z"):
        host = np.fromfile(os.path.join(out, c + ".f64"), dtype=np.float64, count=n)
        host = host.reshape(wl.n_grid_r, wl.n_grid_z)
        assert rel_inf(host, sim.field(c)) <= 1e-12, c
        assert rel_inf(host, orc.field(c)) <= 1e-9, c
    for sid in range(3):
        alive = np.fromfile(os.path.join(out, "out%d_alive.u8" % sid), dtype=np.uint8)
        assert np.array_equal(alive, sim.species(sid)["alive"])
        r = np.fromfile(os.path.join(out, "out%d_r.f64" % sid), dtype=np.float64)
        m = alive.astype(bool)
        assert np.abs(r[m] - sim.species(sid)["r"][m]).max() <= 1e-12 * wl.r_size
