"""Edge sizes and orderings of the FP32 cell-local particle phase.

The kernel stages 128 particles per warp, 4 consecutive per lane, and keeps
running sums of the deposits of a lane's particles.  A particle's own step
(gather, push, moves) does not depend on where it sits in its array, so:

* Sizes that leave partial lane groups and partial warp chunks (1, 3, 127,
  128, 129, 1023, 1025 electrons): every particle's new position and
  momentum equal, bit for bit, those of the same particle stepped as part
  of the full 4096-electron species; from 127 electrons on, the currents
  match the FP64 oracle within 1e-3 of max|J| (at the FP32 offset
  resolution of ~6e-8 cell a 1 eV electron's ~5e-4-cell displacement
  carries ~1e-4 relative error, more for its slow components, which
  averages down only over many particles).
* Orderings: the species shuffled gives each particle the same result as
  in cell order, bit for bit, and the same currents up to the order of the
  FP32/FP64 additions (1e-6 of max|J|); all electrons in one cell (every
  lane on the same deposit nodes) match the oracle within 1e-3 of max|J|.
"""
import numpy as np
import pytest

from helpers import oracle_from_workload, rel_inf, seed_fields
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

KEYS = ("r", "z", "vr", "vphi", "vz")


def subset(sp, idx):
    return W.SpeciesInit(sp.name, sp.charge_e, sp.mass_me, sp.r[idx], sp.z[idx], sp.vr[idx],
                         sp.vphi[idx], sp.vz[idx], sp.w[idx])


def step_fp32(wl, seed=3):
    gpu = api.from_workload(wl, precision="fp32")
    seed_fields([gpu], (wl.n_grid_r, wl.n_grid_z), seed=seed)
    gpu.step()
    gpu.sync()
    out = {"species": gpu.species(0)}
    for c in ("J_r", "J_phi", "J_z"):
        out[c] = gpu.field(c)
    gpu.close()
    return out


def oracle_currents(wl, seed=3):
    orc = oracle_from_workload(wl)
    seed_fields([orc], (wl.n_grid_r, wl.n_grid_z), seed=seed)
    orc.step()
    return {c: orc.field(c) for c in ("J_r", "J_phi", "J_z")}


def base():
    wl = W.small_config(beam=False, steps=1)
    e = wl.species[0]
    wl.species = [e]
    return wl, e


@pytest.fixture(scope="module")
def full():
    wl, e = base()
    return step_fp32(wl)


@pytest.mark.parametrize("n", [1, 3, 127, 128, 129, 1023, 1025])
def test_ragged_species_sizes(n, full):
    wl, e = base()
    wl.species = [subset(e, np.arange(n))]
    got = step_fp32(wl)
    for k in KEYS:
        assert np.array_equal(got["species"][k], full["species"][k][:n]), (n, k)
    if n >= 100:  # a few particles' currents carry their single rounding
        want = oracle_currents(wl)
        for c in ("J_r", "J_phi", "J_z"):
            assert rel_inf(got[c], want[c]) <= 1e-3, (n, c)
    else:
        assert all(np.abs(got[c]).max() > 0 for c in ("J_r", "J_phi", "J_z"))


@pytest.mark.parametrize("order", ["shuffled", "one_cell"])
def test_orderings(order, full):
    wl, e = base()
    rng = np.random.default_rng(11)
    if order == "shuffled":
        perm = rng.permutation(e.n)
        wl.species = [subset(e, perm)]
        got = step_fp32(wl)
        for k in KEYS:
            assert np.array_equal(got["species"][k], full["species"][k][perm]), k
        for c in ("J_r", "J_phi", "J_z"):
            assert rel_inf(got[c], full[c]) <= 1e-6, c
    else:
        # every electron inside cell (5, 9), momenta kept
        r = (5 + rng.uniform(0.05, 0.95, e.n)) * wl.dr
        z = (9 + rng.uniform(0.05, 0.95, e.n)) * wl.dz
        wl.species = [W.SpeciesInit(e.name, e.charge_e, e.mass_me, r, z, e.vr, e.vphi, e.vz,
                                    e.w)]
        got = step_fp32(wl)
        want = oracle_currents(wl)
        for c in ("J_r", "J_phi", "J_z"):
            assert rel_inf(got[c], want[c]) <= 1e-3, c
