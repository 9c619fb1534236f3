"""GPU parity of the FP64 plain form (and, within FP32 rounding, of the FP32
cell-local form) against the oracle on the benchmarked grids, through the
C ABI.

The wake grid (257 x 2049 nodes over 0.1 x 0.8 m, gamma = 5 bunch injected
at z = 0, 10-cell absorbing layer) and the large grid (513 x 4097 nodes,
density ramped over the first 20 % of z, gamma = 10 bunch, Vay pusher,
particles re-sorted by cell every 20 steps) are run at 2 macroparticles per
cell and species instead of 64, so that the oracle steps them in seconds;
grid, time step, layer, bunch and pusher are those of the full cases.

Tolerances (FP64):
  * one step from seeded fields: every grid within 1e-12 of the oracle's
    max|x| per array (J is summed with atomics in another order), every
    particle array within 1e-12 relative, alive flags identical;
  * 20 steps with injection: alive flags identical (integer outcome of the
    injection schedule), time bit-identical, grids and particle arrays
    within 1e-9 (rounding differences grow through the coupled update).
Tolerances (FP32 form, one step): E and H within 2e-4 of max|x|, J within
5e-3 of max|J| (FP32 position resolution against thermal moves), positions
within 1e-6 of a cell, alive flags identical.
"""
import numpy as np
import pytest

from helpers import GRIDS, oracle_from_workload, rel_inf, seed_fields
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

PPC = 2


def compare_particles(gpu, orc, sid, tol):
    a, b = gpu.species(sid), orc.species(sid)
    assert np.array_equal(a["alive"], b["alive"]), sid
    m = b["alive"].astype(bool)
    assert m.any(), sid
    for k in ("r", "z", "vr", "vphi", "vz"):
        scale = max(float(np.abs(b[k][m]).max()), 1e-300)
        err = float(np.abs(a[k][m] - b[k][m]).max()) / scale
        assert err <= tol, (sid, k, err)


def compare_grids(gpu, orc, tol):
    for c in GRIDS:
        err = rel_inf(gpu.field(c), orc.field(c))
        assert err <= tol, (c, err)


def cell_keys(r, z, wl):
    """CELL_NUMBER of r and z (src/geometry.h:33-44) as the sort's key."""
    i = np.clip(np.ceil(r / wl.dr).astype(np.int64) - 1, 0, wl.n_grid_r - 2)
    k = np.clip(np.ceil(z / wl.dz).astype(np.int64) - 1, 0, wl.n_grid_z - 2)
    return i * (wl.n_grid_z - 1) + k


def permute_species(wl, perms):
    for s, p in zip(wl.species, perms):
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            setattr(s, name, getattr(s, name)[p].copy())


def test_wake_grid_one_step_parity():
    """256 x 2048 cells, gamma = 5 bunch: the first step injects the first
    slice of the bunch at z = dz/2 + v dt U (src/bunch.cpp:87-124)."""
    wl = W.wake_config(ppc=PPC, steps=1)
    assert (wl.n_grid_r, wl.n_grid_z) == (257, 2049)
    orc = oracle_from_workload(wl)
    gpu = api.from_workload(wl)
    seed_fields([orc, gpu], (wl.n_grid_r, wl.n_grid_z), seed=31)
    orc.step()
    gpu.step()
    gpu.sync()
    compare_grids(gpu, orc, 1e-12)
    for sid in range(3):
        compare_particles(gpu, orc, sid, 1e-12)
    assert gpu.species(2)["alive"].sum() > 0
    gpu.close()


def test_wake_grid_20_steps_with_injection():
    wl = W.wake_config(ppc=PPC, steps=20)
    orc = oracle_from_workload(wl)
    gpu = api.from_workload(wl)
    for _ in range(20):
        orc.step()
    gpu.step(20)
    gpu.sync()
    assert gpu.time == orc.time
    alive_g, alive_o = gpu.species(2)["alive"], orc.species(2)["alive"]
    assert alive_o.sum() > 0
    assert np.array_equal(alive_g, alive_o)
    compare_grids(gpu, orc, 1e-9)
    for sid in range(3):
        compare_particles(gpu, orc, sid, 1e-9)
    gpu.close()


def test_large_grid_one_step_parity_vay_after_resort():
    """512 x 4096 cells, ramped density, gamma = 10 bunch, Vay pusher
    (src/particles.cpp:1152-1254), re-sort interval 20.  The plasma is handed
    over in a shuffled order; the GPU step sorts it by cell before the push
    (step 0 is a sort step), and the oracle is given the same particles in
    numpy's stable argsort order of the cell keys: after one step every
    particle must sit in the same slot on both sides."""
    wl = W.large_config(ppc=PPC, steps=1, host_plasma=True)
    assert (wl.n_grid_r, wl.n_grid_z) == (513, 4097) and wl.pusher == "vay"
    assert wl.sort_interval == 20
    rng = np.random.default_rng(33)
    permute_species(wl, [rng.permutation(s.n) for s in wl.species])
    gpu = api.from_workload(wl)
    perms = [np.argsort(cell_keys(s.r, s.z, wl), kind="stable") for s in wl.species]
    permute_species(wl, perms)
    orc = oracle_from_workload(wl)
    seed_fields([orc, gpu], (wl.n_grid_r, wl.n_grid_z), seed=32)
    orc.step()
    gpu.step()
    gpu.sync()
    compare_grids(gpu, orc, 1e-12)
    for sid in range(3):
        compare_particles(gpu, orc, sid, 1e-12)
    # the weights travel with their particles through the sort
    for sid, s in enumerate(wl.species):
        assert np.array_equal(gpu.species(sid)["w"], s.w), sid
    gpu.close()


def test_species_on_two_streams_sum_like_species_alone():
    """Three plasma species: the particle phase runs every second species on
    a side stream between a fork and a join event.  J after the step must
    equal the sum of the J each species deposits in a context of its own
    (one stream), within the atomic summation order (1e-12 of max|J|)."""
    wl = W.small_config(n_grid_r=33, n_grid_z=129, r_size=0.02, z_size=0.16, ppc=8)
    el, ion = wl.species
    el2 = W.SpeciesInit("Electrons2", -1.0, 1.0, el.r.copy(), el.z.copy(), -el.vr, el.vphi,
                        0.5 * el.vz, el.w.copy())
    wl.species = [el, ion, el2]
    together = api.from_workload(wl)
    seed_fields([together], (wl.n_grid_r, wl.n_grid_z), seed=34)
    together.step()
    together.sync()
    total = {c: np.zeros((wl.n_grid_r, wl.n_grid_z)) for c in ("J_r", "J_phi", "J_z")}
    species = wl.species
    for s in species:
        wl.species = [s]
        alone = api.from_workload(wl)
        seed_fields([alone], (wl.n_grid_r, wl.n_grid_z), seed=34)
        alone.step()
        alone.sync()
        for c in total:
            total[c] += alone.field(c)
        alone.close()
    for c in total:
        assert np.abs(total[c]).max() > 0, c
        assert rel_inf(together.field(c), total[c]) <= 1e-12, c
    together.close()


@pytest.mark.parametrize("case", ["wake", "large"])
def test_fp32_form_one_step_against_the_oracle(case):
    """The FP32 cell-local form on the same grids, particles and seeded
    fields as the FP64 tests above: one step against the oracle's FP64 step.
    Bounds: E and H within 2e-4 of max|x| per grid (measured up to 1.0e-4,
    E_z on the large grid, from the gamma = 10 bunch's current); J within
    5e-3 of max|J| (measured up to 1.8e-3, J_r on the large grid: an FP32
    offset resolves ~6e-8 of a cell against thermal moves of ~5e-4 cell per
    step, and at 2 ppc J_r is a small sum of nearly cancelling deposits);
    positions within 1e-6 of a cell; alive flags identical."""
    if case == "wake":
        wl = W.wake_config(ppc=PPC, steps=1)
        seed = 35
    else:
        wl = W.large_config(ppc=PPC, steps=1, host_plasma=True, sort_interval=0)
        seed = 36
    orc = oracle_from_workload(wl)
    g32 = api.from_workload(wl, precision="fp32")
    seed_fields([orc, g32], (wl.n_grid_r, wl.n_grid_z), seed=seed)
    orc.step()
    g32.step()
    g32.sync()
    for c in ("E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "J_r", "J_phi", "J_z"):
        err = rel_inf(g32.field(c), orc.field(c))
        assert err <= (5e-3 if c[0] == "J" else 2e-4), (case, c, err)
    for sid in range(3):
        a, b = g32.species(sid), orc.species(sid)
        assert np.array_equal(a["alive"], b["alive"]), (case, sid)
        m = b["alive"].astype(bool)
        assert float(np.abs(a["r"][m] - b["r"][m]).max()) <= 1e-6 * wl.dr, (case, sid)
        assert float(np.abs(a["z"][m] - b["z"][m]).max()) <= 1e-6 * wl.dz, (case, sid)
    g32.close()
