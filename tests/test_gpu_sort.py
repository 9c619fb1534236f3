"""The integer sort of particles by cell on the GPU.

The permutation must equal numpy's stable argsort of the cell keys exactly
(integer work: bit-exact), for both particle layouts, and sorting must not
change the physics beyond summation order (the FP64 step from a sorted
state matches the oracle stepping the same permuted particles).
"""
import numpy as np
import pytest

from helpers import GRIDS, oracle_from_workload, rel_inf
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu


def cell_keys(r, z, wl):
    i = np.clip(np.ceil(r / wl.dr).astype(np.int64) - 1, 0, wl.n_grid_r - 2)
    k = np.clip(np.ceil(z / wl.dz).astype(np.int64) - 1, 0, wl.n_grid_z - 2)
    return i * (wl.n_grid_z - 1) + k


def shuffled_workload(seed, **kw):
    wl = W.thermal_config(**kw)
    rng = np.random.default_rng(seed)
    for s in wl.species:
        p = rng.permutation(s.n)
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            setattr(s, name, getattr(s, name)[p].copy())
    return wl


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sort_is_the_stable_argsort(precision):
    wl = shuffled_workload(11, ppc=4)
    sim = api.from_workload(wl, precision=precision)
    before = [sim.species(s) for s in range(2)]
    sim.sort()
    sim.sync()
    for sid in range(2):
        b = before[sid]
        keys = cell_keys(b["r"], b["z"], wl)
        perm = np.argsort(keys, kind="stable")
        a = sim.species(sid)
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            assert np.array_equal(a[name], b[name][perm]), (precision, sid, name)


@pytest.mark.parametrize("n", [2, 33, 257, 2049, 10007, 70001])
def test_sort_of_ragged_counts(n):
    """Counts that end inside a 32-item step, a load batch and a warp's
    sub-range: the last items of the tail must land like the rest."""
    wl = shuffled_workload(17, ppc=8)
    for s in wl.species:
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            setattr(s, name, getattr(s, name)[:n].copy())
    for precision in ("fp64", "fp32"):
        sim = api.from_workload(wl, precision=precision)
        before = [sim.species(s) for s in range(2)]
        sim.sort()
        sim.sync()
        for sid in range(2):
            b = before[sid]
            assert b["r"].size == n
            perm = np.argsort(cell_keys(b["r"], b["z"], wl), kind="stable")
            a = sim.species(sid)
            for name in ("r", "z", "vr", "vphi", "vz", "w"):
                assert np.array_equal(a[name], b[name][perm]), (precision, n, sid, name)
        sim.close()


@pytest.mark.parametrize("nodes", [(9, 17), (1025, 8193)])
def test_sort_with_one_and_three_digit_passes(nodes):
    """Key ranges of one 8-bit digit pass (8 x 16 cells, 7-bit keys) and of
    three (1024 x 8192 cells, 23-bit keys); the thermal grid of the other
    tests takes two, the wake and large grids three."""
    nr, nz = nodes
    if nr == 9:
        wl = W.small_config(n_grid_r=nr, n_grid_z=nz, ppc=8)
    else:
        wl = W.small_config(n_grid_r=nr, n_grid_z=nz, r_size=0.1, z_size=0.8, ppc=1)
    rng = np.random.default_rng(19)
    for s in wl.species:
        p = rng.permutation(s.n)[:300000]  # a random subset in random order
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            setattr(s, name, getattr(s, name)[p].copy())
    for precision in ("fp64", "fp32"):
        sim = api.from_workload(wl, precision=precision)
        before = [sim.species(s) for s in range(2)]
        sim.sort()
        sim.sync()
        for sid in range(2):
            b = before[sid]
            keys = cell_keys(b["r"], b["z"], wl)
            assert keys.max() >= (nr - 1) * (nz - 1) // 2  # the upper digits are exercised
            perm = np.argsort(keys, kind="stable")
            a = sim.species(sid)
            for name in ("r", "z", "vr", "vphi", "vz", "w"):
                assert np.array_equal(a[name], b[name][perm]), (precision, nodes, sid, name)
        sim.close()


def test_sort_on_large_key_range_and_many_particles():
    """256 x 2048 cells (19-bit keys, three digit passes), 8 ppc, random order."""
    wl = W.wake_config(ppc=8)
    wl.beam = None
    rng = np.random.default_rng(2)
    s = wl.species[0]
    p = rng.permutation(s.n)
    for name in ("r", "z", "vr", "vphi", "vz", "w"):
        setattr(s, name, getattr(s, name)[p].copy())
    wl.species = wl.species[:1]
    sim = api.from_workload(wl, precision="fp32")
    b = sim.species(0)
    sim.sort()
    sim.sync()
    a = sim.species(0)
    perm = np.argsort(cell_keys(b["r"], b["z"], wl), kind="stable")
    assert np.array_equal(a["r"], b["r"][perm])
    assert np.array_equal(a["vz"], b["vz"][perm])


def test_step_after_sort_matches_oracle():
    """sort_interval=1: the step sorts, then advances; the oracle advances the
    same particles given in sorted order."""
    wl = shuffled_workload(5, ppc=4, steps=2)
    gpu = api.from_workload(wl, sort_interval=1)
    gpu.step(1)
    gpu.sync()
    sorted_wl = W.thermal_config(ppc=4, steps=2)
    for s, t in zip(wl.species, sorted_wl.species):
        perm = np.argsort(cell_keys(s.r, s.z, wl), kind="stable")
        for name in ("r", "z", "vr", "vphi", "vz", "w"):
            setattr(t, name, getattr(s, name)[perm].copy())
    orc = oracle_from_workload(sorted_wl)
    orc.step()
    for c in GRIDS:
        assert rel_inf(gpu.field(c), orc.field(c)) <= 1e-12, c
    for sid in range(2):
        a, b = gpu.species(sid), orc.species(sid)
        assert np.abs(a["r"] - b["r"]).max() <= 1e-12 * wl.r_size
        assert np.abs(a["z"] - b["z"]).max() <= 1e-12 * wl.z_size
