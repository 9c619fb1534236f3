"""The batched ensemble: independent FP32 runs of different grid sizes
advanced by one persistent kernel (graph-replayed) or by one captured graph
per step of every run's own kernels, against the same runs stepped one by
one; the cancel flag and the time budget stop either mode with
PDP3G_TIMEOUT without hanging, and the autotuner picks a mode and shape.

Tolerance: each run's grids within 1e-4 of max|x| of the run stepped alone
(same arithmetic; the FP32 running sums and FP64 atomics add in a different
order).  Runs may use different pushers: the ensemble kernel picks each
species' pusher at run time."""
import numpy as np
import pytest

from helpers import rel_inf
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_runs(n=4):
    params = W.ensemble_params(seed=77, n_runs=n, cell=1e-3)
    out = []
    for i, p in enumerate(params):
        p = dict(p)
        p["n_grid_r"] = 17 + 8 * (i % 2)
        p["n_grid_z"] = 65 + 32 * (i % 3)
        p["r_size"] = (p["n_grid_r"] - 1) * 1e-3
        p["z_size"] = (p["n_grid_z"] - 1) * 1e-3
        p["ppc"] = 4 + 2 * i
        out.append(W.ensemble_run_workload(p, steps=10))
    return out


MODES = ["persistent", "step_graph"]


@pytest.mark.parametrize("mode", MODES)
def test_ensemble_matches_runs_stepped_alone(mode):
    wls = small_runs()
    alone = [api.from_workload(wl, precision="fp32") for wl in wls]
    batch = [api.from_workload(wl, precision="fp32") for wl in wls]
    for s in alone:
        s.step(10)
        s.sync()
    ens = api.Ensemble(batch)
    ens.set_mode(mode)
    ens.run(10)
    info = ens.info()
    assert info["last_steps_done"] == 10
    assert info["mode"] == api.Ensemble.MODES[mode]
    assert info["runs"] == len(wls)
    for a, b in zip(alone, batch):
        b.sync()
        assert a.time == b.time
        for c in ("E_r", "E_z", "H_phi", "J_z", "J_r", "J_phi"):
            assert rel_inf(b.field(c), a.field(c)) <= 1e-4, c
        assert np.array_equal(a.species(2)["alive"], b.species(2)["alive"])
    ens.close()


@pytest.mark.parametrize("mode", MODES)
def test_ensemble_of_runs_with_different_pushers(mode):
    wls = small_runs(3)
    pushers = ["vay", "boris_classic", "boris"]
    alone = [api.from_workload(wl, precision="fp32", pusher=p) for wl, p in zip(wls, pushers)]
    batch = [api.from_workload(wl, precision="fp32", pusher=p) for wl, p in zip(wls, pushers)]
    for s in alone:
        s.step(6)
        s.sync()
    ens = api.Ensemble(batch)
    ens.set_mode(mode)
    ens.run(6)
    assert ens.info()["last_steps_done"] == 6
    for a, b in zip(alone, batch):
        b.sync()
        for c in ("E_r", "E_z", "H_phi", "J_z", "J_r", "J_phi"):
            assert rel_inf(b.field(c), a.field(c)) <= 1e-4, c
        sa, sb = a.species(0), b.species(0)
        assert np.abs(sa["vz"] - sb["vz"]).max() <= 1e-5 * np.abs(sa["vz"]).max()
    ens.close()


@pytest.mark.parametrize("mode", MODES)
def test_ensemble_cancel_and_budget_stop_without_hanging(mode):
    wls = small_runs(2)
    sims = [api.from_workload(wl, precision="fp32") for wl in wls]
    ens = api.Ensemble(sims)
    ens.set_mode(mode)
    t0 = [s.time for s in sims]
    ens.cancel(True)
    assert ens.run_status(5) == 6  # PDP3G_TIMEOUT
    assert ens.info()["last_steps_done"] == 0
    assert [s.time for s in sims] == t0
    ens.cancel(False)
    ens.set_budget(1e-9)  # milliseconds: exhausted right away
    st = ens.run_status(1000)
    assert st == 6
    done = ens.info()["last_steps_done"]
    assert 0 <= done < 1000
    ens.set_budget(0)
    ens.run(3)
    assert ens.info()["last_steps_done"] == 3
    for s in sims:
        s.sync()
    ens.close()


def test_ensemble_autotune_and_graph():
    sims = [api.from_workload(wl, precision="fp32") for wl in small_runs(3)]
    ens = api.Ensemble(sims)
    b = ens.autotune(2)
    assert b >= 0
    ens.run(4)
    ens.run(4)  # second call replays the captured graph
    info = ens.info()
    assert info["last_steps_done"] == 4
    if b == 0:  # the step graph won
        assert info["mode"] == 1 and info["used_graph"] == 1
        assert info["graph_blocks_per_sm"] in (2, 4, 8)
    else:
        assert info["mode"] == 0 and info["blocks_per_sm"] == b
        assert info["used_graph"] in (0, 1)
    ens.close()


def test_ensemble_rejects_fp64_runs():
    wl = small_runs(1)[0]
    sim = api.from_workload(wl, precision="fp64")
    with pytest.raises(api.Pdp3gError):
        api.Ensemble([sim])


@pytest.mark.parametrize("mode", MODES)
def test_ensemble_resorts_like_runs_stepped_alone(mode):
    """Runs configured to re-sort every 4 steps: the ensemble sorts them
    between launches (steps 0, 4, 8) as pdp3g_step does."""
    wls = small_runs(3)
    alone = [api.from_workload(wl, precision="fp32", sort_interval=4) for wl in wls]
    batch = [api.from_workload(wl, precision="fp32", sort_interval=4) for wl in wls]
    for s in alone:
        s.step(10)
        s.sync()
    ens = api.Ensemble(batch)
    ens.set_mode(mode)
    ens.run(6)
    ens.run(4)  # crosses the step-8 re-sort inside the call
    assert ens.info()["last_steps_done"] == 4
    for a, b in zip(alone, batch):
        b.sync()
        for c in ("E_z", "J_r", "J_phi"):
            assert rel_inf(b.field(c), a.field(c)) <= 1e-4, c
        sa, sb = a.species(0), b.species(0)
        # same particles in the same slots after the same sorts
        assert np.abs(sa["r"] - sb["r"]).max() <= 1e-6 * wls[0].r_size
    ens.close()
