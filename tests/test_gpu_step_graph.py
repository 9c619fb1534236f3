"""pdp3g_step without timing replays one captured graph per step (the bunch
injection schedule and t += dt evaluated on the device); with timing on it
launches the kernels one by one.  Both paths must give the same run:

* time bit-identical (the same FP64 additions on host and device), alive
  flags identical (the injection schedule is integer), fields and particle
  arrays within the summation-order noise of the FP64 atomics (1e-9 in the
  FP64 form after 8 steps; 1e-4 of max|x| in the FP32 form, whose FP32 field
  copies round that noise);
* with a re-sort interval the re-sort steps run eagerly between graph
  replays and the two paths still agree;
* a species added after stepping is picked up (the graph is recaptured).
"""
import numpy as np
import pytest

from helpers import rel_inf
from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

GRIDS = ("E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "J_r", "J_z")


def run_pair(wl, precision, chunks, sort_interval=0):
    eager = api.from_workload(wl, precision=precision, sort_interval=sort_interval)
    graph = api.from_workload(wl, precision=precision, sort_interval=sort_interval)
    eager.set_timing(True)
    for n in chunks:
        eager.step(n)
        graph.step(n)
    eager.sync()
    graph.sync()
    return eager, graph


def compare(eager, graph, n_species, tol, wl):
    assert graph.time == eager.time
    for c in GRIDS:
        assert rel_inf(graph.field(c), eager.field(c)) <= tol, c
    for sid in range(n_species):
        a, b = eager.species(sid), graph.species(sid)
        assert np.array_equal(a["alive"], b["alive"]), sid
        m = a["alive"].astype(bool)
        for k in ("r", "z", "vr", "vz"):
            scale = max(float(np.abs(a[k][m]).max()), 1e-300)
            assert float(np.abs(a[k][m] - b[k][m]).max()) <= tol * scale, (sid, k)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_graph_steps_equal_eager_steps(precision):
    wl = W.small_config(beam=True, steps=8)
    eager, graph = run_pair(wl, precision, (3, 4, 1))
    assert graph.species(2)["alive"].sum() > 0  # the bunch was injected
    compare(eager, graph, 3, 1e-9 if precision == "fp64" else 1e-4, wl)
    t = graph.timing()
    assert t["launches"] > 0 and t["steps"] == 8
    eager.close()
    graph.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_graph_steps_with_resorting(precision):
    wl = W.small_config(beam=True, steps=8)
    eager, graph = run_pair(wl, precision, (5, 3), sort_interval=3)
    compare(eager, graph, 3, 1e-9 if precision == "fp64" else 1e-4, wl)
    eager.close()
    graph.close()


def test_species_added_after_stepping_is_stepped():
    wl = W.small_config(beam=False, steps=4)
    el = wl.species[0]
    eager, graph = run_pair(wl, "fp64", (2,))
    for s_ in (eager, graph):
        s_.add_species(-1.0, 1.0, el.r, el.z, -el.vr, el.vphi, el.vz, el.w)
        s_.step(2)
        s_.sync()
    compare(eager, graph, 3, 1e-9, wl)
    eager.close()
    graph.close()
