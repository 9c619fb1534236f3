"""The adjoint window (pdp3g_forward_window / pdp3g_backward_window) on B200.

* Fields only (no particles): the window is linear in the initial E and H and
  the loss quadratic, so the adjoint of every initial field component must
  equal central differences to rounding (1e-9 of the largest entry).
* Small differentiable window (32x256 cells, 8 ppc per species, gamma=5
  bunch, 100 steps, checkpoints every 20): the gradient with respect to the
  three density coefficients nearest the probe (norm-wise) and the bunch
  gamma against FP64 central differences with a relative step of 1e-4, to
  1e-3; pathwise mode, whose derivative is the one such small steps measure
  at this size (few particles cross a jump of the gather weights).
* Forward + backward leaves the state the forward ended in, and the adjoint
  rejects what it does not support.
* The forward stores its last interval's particle-phase inputs, which the
  first backward reverses without recomputing; a second backward recomputes
  every interval and must give the same gradient (1e-9: the recompute's
  atomic summation order differs from the forward's).
* The mean-field terms one by one: none is the pathwise derivative, the
  gather terms alone are the default mean field, the wall terms change the
  gradient, unknown bits are rejected.
"""
import numpy as np
import pytest

from pdp3_b200 import api
from pdp3_b200 import workloads as W

pytestmark = pytest.mark.gpu

SMALL = dict(n_grid_r=33, n_grid_z=257, r_size=0.025, z_size=0.2, ppc=8)
PROBE = (0, 8, 10, 42)


def test_field_adjoint_is_exact():
    wl = W.small_config(beam=False)
    sim = api.Simulation(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, pml=wl.pml,
                         precision="fp32")
    rng = np.random.default_rng(3)
    comps = ("E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z")
    init = {c: rng.normal(0, 1e3 if c[0] == "E" else 1.0, (wl.n_grid_r, wl.n_grid_z))
            for c in comps}

    def load(pert=None):
        for c, a in init.items():
            b = a.copy()
            if pert is not None and pert[0] == c:
                b[pert[1], pert[2]] += pert[3]
            sim.set_field(c, b)

    probe = (0, 4, 10, 20)
    load()
    adj = api.Adjoint(sim, 30, 7, probe)
    adj.forward()
    adj.backward()
    grads = {c: adj.field(c) for c in comps}
    adj.close()
    # E_phi, H_r and H_z form the decoupled azimuthal mode: without
    # particles they never reach E_z, so their adjoints vanish
    for c in ("E_phi", "H_r", "H_z"):
        assert np.abs(grads[c]).max() == 0.0, c
    for c in ("E_r", "E_z", "H_phi"):
        scale = np.abs(grads[c]).max()
        assert scale > 0, c
        h = 1.0 if c[0] == "E" else 1e-3
        for (i, k) in [(1, 12), (2, 15), (0, 14), (3, 11), (5, 20)]:
            vals = []
            for sgn in (1, -1):
                load((c, i, k, sgn * h))
                a2 = api.Adjoint(sim, 30, 7, probe)
                vals.append(a2.forward())
                a2.close()
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - grads[c][i, k]) <= 1e-9 * scale, (c, i, k, fd, grads[c][i, k])
    sim.close()


def central_fd(fam, th, j, steps, h=1e-4):
    """(L(theta_j (1 + h)) - L(theta_j (1 - h))) / (2 h theta_j), FP64 form."""
    ls = []
    for x in (h, -h):
        t = th.copy()
        t[j] = th[j] * (1 + x)
        wl, _ = fam.workload(t)
        sim = api.from_workload(wl, precision="fp64")
        sim.step(steps)
        sim.sync()
        ls.append(W.probe_loss(sim.field("E_z"), wl.dr, wl.dz, PROBE))
        sim.close()
    return (ls[0] - ls[1]) / (2 * h * th[j])


def test_gradient_matches_fp64_finite_differences():
    th = W.adjoint_theta()
    fam = W.AdjointFamily(th, **SMALL)
    wl, aux = fam.workload(th)
    sim = api.from_workload(wl, precision="fp32")
    adj = api.Adjoint(sim, 100, 20, PROBE)
    adj.set_mode("pathwise")
    adj.forward()
    adj.backward()
    g = W.adjoint_gradient(wl, aux, [adj.species(0), adj.species(1)], adj.species(2),
                           adj.bunch_velocity(2))
    adj.close()
    sim.close()
    dens = [0, 1, 2]
    fd = {j: central_fd(fam, th, j, 100) for j in dens + [16]}
    gd, fdd = np.array([g[j] for j in dens]), np.array([fd[j] for j in dens])
    assert np.linalg.norm(gd - fdd) <= 1e-3 * np.linalg.norm(fdd), (gd, fdd)
    assert abs(g[16] - fd[16]) <= 1e-3 * abs(fd[16]), (g[16], fd[16])


def test_backward_restores_forward_end_state_and_rejects_misuse():
    th = W.adjoint_theta()
    wl, _ = W.AdjointFamily(th, **SMALL).workload(th)
    sim = api.from_workload(wl, precision="fp32")
    adj = api.Adjoint(sim, 40, 15, PROBE)
    with pytest.raises(api.Pdp3gError):
        adj.backward()  # nothing to reverse yet
    adj.forward()
    after = {c: sim.field(c) for c in ("E_z", "H_phi")}
    sp = sim.species(0)
    t_end = sim.time
    adj.backward()
    for c, a in after.items():
        assert np.array_equal(sim.field(c), a), c
    sp2 = sim.species(0)
    for k in ("r", "z", "vr", "vz"):
        assert np.array_equal(sp2[k], sp[k]), k
    assert sim.time == t_end
    with pytest.raises(api.Pdp3gError):
        api.Adjoint(sim, 10, 5, (0, 8, 10, 10_000))  # probe outside the grid
    adj.close()
    sim.close()
    s64 = api.from_workload(wl, precision="fp64")
    with pytest.raises(api.Pdp3gError):
        api.Adjoint(s64, 10, 5, PROBE)  # the FP64 form has no adjoint
    s64.close()


def test_first_backward_reuses_the_last_interval():
    th = W.adjoint_theta()
    wl, aux = W.AdjointFamily(th, **SMALL).workload(th)
    sim = api.from_workload(wl, precision="fp32")
    # 45 steps at 20 per checkpoint: a last interval of 5 steps
    adj = api.Adjoint(sim, 45, 20, PROBE)
    adj.forward()
    grads = []
    for _ in range(2):
        adj.backward()
        grads.append(np.array(W.adjoint_gradient(
            wl, aux, [adj.species(0), adj.species(1)], adj.species(2), adj.bunch_velocity(2))))
    assert np.abs(grads[0]).max() > 0
    assert np.allclose(grads[0], grads[1], rtol=1e-9, atol=0), (grads[0], grads[1])
    adj.close()
    sim.close()


def test_jump_terms_select_the_mean_field_parts():
    """With the uniform jump density (face width 0), where the wall-cell
    term applies; the box-kernel default is exercised by the config-4 test."""
    th = W.adjoint_theta()
    wl, aux = W.AdjointFamily(th, **SMALL).workload(th)
    sim = api.from_workload(wl, precision="fp32")
    adj = api.Adjoint(sim, 40, 15, PROBE)
    adj.set_face_width(0.0)
    adj.forward()
    grads = {}
    for name, select in [("pathwise", lambda: adj.set_mode("pathwise")),
                         ("none", lambda: adj.set_jump_terms()),
                         ("default", lambda: adj.set_mode("mean_field")),
                         ("gather", lambda: adj.set_jump_terms("gather")),
                         ("all", lambda: adj.set_jump_terms("gather", "walls", "wall_cells"))]:
        select()
        adj.backward()
        grads[name] = np.array(W.adjoint_gradient(
            wl, aux, [adj.species(0), adj.species(1)], adj.species(2), adj.bunch_velocity(2)))
    # the FP64 adjoint grids sum by atomics, whose order varies run to run
    for a, b in (("none", "pathwise"), ("gather", "default")):
        assert np.allclose(grads[a], grads[b], rtol=1e-9, atol=0), (a, b)
    assert not np.allclose(grads["all"], grads["gather"], rtol=1e-6, atol=0)
    with pytest.raises(api.Pdp3gError):
        sim._check(adj.L.pdp3g_adjoint_set_jump_terms(adj.h, 8), "adjoint_set_jump_terms")
    for bad in (-0.1, 0.6):
        with pytest.raises(api.Pdp3gError):
            adj.set_face_width(bad)
    # the box kernel moves the gradient away from the uniform shares
    adj.set_mode("mean_field")
    adj.set_face_width(0.125)
    adj.backward()
    g_box = np.array(W.adjoint_gradient(
        wl, aux, [adj.species(0), adj.species(1)], adj.species(2), adj.bunch_velocity(2)))
    assert not np.allclose(g_box, grads["default"], rtol=1e-6, atol=0)
    adj.close()
    sim.close()
