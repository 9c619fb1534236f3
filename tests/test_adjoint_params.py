"""Host side of the differentiable window (CPU): the parameter map from
theta (16 density-bump coefficients, bunch gamma, bunch radius) to the
initial state, and its derivatives used to chain the per-particle adjoints.

* The bunch radii and weights restated in numpy equal the oracle's
  Bunch::Bunch (src/bunch.cpp:6-80) to rounding.
* d(r, w)/dR of the bunch and dw/dc of the plasma match central differences.
* adjoint_gradient applied to synthetic adjoints equals the directional
  derivative of the linear functional sum(lw * w) + sum(lr * r) + lv * v.
"""
import numpy as np

from helpers import oracle_from_workload
from pdp3_b200 import workloads as W

SMALL = dict(n_grid_r=17, n_grid_z=65, r_size=0.05 / 8, z_size=0.4 / 16, ppc=4, steps=10,
             bunch_ppc=2, nominal_radius=2e-3)


def test_bunch_init_matches_oracle():
    th = W.adjoint_theta()
    th[-1] = 2e-3
    wl, _ = W.adjoint_config(th, **SMALL)
    o = oracle_from_workload(wl)
    sp = o.species(2)
    b = wl.beam
    r, w, _, _ = W.bunch_init_np(b.number_macro, b.radius, b.bunch_length / b.velocity,
                                 b.velocity, b.density, wl.dr, wl.dz)
    assert np.abs(sp["r"] - r).max() <= 1e-15 * wl.r_size
    assert np.abs(sp["w"] - w).max() <= 1e-12 * np.abs(w).max()


def test_bunch_radius_derivatives():
    b = dict(n=5000, duration=0.02 / 2.9e8, velocity=2.9e8, density=5e16, dr=3.9e-4, dz=3.9e-4)
    R, h = 5e-3, 1e-9
    _, _, dr_dR, dw_dR = W.bunch_init_np(b["n"], R, b["duration"], b["velocity"], b["density"],
                                         b["dr"], b["dz"])
    rp, wp, _, _ = W.bunch_init_np(b["n"], R + h, b["duration"], b["velocity"], b["density"],
                                   b["dr"], b["dz"])
    rm, wm, _, _ = W.bunch_init_np(b["n"], R - h, b["duration"], b["velocity"], b["density"],
                                   b["dr"], b["dz"])
    assert np.abs((rp - rm) / (2 * h) - dr_dR).max() <= 1e-6
    assert np.abs((wp - wm) / (2 * h) - dw_dR).max() <= 1e-6 * np.abs(dw_dR).max()


def test_gradient_chain_rule():
    th = W.adjoint_theta()
    th[-1] = 2e-3
    wl, aux = W.adjoint_config(th, **SMALL)
    rng = np.random.default_rng(11)
    plasma = [{"w": rng.normal(size=s.n)} for s in wl.species]
    bunch = {"r": rng.normal(size=wl.beam.number_macro),
             "w": rng.normal(size=wl.beam.number_macro)}
    lv = 1.7e-3
    g = W.adjoint_gradient(wl, aux, plasma, bunch, lv)

    def functional(t):
        wl2, _ = W.adjoint_config(t, **SMALL)
        b = wl2.beam
        r, w, _, _ = W.bunch_init_np(b.number_macro, b.radius, b.bunch_length / b.velocity,
                                     b.velocity, b.density, wl2.dr, wl2.dz)
        val = sum(float(np.dot(p["w"], s.w)) for p, s in zip(plasma, wl2.species))
        return val + float(np.dot(bunch["r"], r) + np.dot(bunch["w"], w)) + lv * b.velocity

    for j in (0, 7, 15, 16, 17):
        # gamma moves only the lv * v term of a large sum: a wider step keeps
        # the difference above the sum's rounding
        h = (1e-4 if j == 16 else 1e-6) * abs(th[j])
        tp, tm = th.copy(), th.copy()
        tp[j] += h
        tm[j] -= h
        fd = (functional(tp) - functional(tm)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-6 * max(abs(fd), abs(g[j])), (j, fd, g[j])


def test_bunch_weight_jump_term():
    """Bunch::Bunch's volume sum switches branch at r = dr; over an R step
    that moves many radii across it, the mean weight's difference quotient
    equals the pathwise derivative plus bunch_weight_jump_dR (and not the
    pathwise derivative alone)."""
    n, R, dr, dz, v = 10486, 5e-3, 7.8125e-4, 7.8125e-4, 2.9394e8
    dur = 0.02 / v
    _, _, _, dw = W.bunch_init_np(n, R, dur, v, 5e16, dr, dz)
    jump = W.bunch_weight_jump_dR(n, R, dur, v, 5e16, dr, dz)
    h = 1e-4
    wp = W.bunch_init_np(n, R + h, dur, v, 5e16, dr, dz)[1]
    wm = W.bunch_init_np(n, R - h, dur, v, 5e16, dr, dz)[1]
    fd = np.mean((wp - wm) / (2 * h))
    assert abs(fd / np.mean(dw + jump) - 1) <= 1e-4
    assert abs(fd / np.mean(dw) - 1) >= 5e-3
