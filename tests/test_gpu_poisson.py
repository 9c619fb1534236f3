"""PoissonDirichlet::poisson_solve on the device (pdp3g_poisson_solve)
against the upstream solver itself (oracle/_ref) and the numpy restatement
(oracle.poisson): phi, E_r (rows i < n_grid_r-1) and E_z (columns
k < n_grid_z-1) within 1e-11 of each grid's largest magnitude; the E values
the solve does not write are kept; grids the radix-2 transform cannot take
are refused."""
import numpy as np
import pytest

from oracle import refsim
from oracle.poisson import poisson_dirichlet
from pdp3_b200 import api

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refsim.available("boris"),
                                 reason="oracle/_ref not built (needs the upstream sources)")]


def close(a, b, tol=1e-11):
    scale = np.abs(b).max()
    assert scale > 0
    return np.abs(a - b).max() <= tol * scale


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("shape,size", [((33, 127), (0.02, 0.1)), ((255, 2047), (0.25, 2.0))])
def test_poisson_matches_reference(shape, size, precision):
    nr, nz = shape
    dr, dz = size[0] / (nr - 1), size[1] / (nz - 1)
    rng = np.random.default_rng(5)
    rho = rng.normal(0.0, 1e-4, shape)
    ref = refsim.RefSim(size[0], size[1], nr, nz, 1e-12)
    phi_w, er_w, ez_w = ref.poisson_dirichlet(rho)
    sim = api.Simulation(size[0], size[1], nr, nz, 1e-12, precision=precision)
    marker = rng.normal(0.0, 1.0, shape)
    sim.set_field("E_r", marker)
    sim.set_field("E_z", marker)
    phi = sim.poisson_solve(rho)
    er, ez = sim.field("E_r"), sim.field("E_z")
    assert close(phi, phi_w)
    assert close(er[:-1], er_w[:-1])
    assert close(ez[:, :-1], ez_w[:, :-1])
    assert np.array_equal(er[-1], marker[-1]) and np.array_equal(ez[:, -1], marker[:, -1])
    o_phi, o_er, o_ez = poisson_dirichlet(rho, dr, dz)
    assert close(phi, o_phi) and close(er[:-1], o_er[:-1]) and close(ez[:, :-1], o_ez[:, :-1])
    sim.close()
    ref.close()


def test_poisson_from_the_species_charge_density():
    size, nr, nz = (0.02, 0.1), 33, 127
    sim = api.Simulation(size[0], size[1], nr, nz, 1e-12)
    sim.add_species_upstream(-1.0, 1.0, 20000, 1e16, 2e16, 1.0)
    sim.add_species_upstream(1.0, 1836.0, 10000, 1e16, 1e16, 0.1)
    rho = sim.charge_density()
    phi = sim.poisson_solve()
    o_phi, o_er, o_ez = poisson_dirichlet(rho, size[0] / (nr - 1), size[1] / (nz - 1))
    assert close(phi, o_phi)
    assert close(sim.field("E_r")[:-1], o_er[:-1])
    assert close(sim.field("E_z")[:, :-1], o_ez[:, :-1])
    sim.close()


def test_poisson_refuses_other_grids():
    sim = api.Simulation(0.05, 0.2, 65, 257, 1e-12)
    with pytest.raises(api.Pdp3gError):
        sim.poisson_solve(np.zeros((65, 257)))
    sim.close()
