"""Seeded synthetic inputs for the PDP3 step.

The upstream code initialises particles with its own samplers
(src/particles.cpp:228-331, src/math/maxwellJuttner.cpp); those generate
inputs rather than advance the step, so this module builds the input arrays
directly with numpy and hands the same arrays to every implementation.

Conventions (SI units, upstream constants, include/constant.h:10-27):
  * the particle domain is [dr/2, R - dr/2] x [dz/2, Z - dz/2], the region
    the upstream reflection walls keep plasma in (src/particles.cpp:1318-1353);
  * each domain cell receives `ppc` macroparticles, r drawn with pdf ~ r,
    z uniform; a macroparticle's weight is the physical particle count it
    carries, n * (cell volume) / ppc;
  * ions are placed on the electron positions, so the plasma starts exactly
    neutral (as the upstream loader does, src/particles.cpp:291-292);
  * electrons get a Maxwellian with each component ~ N(0, sqrt(kT/m_e)).
"""
import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

EL_CHARGE = 1.6e-19
EL_MASS = 9.1e-31
LIGHT_SPEED = 3.0e8
PI = 3.1415926535897932


@dataclass
class SpeciesInit:
    name: str
    charge_e: float
    mass_me: float
    r: np.ndarray
    z: np.ndarray
    vr: np.ndarray
    vphi: np.ndarray
    vz: np.ndarray
    w: np.ndarray

    @property
    def n(self):
        return int(self.r.size)


@dataclass
class BeamInit:
    """Electron bunch train parameters (upstream <particle_beam>)."""
    charge_e: float = -1.0
    mass_me: float = 1.0
    number_macro: int = 0
    bunch_length: float = 0.0
    radius: float = 0.0
    density: float = 0.0
    velocity: float = 0.0
    number_bunches: int = 1
    bunches_distance: float = 0.0
    inject_rng: str = "reverse"   # "reverse" = upstream TESTMODE sequence, "hash" = seeded
    seed: int = 0


@dataclass
class Workload:
    name: str
    r_size: float
    z_size: float
    n_grid_r: int
    n_grid_z: int
    dt: float
    steps: int
    pml: Optional[List[float]] = None     # l1, l2, l3, sigma1, sigma2
    pusher: str = "boris"
    species: List[SpeciesInit] = field(default_factory=list)
    beam: Optional[BeamInit] = None

    @property
    def dr(self):
        return self.r_size / (self.n_grid_r - 1)

    @property
    def dz(self):
        return self.z_size / (self.n_grid_z - 1)

    @property
    def n_particles(self):
        n = sum(s.n for s in self.species)
        if self.beam is not None:
            n += self.beam.number_macro * self.beam.number_bunches
        return n


def courant_dt(dr, dz, courant=0.5):
    return courant / (LIGHT_SPEED * math.sqrt(dr ** -2 + dz ** -2))


def plasma_positions(rng, r_size, z_size, n_grid_r, n_grid_z, ppc, density_fn):
    """Positions and weights for `ppc` particles in every domain cell."""
    dr = r_size / (n_grid_r - 1)
    dz = z_size / (n_grid_z - 1)
    # cell edges of the particle domain [dr/2, R-dr/2] x [dz/2, Z-dz/2]
    r_edges = np.concatenate(([dr / 2], dr * np.arange(1, n_grid_r - 1), [r_size - dr / 2]))
    z_edges = np.concatenate(([dz / 2], dz * np.arange(1, n_grid_z - 1), [z_size - dz / 2]))
    nrc, nzc = r_edges.size - 1, z_edges.size - 1
    ic = np.repeat(np.arange(nrc), nzc * ppc)
    kc = np.tile(np.repeat(np.arange(nzc), ppc), nrc)
    a, b = r_edges[ic], r_edges[ic + 1]
    u = rng.random(ic.size)
    r = np.sqrt(a * a + u * (b * b - a * a))
    za, zb = z_edges[kc], z_edges[kc + 1]
    z = za + rng.random(ic.size) * (zb - za)
    vol = PI * (b * b - a * a) * (zb - za)
    n_phys = density_fn(0.5 * (za + zb))
    w = n_phys * vol / ppc
    return r, z, w


def thermal_plasma(rng, r_size, z_size, n_grid_r, n_grid_z, ppc, density_fn, t_ev,
                   ion_mass_me=1836.0):
    r, z, w = plasma_positions(rng, r_size, z_size, n_grid_r, n_grid_z, ppc, density_fn)
    n = r.size
    sig = math.sqrt(t_ev * EL_CHARGE / EL_MASS)
    ve = rng.normal(0.0, sig, size=(3, n))
    zero = np.zeros(n)
    el = SpeciesInit("Electrons", -1.0, 1.0, r, z, ve[0].copy(), ve[1].copy(), ve[2].copy(), w)
    ion = SpeciesInit("Ions", 1.0, ion_mass_me, r.copy(), z.copy(), zero, zero.copy(),
                      zero.copy(), w.copy())
    return [el, ion]


def absorbing_layer(n_grid_r, n_grid_z, cells, sigma1=1e-5, sigma2=7e-2):
    """set_pml arguments for a `cells`-cell layer at r_max and both z ends
    (the upstream code takes floor(n_grid * comparative_l) cells,
    src/geometry.cpp:60-66; the +0.5 keeps floor() off the integer edge)."""
    return [(cells + 0.5) / n_grid_z, (cells + 0.5) / n_grid_z, (cells + 0.5) / n_grid_r,
            sigma1, sigma2]


def gamma_velocity(gamma):
    return LIGHT_SPEED * math.sqrt(1.0 - 1.0 / (gamma * gamma))


def thermal_config(seed=1001, n_grid_r=65, n_grid_z=257, r_size=0.05, z_size=0.2, ppc=32,
                   density=1e16, steps=200):
    """Plain FP64 thermal plasma: 64x256 cells, 32 ppc per species, 1 eV
    electrons, cold protons, 10-cell absorbing layer at r_max and both z ends."""
    rng = np.random.default_rng(seed)
    dr = r_size / (n_grid_r - 1)
    dz = z_size / (n_grid_z - 1)
    sp = thermal_plasma(rng, r_size, z_size, n_grid_r, n_grid_z, ppc,
                        lambda zc: np.full_like(zc, density), 1.0)
    pml = absorbing_layer(n_grid_r, n_grid_z, 10)
    return Workload("thermal_%dx%d_ppc%d" % (n_grid_r - 1, n_grid_z - 1, ppc), r_size, z_size,
                    n_grid_r, n_grid_z, courant_dt(dr, dz), steps, pml, "boris", sp)


def wake_config(seed=1002, n_grid_r=257, n_grid_z=2049, r_size=0.1, z_size=0.8, ppc=64,
                density=1e17, steps=1000, beam_gamma=5.0, beam_radius=5e-3, beam_length=0.02,
                beam_density=5e16, pusher="boris"):
    """Beam-plasma wake: 256x2048 cells, 64 ppc per species at 1e17 m^-3,
    1 eV electrons, gamma=5 electron bunch (r 5 mm, length 2 cm, 5e16 m^-3)
    injected at z=0, 10-cell absorbing layer."""
    rng = np.random.default_rng(seed)
    dr = r_size / (n_grid_r - 1)
    dz = z_size / (n_grid_z - 1)
    sp = thermal_plasma(rng, r_size, z_size, n_grid_r, n_grid_z, ppc,
                        lambda zc: np.full_like(zc, density), 1.0)
    pml = absorbing_layer(n_grid_r, n_grid_z, 10)
    bunch_cells = (beam_radius / dr) * (beam_length / dz)
    beam = BeamInit(-1.0, 1.0, int(round(64 * bunch_cells)), beam_length, beam_radius,
                    beam_density, gamma_velocity(beam_gamma), 1, 0.0, "reverse", seed)
    return Workload("wake_%dx%d_ppc%d" % (n_grid_r - 1, n_grid_z - 1, ppc), r_size, z_size,
                    n_grid_r, n_grid_z, courant_dt(dr, dz), steps, pml, pusher, sp, beam)


def small_config(seed=7, n_grid_r=17, n_grid_z=33, r_size=0.01, z_size=0.04, ppc=8,
                 density=1e16, t_ev=1.0, beam=False, steps=10, pusher="boris"):
    """Small grid for parity tests (seconds on the oracle)."""
    rng = np.random.default_rng(seed)
    dr = r_size / (n_grid_r - 1)
    dz = z_size / (n_grid_z - 1)
    sp = thermal_plasma(rng, r_size, z_size, n_grid_r, n_grid_z, ppc,
                        lambda zc: np.full_like(zc, density), t_ev)
    pml = [3.0 / n_grid_z, 3.0 / n_grid_z, 3.0 / n_grid_r, 1e-5, 7e-2]
    bm = None
    if beam:
        bm = BeamInit(-1.0, 1.0, 2000, 4 * dz * 10, 4 * dr, 1e16, gamma_velocity(3.0), 1, 0.0,
                      "reverse", seed)
    return Workload("small_%dx%d" % (n_grid_r - 1, n_grid_z - 1), r_size, z_size, n_grid_r,
                    n_grid_z, courant_dt(dr, dz), steps, pml, pusher, sp, bm)
