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
    sort_interval: int = 0
    # plasma generated on the GPU instead of `species` (cases too large for
    # host arrays): a DevicePlasma
    device_plasma: Optional["DevicePlasma"] = None

    @property
    def dr(self):
        return self.r_size / (self.n_grid_r - 1)

    @property
    def dz(self):
        return self.z_size / (self.n_grid_z - 1)

    @property
    def n_particles(self):
        n = sum(s.n for s in self.species)
        if self.device_plasma is not None:
            n += 2 * self.device_plasma.n
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


def ensemble_params(seed=1005, n_runs=64, cell=3.90625e-4, scale=1):
    """Run parameters of the batched-ensemble case: grids drawn uniformly from
    r in {64, 128, 256} x z in {256, 512, 1024} cells (cell size fixed; each
    divided by scale for a case of smaller runs), 16-64 ppc, density
    log-uniform in [1e15, 1e17] m^-3, an electron bunch with gamma uniform in
    [3, 10] per run.  Returns one dict per run; build each Workload with
    ensemble_run_workload (so only one run's arrays are on the host at a
    time)."""
    rng = np.random.default_rng(seed)
    runs = []
    for r in range(n_runs):
        nrc = int(rng.choice([64, 128, 256])) // scale
        nzc = int(rng.choice([256, 512, 1024])) // scale
        runs.append({"seed": seed * 1000 + r, "n_grid_r": nrc + 1, "n_grid_z": nzc + 1,
                     "r_size": nrc * cell, "z_size": nzc * cell,
                     "ppc": int(rng.integers(16, 65)),
                     "density": float(10 ** rng.uniform(15, 17)),
                     "gamma": float(rng.uniform(3, 10))})
    return runs


def ensemble_run_workload(p, steps=500):
    """Workload of one ensemble run (see ensemble_params)."""
    rng = np.random.default_rng(p["seed"])
    nr, nz = p["n_grid_r"], p["n_grid_z"]
    dr = p["r_size"] / (nr - 1)
    dz = p["z_size"] / (nz - 1)
    sp = thermal_plasma(rng, p["r_size"], p["z_size"], nr, nz, p["ppc"],
                        lambda zc: np.full_like(zc, p["density"]), 1.0)
    radius, length = 0.1 * p["r_size"], 0.05 * p["z_size"]
    bunch_cells = (radius / dr) * (length / dz)
    beam = BeamInit(-1.0, 1.0, int(round(64 * bunch_cells)), length, radius, 0.5 * p["density"],
                    gamma_velocity(p["gamma"]), 1, 0.0, "reverse", p["seed"])
    return Workload("ens_%dx%d_ppc%d" % (nr - 1, nz - 1, p["ppc"]), p["r_size"], p["z_size"],
                    nr, nz, courant_dt(dr, dz), steps, absorbing_layer(nr, nz, 10), "boris", sp,
                    beam)


# ---------------------------------------------------------------- adjoint

N_BUMPS = 16


def bump_basis(z, z_size, n_bumps=N_BUMPS):
    """phi_j(z), j < n_bumps: Gaussian bumps exp(-(z - z_j)^2 / (2 sigma^2))
    centred at z_j = (j + 1/2) Z / n_bumps with sigma = Z / n_bumps, scaled by
    1 / sqrt(2 pi) so that sum_j phi_j(z) ~ 1 away from the ends (the density
    is then about the mean coefficient).  Returns an array (z.size, n_bumps)."""
    z = np.asarray(z, dtype=np.float64)
    centres = (np.arange(n_bumps) + 0.5) * z_size / n_bumps
    sig = z_size / n_bumps
    g = np.exp(-0.5 * ((z[:, None] - centres[None, :]) / sig) ** 2)
    return g / math.sqrt(2.0 * math.pi)


def random_reverse_np(idx, base):
    """Radical inverse of idx in `base` (upstream random_reverse,
    src/math/rand.cpp:40-53), vectorised."""
    x = np.asarray(idx, dtype=np.int64).copy()
    out = np.zeros(x.shape)
    scale = 1.0 / base
    while np.any(x >= 1):
        out += (x % base) * scale
        x //= base
        scale /= base
    return out


def adjoint_theta(seed=1004):
    """Parameters of the differentiable window: 16 bump coefficients drawn
    from N(1e17, (1e16)^2) m^-3, bunch gamma 5, bunch radius 5 mm."""
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.normal(1e17, 1e16, N_BUMPS), [5.0, 5e-3]])


def adjoint_config(theta, seed=1004, n_grid_r=129, n_grid_z=1025, r_size=0.1, z_size=0.8,
                   ppc=32, steps=500, beam_length=0.02, beam_density=5e16, nominal_radius=5e-3,
                   bunch_ppc=64):
    """Differentiable window: 128x1024 cells, 32 ppc per species, background
    density sum_j c_j phi_j(z) (theta[:16] = c), electron bunch with
    gamma = theta[16] and radius theta[17] injected at z = 0.  Every
    particle's position and velocity is independent of theta; weights carry
    the density and the bunch radius, and the bunch's macroparticle count is
    fixed by the nominal radius, so theta only moves continuous quantities.
    Returns (Workload, aux) with aux holding what adjoint_gradient needs."""
    theta = np.asarray(theta, dtype=np.float64)
    c, gamma, radius = theta[:N_BUMPS], float(theta[N_BUMPS]), float(theta[N_BUMPS + 1])
    rng = np.random.default_rng(seed)
    dr = r_size / (n_grid_r - 1)
    dz = z_size / (n_grid_z - 1)
    dens = lambda zc: bump_basis(zc, z_size) @ c
    sp = thermal_plasma(rng, r_size, z_size, n_grid_r, n_grid_z, ppc, dens, 1.0)
    # z-cell column of every plasma particle (cells of the particle domain)
    kc = np.tile(np.repeat(np.arange(n_grid_z - 1, dtype=np.int32), ppc), n_grid_r - 1)
    bunch_cells = (nominal_radius / dr) * (beam_length / dz)
    beam = BeamInit(-1.0, 1.0, int(round(bunch_ppc * bunch_cells)), beam_length, radius,
                    beam_density, gamma_velocity(gamma), 1, 0.0, "reverse", seed)
    pml = absorbing_layer(n_grid_r, n_grid_z, 10)
    wl = Workload("adjoint_%dx%d_ppc%d" % (n_grid_r - 1, n_grid_z - 1, ppc), r_size, z_size,
                  n_grid_r, n_grid_z, courant_dt(dr, dz), steps, pml, "boris", sp, beam)
    z_edges = np.concatenate(([dz / 2], dz * np.arange(1, n_grid_z - 1), [z_size - dz / 2]))
    zc = 0.5 * (z_edges[:-1] + z_edges[1:])
    aux = {"kc": kc, "zc": zc, "theta": theta.copy()}
    return wl, aux


class AdjointFamily:
    """adjoint_config for many theta at one seed: the theta-independent
    arrays (positions, velocities, cell volumes) are built once and each
    workload() only rescales the plasma weights and replaces the bunch."""

    def __init__(self, theta0, **kw):
        self.kw = kw
        self.wl0, self.aux0 = adjoint_config(theta0, **kw)
        c0 = np.asarray(theta0, dtype=np.float64)[:N_BUMPS]
        self.n0_col = bump_basis(self.aux0["zc"], self.wl0.z_size) @ c0

    def workload(self, theta):
        import dataclasses
        theta = np.asarray(theta, dtype=np.float64)
        n_col = bump_basis(self.aux0["zc"], self.wl0.z_size) @ theta[:N_BUMPS]
        scale = (n_col / self.n0_col)[self.aux0["kc"]]
        species = [dataclasses.replace(s, w=s.w * scale) for s in self.wl0.species]
        beam = dataclasses.replace(self.wl0.beam, radius=float(theta[N_BUMPS + 1]),
                                   velocity=gamma_velocity(float(theta[N_BUMPS])))
        wl = dataclasses.replace(self.wl0, species=species, beam=beam)
        aux = dict(self.aux0, theta=theta.copy())
        return wl, aux


def bunch_init_np(n, radius, duration, velocity, density, dr, dz):
    """Radii and weights of Bunch::Bunch (src/bunch.cpp:6-80, TESTMODE
    radial sequence) and their derivatives with respect to the radius."""
    rnd = random_reverse_np(np.arange(n), 9)
    r = (radius - dr) * rnd + dr / 2
    dr_dR = rnd
    b_len = duration * velocity
    N_total = PI * radius ** 2 * b_len * density
    dN_dR = 2.0 * PI * radius * b_len * density
    far = r > dr
    vol = np.where(far, 2 * PI * r * dr * dz, PI * r * r * dz)
    dvol = np.where(far, 2 * PI * dr * dz, 2 * PI * r * dz) * dr_dR
    v_avg = vol.sum() / n
    dv_avg = dvol.sum() / n
    half = r > dr / 2
    num = np.where(half, 2 * PI * r * dr * dz, PI * (r * r + r * dr + dr * dr / 4) * dz)
    dnum = np.where(half, 2 * PI * dr * dz, PI * (2 * r + dr) * dz) * dr_dR
    norm = num / v_avg
    dnorm = (dnum * v_avg - num * dv_avg) / (v_avg * v_avg)
    w = N_total / n * norm
    dw_dR = dN_dR / n * norm + N_total / n * dnorm
    return r, w, dr_dR, dw_dR


def bunch_weight_jump_dR(n, radius, duration, velocity, density, dr, dz):
    """Expected-jump part of dw_i/dR for Bunch::Bunch's weights.  The volume
    sum v_total switches from pi r^2 dz to 2 pi r dr dz at r = dr, a jump of
    pi dr^2 dz; the radii (R - dr) U_i + dr/2 (U_i the radical-inverse
    sequence, uniform in [0, 1)) cross r = dr at the rate n (dr/2)/(R - dr)^2
    per unit R, so the mean of v_total over the sequence moves by that rate
    times the jump, which every weight feels through v_avg."""
    r, w, _, _ = bunch_init_np(n, radius, duration, velocity, density, dr, dz)
    far = r > dr
    vol = np.where(far, 2 * PI * r * dr * dz, PI * r * r * dz)
    v_avg = vol.sum() / n
    dv_avg_jump = PI * dr * dr * dz * (dr / 2) / (radius - dr) ** 2
    return -w * dv_avg_jump / v_avg


def adjoint_gradient(wl, aux, plasma_adj, bunch_adj, bunch_dl_dv, mean_field=False):
    """dL/dtheta from the adjoints of the window's initial state.
    plasma_adj: per plasma species dict with "w" (dL/dw per particle);
    bunch_adj: dict with "r" (dL/dr) and "w"; bunch_dl_dv: dL/dv_beam.
    mean_field adds the expected jump term of the bunch weights' volume
    branch (bunch_weight_jump_dR), to go with the adjoint's mean-field mode."""
    theta = aux["theta"]
    c = theta[:N_BUMPS]
    phi = bump_basis(aux["zc"], wl.z_size)           # (columns, bumps)
    n_col = phi @ c
    g = np.zeros(theta.size)
    for a, s in zip(plasma_adj, wl.species):
        # w_p = n(zc) vol/ppc  ->  dw_p/dc_j = w_p phi_j(zc) / n(zc)
        col = np.bincount(aux["kc"], weights=a["w"] * s.w, minlength=phi.shape[0])
        g[:N_BUMPS] += (col / n_col) @ phi
    b = wl.beam
    gamma = theta[N_BUMPS]
    v = gamma_velocity(gamma)
    dv_dgamma = LIGHT_SPEED / (gamma ** 3 * math.sqrt(1.0 - 1.0 / (gamma * gamma)))
    g[N_BUMPS] = bunch_dl_dv * dv_dgamma
    _, _, dr_dR, dw_dR = bunch_init_np(b.number_macro, b.radius, b.bunch_length / v, v,
                                       b.density, wl.dr, wl.dz)
    if mean_field:
        dw_dR = dw_dR + bunch_weight_jump_dR(b.number_macro, b.radius, b.bunch_length / v, v,
                                             b.density, wl.dr, wl.dz)
    g[N_BUMPS + 1] = float(np.dot(bunch_adj["r"], dr_dR) + np.dot(bunch_adj["w"], dw_dR))
    return g


def probe_loss(ez, dr, dz, probe):
    """sum over probe nodes of E_z^2 times the node ring volume (the loss of
    the adjoint window)."""
    r0, r1, z0, z1 = probe
    i = np.arange(r0, r1, dtype=np.float64)
    vol = np.where(i == 0, PI * dz * dr * dr / 4.0, 2.0 * PI * dz * dr * dr * i)
    return float(np.sum(ez[r0:r1, z0:z1] ** 2 * vol[:, None]))


# probe nodes (r0, r1, z0, z1): 16 x 64 cells on the axis over z in
# [0.094, 0.144] m, which holds the bunch's tail and the start of its wake
# after the 500-step window (the head is then 173 cells from the entrance)
ADJOINT_PROBE = (0, 16, 120, 184)


# ------------------------------------------------------- device-side plasma


@dataclass
class DevicePlasma:
    """Electrons and protons generated on the GPU with torch (seeded CUDA
    generator), with the same conventions as thermal_plasma: `ppc` particles
    per domain cell, r with pdf ~ r and z uniform inside the cell, weight
    n(z_cell) * (cell volume) / ppc, ions on the electron positions, 1 eV
    Maxwellian electrons, cold ions.  The density is n_max * min(z / z_ramp, 1)
    (z_ramp = 0: uniform n_max)."""
    seed: int
    r_size: float
    z_size: float
    n_grid_r: int
    n_grid_z: int
    ppc: int
    n_max: float
    z_ramp: float = 0.0
    t_ev: float = 1.0
    ion_mass_me: float = 1836.0

    @property
    def n(self):
        return (self.n_grid_r - 1) * (self.n_grid_z - 1) * self.ppc

    def add_to(self, sim, device):
        """Generates the two species on `device` and adds them to sim."""
        import torch
        dev = torch.device("cuda", device)
        gen = torch.Generator(device=dev)
        gen.manual_seed(self.seed)
        nr, nz, ppc = self.n_grid_r, self.n_grid_z, self.ppc
        dr = self.r_size / (nr - 1)
        dz = self.z_size / (nz - 1)
        nrc, nzc = nr - 1, nz - 1
        n = nrc * nzc * ppc
        idx = torch.arange(n, device=dev, dtype=torch.int64)
        ic = idx // (nzc * ppc)
        kc = (idx // ppc) % nzc
        del idx
        # cell edges of the particle domain [dr/2, R - dr/2] x [dz/2, Z - dz/2]
        lo_r = torch.where(ic == 0, torch.full_like(ic, 0, dtype=torch.float64) + dr / 2,
                           ic.to(torch.float64) * dr)
        hi_r = torch.where(ic == nrc - 1, torch.full_like(lo_r, self.r_size - dr / 2),
                           (ic + 1).to(torch.float64) * dr)
        del ic
        u = torch.rand(n, generator=gen, device=dev, dtype=torch.float64)
        r = torch.sqrt(lo_r * lo_r + u * (hi_r * hi_r - lo_r * lo_r))
        vol = math.pi * (hi_r * hi_r - lo_r * lo_r)
        del lo_r, hi_r
        lo_z = torch.where(kc == 0, torch.full_like(u, dz / 2), kc.to(torch.float64) * dz)
        hi_z = torch.where(kc == nzc - 1, torch.full_like(u, self.z_size - dz / 2),
                           (kc + 1).to(torch.float64) * dz)
        del kc
        torch.rand(n, generator=gen, device=dev, dtype=torch.float64, out=u)
        z = lo_z + u * (hi_z - lo_z)
        vol *= hi_z - lo_z
        zc = 0.5 * (lo_z + hi_z)
        del lo_z, hi_z
        if self.z_ramp > 0:
            dens = self.n_max * torch.clamp(zc / self.z_ramp, max=1.0)
        else:
            dens = torch.full_like(zc, self.n_max)
        w = dens * vol / ppc
        del dens, vol, zc
        sig = math.sqrt(self.t_ev * EL_CHARGE / EL_MASS)
        v = [torch.randn(n, generator=gen, device=dev, dtype=torch.float64) * sig
             for _ in range(3)]
        torch.cuda.synchronize(dev)  # the library reads them on its own stream
        sim.add_species_device(-1.0, 1.0, r, z, v[0], v[1], v[2], w)
        del v
        zero = torch.zeros(n, device=dev, dtype=torch.float64)
        torch.cuda.synchronize(dev)
        sim.add_species_device(1.0, self.ion_mass_me, r, z, zero, zero, zero, w)
        del r, z, w, zero, u
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()


def large_config(seed=1003, n_grid_r=513, n_grid_z=4097, r_size=0.1, z_size=0.8, ppc=64,
                 density=1e17, ramp_fraction=0.2, steps=2000, beam_gamma=10.0,
                 beam_radius=5e-3, beam_length=0.02, beam_density=5e16, pusher="vay",
                 sort_interval=20, host_plasma=False):
    """Large FP32 case: 512x4096 cells, electrons and protons at 64 ppc
    (268,435,456 particles, generated on the GPU), density ramped linearly
    from 0 to 1e17 m^-3 over the first 20% of z, gamma = 10 electron bunch
    (r 5 mm, length 2 cm, 5e16 m^-3) with the Vay pusher, particles re-sorted
    by cell every 20 steps.  host_plasma=True builds the plasma as host
    arrays instead (same conventions, numpy generator; for reduced ppc,
    where the same particles must also reach the oracle)."""
    dr = r_size / (n_grid_r - 1)
    dz = z_size / (n_grid_z - 1)
    z_ramp = ramp_fraction * z_size
    species, plasma = [], None
    if host_plasma:
        rng = np.random.default_rng(seed)
        species = thermal_plasma(rng, r_size, z_size, n_grid_r, n_grid_z, ppc,
                                 lambda zc: density * np.minimum(zc / z_ramp, 1.0), 1.0)
    else:
        plasma = DevicePlasma(seed, r_size, z_size, n_grid_r, n_grid_z, ppc, density, z_ramp)
    bunch_cells = (beam_radius / dr) * (beam_length / dz)
    beam = BeamInit(-1.0, 1.0, int(round(64 * bunch_cells)), beam_length, beam_radius,
                    beam_density, gamma_velocity(beam_gamma), 1, 0.0, "reverse", seed)
    return Workload("large_%dx%d_ppc%d" % (n_grid_r - 1, n_grid_z - 1, ppc), r_size, z_size,
                    n_grid_r, n_grid_z, courant_dt(dr, dz), steps,
                    absorbing_layer(n_grid_r, n_grid_z, 10), pusher, species, beam,
                    sort_interval, plasma)
