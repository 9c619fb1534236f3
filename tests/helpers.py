"""Shared test helpers: building the same simulation in the oracle, the
compiled upstream sources and the GPU library from one Workload."""
import os

import numpy as np

from oracle import refsim
from oracle.oracle import OracleSim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "smoke_frame4.npz")

GRIDS = ["E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z", "H_r_half", "H_phi_half",
         "H_z_half", "J_r", "J_phi", "J_z"]

# upstream functional smoke template, test/functional/parameters.xml.tmpl.in
SMOKE = dict(r_size=0.25, z_size=2.0, n_grid_r=255, n_grid_z=2047, dt=1e-12, end_time=2.2e-11,
             species=[("Electrons", -1.0, 1.0, 100000, 2e16, 2.05e16, 1.0),
                      ("Ions", 1.0, 1836.0, 100000, 2e16, 2.05e16, 0.1)],
             beam=dict(charge_e=-1.0, mass_me=1.0, number_macro=1000000, bunch_length=2.0,
                       radius=0.02, density=1e15, velocity=2e8, number_bunches=1,
                       bunches_distance=0.02))


def recover_weights(q, m, charge, mass):
    """Finds w with charge*w == q and mass*w == m bit for bit (the upstream
    loader stores q = charge*n_per_macro and m = mass*n_per_macro)."""
    w0 = q / charge
    best = np.full_like(w0, np.nan)
    for d in (0, 1, -1, 2, -2, 3, -3):
        w = w0.copy()
        for _ in range(abs(d)):
            w = np.nextafter(w, np.inf if d > 0 else -np.inf)
        ok = (charge * w == q) & (mass * w == m) & np.isnan(best)
        best[ok] = w[ok]
    return best


def golden_match(values, golden):
    """6-significant-digit agreement (the golden files are printed with the
    default ostream precision; float32 storage adds < 1e-7 relative)."""
    g = golden.astype(np.float64)
    scale = max(float(np.abs(g).max()), 1e-300)
    return np.abs(values - g) <= 5.2e-6 * np.abs(g) + 1e-12 * scale


def oracle_from_workload(wl, pusher=None):
    o = OracleSim(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, pml=wl.pml,
                  pusher=pusher or wl.pusher)
    o._dr, o._dz = wl.dr, wl.dz
    o._species_mass = [s.mass_me * 9.1e-31 for s in wl.species]
    for s in wl.species:
        o.add_species(s.charge_e, s.mass_me, s.r, s.z, s.vr, s.vphi, s.vz, s.w)
    if wl.beam is not None:
        b = wl.beam
        assert b.inject_rng == "reverse", "the oracle injects with the upstream TESTMODE sequence"
        o._species_mass += [b.mass_me * 9.1e-31] * b.number_bunches
        for nb in range(b.number_bunches):
            o.add_bunch(b.charge_e, b.mass_me, b.number_macro, b.bunch_length / b.velocity,
                        b.radius, b.density, b.velocity, nb, b.bunches_distance / b.velocity)
    return o


def ref_from_workload(wl, pusher=None):
    r = refsim.RefSim(wl.r_size, wl.z_size, wl.n_grid_r, wl.n_grid_z, wl.dt, end_time=1.0,
                      pml=wl.pml, pusher=pusher or wl.pusher)
    for s in wl.species:
        r.add_species(s.name, s.charge_e, s.mass_me, s.r, s.z, s.vr, s.vphi, s.vz, s.w)
    if wl.beam is not None:
        b = wl.beam
        r.set_beam(b.charge_e, b.mass_me, b.number_macro, b.bunch_length, b.radius, b.density,
                   b.velocity, b.number_bunches, b.bunches_distance)
    return r


def seed_fields(sims, shape, seed=5, e_scale=1e4, h_scale=10.0):
    """Writes the same random E and H into every simulation (exercises the
    gather and the pushers from the first step)."""
    rng = np.random.default_rng(seed)
    for c, sc in (("E_r", e_scale), ("E_phi", e_scale), ("E_z", e_scale), ("H_r", h_scale),
                  ("H_phi", h_scale), ("H_z", h_scale)):
        a = rng.normal(0.0, sc, shape)
        for s in sims:
            s.set_field(c, a)


def rel_inf(a, b):
    """max|a-b| / max|b| (infinity norm relative to the array's scale)."""
    scale = float(np.abs(b).max())
    if scale == 0.0:
        return float(np.abs(a).max())
    return float(np.abs(a - b).max()) / scale


EPS0, MU0, C2 = 8.85e-12, 1.26e-6, 9.0e16


def diagnostics_np(sim, n_species, rho0=None):
    """The pdp3g_diagnostics quantities computed with numpy from an oracle
    simulation built by oracle_from_workload (grids and particles)."""
    nr, nz = sim.nr, sim.nz
    sig = sim.field("sigma")
    er, ez = sim.field("E_r"), sim.field("E_z")
    dr, dz = sim._dr, sim._dz
    i = np.arange(nr, dtype=np.float64)[:, None]
    vol = np.where(i == 0, np.pi * dz * dr * dr / 4.0, 2.0 * np.pi * dz * dr * dr * i)
    e2 = sum(sim.field(c) ** 2 for c in ("E_r", "E_phi", "E_z"))
    h2 = sum(sim.field(c) ** 2 for c in ("H_r", "H_phi", "H_z"))
    fe = float((0.5 * (EPS0 * e2 + MU0 * h2) * vol).sum())
    rho = sim.charge_density()
    mask = np.zeros((nr, nz), dtype=bool)
    mask[2:nr - 2, 2:nz - 2] = True
    mask &= sig == 0.0
    mask[1:, :] &= sig[:-1, :] == 0.0   # E_r(i - 1/2) stored at node (i-1, k)
    mask[:, 1:] &= sig[:, :-1] == 0.0   # E_z(k - 1/2) stored at node (i, k-1)
    div = np.zeros((nr, nz))
    div[1:, 1:] = (er[1:, 1:] * (i[1:] + 0.5) - er[:-1, 1:] * (i[1:] - 0.5)) / (i[1:] * dr) + \
        (ez[1:, 1:] - ez[1:, :-1]) / dz
    r0 = 0.0 if rho0 is None else rho0
    res = EPS0 * div - (rho - r0)
    rho_sq = sum(float((sim.charge_density(1 << s)[mask] ** 2).sum()) for s in range(n_species))
    kin, alive = 0.0, 0
    for s in range(n_species):
        p = sim.species(s)
        m = p["alive"].astype(bool)
        mass = sim._species_mass[s] * p["w"][m]
        b2 = (p["vr"][m] ** 2 + p["vphi"][m] ** 2 + p["vz"][m] ** 2) / C2
        sq = np.sqrt(1.0 - b2)
        kin += float((mass * C2 * b2 / (sq * (1.0 + sq))).sum())
        alive += int(m.sum())
    return {"field_energy": fe, "gauss_residual": float(np.sqrt((res[mask] ** 2).sum())),
            "gauss_norm": float(np.sqrt(rho_sq)), "charge_total": float((rho * vol).sum()),
            "kinetic_energy": kin, "alive": alive}
