"""CPU restatement of the upstream per-species diagnostics (numpy).

ORACLE ONLY (test infrastructure): tests/ use it as the checker for the
GPU diagnostics; the product never imports this module.

temperature_classic follows TemperatureClassic (src/temperatureClassic.cpp):
calc_t (:57-103) adds, per particle in slot order, |v|, v_r, v_phi, v_z and 1
into the cell (CELL_NUMBER(r, dr), CELL_NUMBER(z, dz)) = (ceil(r/dr) - 1,
ceil(z/dz) - 1) of every slot, alive or not; normalize (:130-159) gives, for
r < n_grid_r - 1 and z < n_grid_z - 1,
    v_sc^2 = ((sum |v|)^2 - |sum v|^2) / count^2,
    T = m v_sc^2 / 2                    (v_sc^2 < REL_LIMIT^2 = (5e7 m/s)^2)
    T = m c^2 (gamma(v_sc^2) - 1)      (otherwise; lib::get_gamma, src/lib.cpp:45-70)
divided by |charge| (joules to electronvolts).  Empty cells are 0/0 = NaN.

particles_density follows ParticlesDensity::calc_density
(src/particlesDensity.cpp:45-257): each particle's mass_array / EL_MASS
spread over the four nodes (i, k), (i+1, k), (i, k+1), (i+1, k+1) by the
volumes of the ring pieces it overlaps, with the three radial branches
(r > dr; r <= dr/2 with i = 0; dr/2 < r <= dr) and the upstream's expression
order (the macros of include/geometry.h:33-44).
"""
import numpy as np

LIGHT_SPEED = 3.0e8  # include/constant.h:18
REL_LIMIT = 5e7
PI = 3.1415926535897932  # include/constant.h:10
EL_MASS = 9.1e-31  # include/constant.h:14


def temperature_classic(r, z, vr, vphi, vz, dr, dz, n_grid_r, n_grid_z, mass, charge,
                        rounding=False):
    """[n_grid_r - 1, n_grid_z - 1] temperature grid in eV (mass and charge
    of one particle of the species, SI).  With rounding=True also returns a
    per-cell bound on the rounding of T by the order of the sums:
    (sum |v|)^2 - |sum v|^2 cancels, so summing count terms in another order
    moves T by up to about 2 count eps m (sum |v| / count)^2 / (2 |charge|)."""
    ri = np.ceil(np.asarray(r) / dr).astype(np.int64) - 1
    zk = np.ceil(np.asarray(z) / dz).astype(np.int64) - 1
    ok = (ri >= 0) & (ri < n_grid_r) & (zk >= 0) & (zk < n_grid_z)
    cell = ri[ok] * n_grid_z + zk[ok]
    vr, vphi, vz = (np.asarray(a, dtype=np.float64)[ok] for a in (vr, vphi, vz))
    vel = np.sqrt(vr * vr + vphi * vphi + vz * vz)
    ng = n_grid_r * n_grid_z
    sums = []
    for v in (vel, vr, vphi, vz, np.ones_like(vel)):
        acc = np.zeros(ng)
        np.add.at(acc, cell, v)  # unbuffered, in slot order per cell
        sums.append(acc.reshape(n_grid_r, n_grid_z)[:-1, :-1])
    t_sum, t_r, t_phi, t_z, cnt = sums
    v_vec_sum_2 = t_r * t_r + t_phi * t_phi + t_z * t_z
    with np.errstate(invalid="ignore", divide="ignore"):
        v_sc_sum_2 = (t_sum * t_sum - v_vec_sum_2) / (cnt * cnt)
        beta = v_sc_sum_2 / LIGHT_SPEED ** 2
        gamma = 1.0 / np.sqrt(1.0 - np.minimum(beta, 1.0))
        gamma = np.where(np.isinf(gamma), 1e100, gamma)  # lib::get_gamma at beta == 1
        gamma = np.where(beta > 1, 1.0, gamma)  # an upstream exit
        t = np.where(v_sc_sum_2 < REL_LIMIT * REL_LIMIT, mass * v_sc_sum_2 / 2,
                     mass * LIGHT_SPEED ** 2 * (gamma - 1))
    t = t / abs(charge)
    if not rounding:
        return t
    with np.errstate(invalid="ignore", divide="ignore"):
        kin = mass * (t_sum / cnt) ** 2 / 2 / abs(charge)
    return t, 4 * np.finfo(np.float64).eps * cnt * kin


def particles_density(r, z, mass_array, dr, dz, n_grid_r, n_grid_z):
    """[n_grid_r, n_grid_z] density grid (particles per m^3 in electron
    masses) with the upstream's per-particle order of the four additions."""
    r = np.asarray(r, dtype=np.float64)
    z = np.asarray(z, dtype=np.float64)
    m = np.asarray(mass_array, dtype=np.float64)
    ri = np.ceil(r / dr).astype(np.int64) - 1
    zk = np.ceil(z / dz).astype(np.int64) - 1
    a = r > dr
    b = (~a) & (r <= dr / 2.)
    c = ~(a | b)
    ri = np.where(b, 0, ri)
    rif = ri.astype(np.float64)
    dz1 = (zk + 0.5) * dz - (z - 0.5 * dz)
    dz2 = (z + 0.5 * dz) - (zk + 0.5) * dz
    r1 = np.where(b, 0.0, r - 0.5 * dr)
    r2 = (rif + 0.5) * dr
    r3 = r + 0.5 * dr
    v0 = np.where(b, PI * dz * (2. * r * r + dr * dr / 2.), 2. * PI * dz * dr * r)
    ro_p = m / EL_MASS / v0
    v1 = np.where(a, PI * dz * dr * dr * 2.0 * rif, PI * dz * dr * dr / 4.)
    v2 = PI * dz * dr * dr * 2.0 * (rif + 1)

    def ring(h, lo, hi):  # CYL_RNG_VOL
        return PI * h * (hi * hi - lo * lo)

    def axis(h):  # the r <= dr/2 inner piece
        return PI * h * (dr * dr / 2. - r * dr + r * r)

    val = np.stack([
        np.where(b, axis(dz1), ring(dz1, r1, r2)) / v1,
        ring(dz1, r2, r3) / v2,
        np.where(b, axis(dz2), ring(dz2, r1, r2)) / v1,
        ring(dz2, r2, r3) / v2], axis=1) * ro_p[:, None]
    ii = np.stack([ri, ri + 1, ri, ri + 1], axis=1)
    kk = np.stack([zk, zk, zk + 1, zk + 1], axis=1)
    ok = (ii >= 0) & (ii < n_grid_r) & (kk >= 0) & (kk < n_grid_z)
    acc = np.zeros(n_grid_r * n_grid_z)
    np.add.at(acc, (ii * n_grid_z + kk)[ok], val[ok])  # row-major: particle order
    return acc.reshape(n_grid_r, n_grid_z)
