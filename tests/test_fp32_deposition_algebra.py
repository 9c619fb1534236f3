"""The FP32 cell-local form's r-z deposition formulas (piece_values in
pdp3_b200/csrc/particles_f32.cuh) are the upstream closed forms of
Particles::simple_current_distribution (src/particles.cpp:333-474) rewritten
in cell-local units; this checks the rewriting in 50-digit arithmetic, where
both sides are exact, for straight segments inside one cell:

  upstream  (i >= 1):  j_z(i) = DENS_R(q, i dr) (dr dz' - k dz'^2/2 - dz' r_o
                         + dr^2/k ((i + 1/2)^2 - 1/4) log(r_n / r_o)), ...
  cell-local:          j_z(i) = kz dzeta ((1 - f_m)(2i + f_m) + i(i+1) eps)
                         / (i rho_m),  eps = atanh(s)/s - 1, s = drho/(2 rho_m)

with kz = q / (4 pi dr^2 dt), kr = q / (2 pi dr dz dt) (the kernel's species
constants), for the four deposits j_z(i,k), j_z(i+1,k), j_r(i,k),
j_r(i,k+1), at i >= 1 and on the axis cell i = 0.  CPU only."""
import mpmath as mp
import numpy as np

PI = mp.mpf("3.1415926535897932")  # the same constant on both sides


def upstream(q, dr, dz, dt, i, k, ao, an, co, cn):
    """src/particles.cpp:333-474, res_cell == 0 (particles_f64.cu restates it)."""
    r_o, r_n = (i + ao) * dr, (i + an) * dr
    z_o, z_n = (k + co) * dz, (k + cn) * dz
    d_r, d_z = r_n - r_o, z_n - z_o
    kk = d_r / d_z
    b = r_o
    out = []
    if i >= 1:
        lg = mp.log((kk * d_z + b) / b)
        dens = q / (2 * PI * (i * dr) * dr * dz * dt * 2 * dr)
        out.append(dens * (dr * d_z - kk * d_z * d_z / 2 - d_z * b +
                           dr * dr / kk * ((i + mp.mpf(0.5)) ** 2 - mp.mpf(0.25)) * lg))
        dens = q / (2 * PI * ((i + 1) * dr) * dr * dz * dt * 2 * dr)
        out.append(dens * (kk * d_z * d_z / 2 + d_z * b + d_z * dr +
                           dr * dr / kk * (mp.mpf(0.25) - (i + mp.mpf(0.5)) ** 2) * lg))
    else:
        dens = q / (2 * PI * dr / 4 * dr * dz * dt * dr)
        out.append(dens * (dr * d_z - kk * d_z * d_z / 2 - d_z * b))
        dens = q / (2 * PI * dr * dr * dz * dt * 2 * dr)
        out.append(dens * (kk * d_z * d_z / 2 + d_z * dr + d_z * b))
    kk = -d_z / d_r
    r0 = (i + mp.mpf(0.5)) * dr
    r1 = r_o
    b = (k + 1) * dz - z_o
    dens = q / (2 * PI * r0 * dr * dz * dt * dz)
    lr = mp.log((r_o + d_r) / r_o)
    out.append(dens * (r0 * kk * d_r + kk / 2 * d_r * (r_o + d_r / 2) +
                       mp.mpf(0.5) * d_r * (b - kk * (2 * r0 + r1)) +
                       d_r * (b - kk * r1) * (4 * r0 * r0 - dr * dr) / (8 * r_o * (r_o + d_r)) +
                       (kk * (r0 * r0 / 2 - dr * dr / 8)) * lr))
    b = z_o - k * dz
    out.append(dens * (-r0 * kk * d_r - kk / 2 * d_r * (r_o + d_r / 2) +
                       mp.mpf(0.5) * d_r * (b + kk * (2 * r0 + r1)) +
                       d_r * (b + kk * r1) * (4 * r0 * r0 - dr * dr) / (8 * r_o * (r_o + d_r)) -
                       (kk * (r0 * r0 / 2 - dr * dr / 8)) * lr))
    return out


def cell_local(q, dr, dz, dt, i, ao, an, co, cn):
    """piece_values of particles_f32.cuh in exact arithmetic."""
    kz = q / (4 * PI * dr * dr * dt)
    kr = q / (2 * PI * dr * dz * dt)
    drho, dzeta = an - ao, cn - co
    fi = mp.mpf(i)
    fm = (ao + an) / 2
    rho_m = fi + fm
    beta = 1 - co
    if i >= 1:
        s = drho / (2 * rho_m)
        eps = mp.atanh(s) / s - 1
        ii1 = fi * (fi + 1)
        o0 = kz * dzeta * ((1 - fm) * (2 * fi + fm) + ii1 * eps) / rho_m / fi
        o1 = kz * dzeta * (fm * (2 * fi + 1 + fm) - ii1 * eps) / rho_m / (fi + 1)
        rho_o, rho_n = fi + ao, fi + an
        q1 = drho / (rho_o * rho_n)
        q2 = dzeta * drho / 2 / rho_m / rho_n
        q3 = dzeta * eps / rho_m
        h = ii1 / 2
        inv_r0 = kr / (fi + mp.mpf(0.5))
        o2 = inv_r0 * (drho * beta / 2 - dzeta * drho / 4 + h * (q1 * beta - q2 - q3))
        o3 = inv_r0 * (drho * co / 2 + dzeta * drho / 4 + h * (q1 * co + q2 + q3))
    else:
        o0 = 8 * kz * dzeta * (1 - fm)
        o1 = kz * dzeta * (1 + fm)
        o2 = 2 * kr * (drho * beta / 2 - dzeta * drho / 4)
        o3 = 2 * kr * (drho * co / 2 + dzeta * drho / 4)
    return [o0, o1, o2, o3]


def test_cell_local_deposition_equals_upstream_closed_forms():
    with mp.workdps(50):  # other modules set mpmath's global precision
        check()


def check():
    rng = np.random.default_rng(23)
    q, dr, dz, dt = mp.mpf("-1.6e-19") * 1e6, mp.mpf("3.9e-4"), mp.mpf("3.9e-4"), \
        mp.mpf("4.6e-13")
    worst = mp.mpf(0)
    for trial in range(300):
        i = int(rng.integers(0, 200)) if trial % 5 else 0
        k = int(rng.integers(0, 2000))
        ao, an, co, cn = (mp.mpf(float(x)) for x in rng.uniform(0.02, 0.98, 4))
        want = upstream(q, dr, dz, dt, i, k, ao, an, co, cn)
        got = cell_local(q, dr, dz, dt, i, ao, an, co, cn)
        scale = max(abs(w) for w in want)
        for a, b in zip(got, want):
            worst = max(worst, abs(a - b) / scale)
    # 50 digits: the two agree to the rounding of the upstream form's
    # cancellations (observed 4e-45)
    assert worst < mp.mpf("1e-42"), worst
