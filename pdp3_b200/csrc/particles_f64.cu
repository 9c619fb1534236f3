// FP64 plain form of the particle phase of one PDP3 step, fused into one
// kernel per species: gather E/H, push (Boris or Vay), first half move and
// rz rotation, azimuthal deposition at the mid-step position, second half
// move with wall reflection (plasma) or removal (bunch), charge-conserving
// r-z deposition along the step, and the velocity rotation back to (r,phi,z).
//
// The upstream code runs these as separate passes over all particles
// (ParticlesList::step_v then full_current_distribution,
// src/particlesList.cpp:20-54); the passes only read E/H and only add into J,
// so one pass per particle is equivalent.
//
// Compiled with --fmad=false and written in the upstream evaluation order so
// that every per-particle result is the CPU step's, bit for bit, except for
// log(), whose CUDA implementation may differ from glibc's by an ulp or two,
// and get_gamma_inv (see there); J is accumulated with FP64 atomics, so its
// summation order (not its terms) differs from the serial CPU loop.
//
// Algorithmic bytes per particle-step: reads r, z, v_r, v_phi, v_z, w
// (48 B), writes r, z, v_r, v_phi, v_z (40 B), plus 1 B alive flag read and
// written for bunch species.
#include "pdp3g_internal.cuh"

namespace pdp3g {

#define IDX(i, k) ((size_t)(i) * (size_t)g.nz + (size_t)(k))

__device__ __forceinline__ int cell_number(double x, double dx) {  // include/geometry.h:44
  return (int)ceil(x / dx) - 1;
}

template <typename G>
__device__ __forceinline__ void flag(const G &g, unsigned bit) { atomicOr(g.err, bit); }

// what the r-z deposition reads of the grid, passed by value to its
// out-of-line parts (no pointer to the kernel's parameters)
struct DepGrid64 {
  double *jr, *jz;
  unsigned *err;
  int nr, nz;
  double dr, dz, dt;
};

// J accumulation with a bounds check: a node outside the grid is never
// written; it raises ERR_OUT_OF_GRID instead.
template <typename G>
__device__ __forceinline__ void add(const G &g, double *base, int i, int k, double v) {
  if ((unsigned)i >= (unsigned)g.nr || (unsigned)k >= (unsigned)g.nz) {
    flag(g, ERR_OUT_OF_GRID);
    return;
  }
  atomicAdd(base + IDX(i, k), v);
}

// Clamps a gather/deposit cell to [0, n-2] so its +1 neighbour exists;
// a clamp from above raises ERR_OUT_OF_GRID.
__device__ __forceinline__ int clamp_cell(const GridDev &g, int c, int n) {
  if (c < 0) return 0;  // the upstream "sometimes it gives -1" workaround
  if (c > n - 2) {
    flag(g, ERR_OUT_OF_GRID);
    return n - 2;
  }
  return c;
}

// One staggered component, 4 nodes: EField::get_field src/eField.cpp:204-316,
// HField::get_field src/hField.cpp:159-267.
__device__ __forceinline__ double gather_one(const GridDev &g, const double *__restrict__ f,
                                             double radius, double longitude, bool rhalf,
                                             bool zhalf) {
  const double dr = g.dr, dz = g.dz;
  const double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr;
  int i_r = rhalf ? cell_number(radius - 0.5 * dr, dr) : cell_number(radius, dr);
  int k_z = zhalf ? cell_number(longitude - 0.5 * dz, dz) : cell_number(longitude, dz);
  i_r = clamp_cell(g, i_r, g.nr);
  k_z = clamp_cell(g, k_z, g.nz);
  double vol_1, vol_2, r2, dz1, dz2;
  if (rhalf) {
    vol_1 = PI * dz * dr * dr * 2.0 * (i_r + 1);
    vol_2 = PI * dz * dr * dr * 2.0 * (i_r + 3);
    r2 = (i_r + 1) * dr;
  } else {
    if (radius > dr)
      vol_1 = PI * dz * dr * dr * 2.0 * (i_r);
    else
      vol_1 = PI * (dz) * (dr) * (dr) / 4.;
    r2 = (i_r + 0.5) * dr;
    vol_2 = PI * dz * dr * dr * 2.0 * (i_r + 2);
  }
  if (zhalf) {
    dz1 = (k_z + 1.5) * dz - longitude;
    dz2 = longitude - (k_z + 0.5) * dz;
  } else {
    dz1 = (k_z + 1) * dz - longitude;
    dz2 = longitude - k_z * dz;
  }
  const double f00 = __ldg(f + IDX(i_r, k_z)), f10 = __ldg(f + IDX(i_r + 1, k_z));
  const double f01 = __ldg(f + IDX(i_r, k_z + 1)), f11 = __ldg(f + IDX(i_r + 1, k_z + 1));
  double acc = 0;
  acc = acc + f00 * PI * (dz1) * ((r2) * (r2) - (r1) * (r1)) / vol_1;
  acc = acc + f10 * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / vol_2;
  acc = acc + f01 * PI * (dz2) * ((r2) * (r2) - (r1) * (r1)) / vol_1;
  acc = acc + f11 * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / vol_2;
  return acc;
}

__device__ __forceinline__ double dot3(const double *a, const double *b) {
  double res = 0;
  res += a[0] * b[0];
  res += a[1] * b[1];
  res += a[2] * b[2];
  return res;
}

// lib::get_gamma, src/lib.cpp:45-70 (v > c raises ERR_V_GE_C instead of exit)
__device__ __forceinline__ double get_gamma(const GridDev &g, double sq_velocity) {
  const double beta = sq_velocity / LIGHT_SPEED_POW_2;
  if (beta > 1) {
    flag(g, ERR_V_GE_C);
    return 1.0;
  }
  const double gamma = 1 / sqrt(1.0 - beta);
  if (isinf(gamma)) return 1e100;
  return gamma;
}

// lib::get_gamma_inv, src/lib.cpp:72-80: pow(x, -0.5) there.  Here y =
// 1/sqrt(x) refined by one Newton step whose residual 1 - x y^2 is formed
// exactly with fused multiply-adds (y^2 = t + h split by fma, Markstein's
// method).  On the host it equals glibc's pow(x, -0.5) for all but 0.05% of
// 2e7 random x in [1, 100] (plain 1/sqrt(x): 40%); on the device it is closer
// to the CPU step than CUDA's pow (one-step deviation of the wake and large
// grids from the oracle 1e-16 instead of 1e-14), at a fraction of pow's
// cost on the FP64 pipe.  The fma calls are explicit: they are not
// contractions, which --fmad=false disables.
__device__ __forceinline__ double get_gamma_inv(double sq_velocity) {
  const double x = 1.0 + sq_velocity / LIGHT_SPEED_POW_2;
  const double y = 1.0 / sqrt(x);
  const double t = y * y;
  const double h = fma(y, y, -t);  // y * y = t + h exactly
  double r = fma(-x, t, 1.0);
  r = fma(-x, h, r);               // 1 - x y^2
  return fma(0.5 * y, r, y);
}

// Particles::boris_pusher_single, src/particles.cpp:1025-1150
__device__ __forceinline__ void boris(const GridDev &g, double q, double m, double *e,
                                      double *b, double *v, bool rel) {
  const double const1 = q * g.dt / (2 * m);
  double velocity[3], vtmp[3];
#pragma unroll
  for (int i = 0; i < 3; i++) e[i] *= const1;
#pragma unroll
  for (int i = 0; i < 3; i++) b[i] *= MAGN_CONST * const1;
#pragma unroll
  for (int i = 0; i < 3; i++) velocity[i] = (fabs(v[i]) < MNZL) ? 0 : v[i];
  if (rel) {
    const double gm = get_gamma(g, dot3(velocity, velocity));
#pragma unroll
    for (int i = 0; i < 3; i++) velocity[i] *= gm;
  }
#pragma unroll
  for (int i = 0; i < 3; i++) velocity[i] += e[i];
  if (rel) {
    const double gm = get_gamma_inv(dot3(velocity, velocity));
#pragma unroll
    for (int i = 0; i < 3; i++) b[i] *= gm;
  }
  const double const2 = 2. / (1. + dot3(b, b));
#pragma unroll
  for (int i = 0; i < 3; i++) vtmp[i] = velocity[i];
  velocity[0] = vtmp[0] + const2 * ((vtmp[1] - vtmp[0] * b[2] + vtmp[2] * b[0]) * b[2] -
                                    (vtmp[2] + vtmp[0] * b[1] - vtmp[1] * b[0]) * b[1]);
  velocity[1] = vtmp[1] + const2 * (-(vtmp[0] + vtmp[1] * b[2] - vtmp[2] * b[1]) * b[2] +
                                    (vtmp[2] + vtmp[0] * b[1] - vtmp[1] * b[0]) * b[0]);
  velocity[2] = vtmp[2] + const2 * ((vtmp[0] + vtmp[1] * b[2] - vtmp[2] * b[1]) * b[1] -
                                    (vtmp[1] - vtmp[0] * b[2] + vtmp[2] * b[0]) * b[0]);
#pragma unroll
  for (int i = 0; i < 3; i++) velocity[i] += e[i];
  if (rel) {
    const double gm = get_gamma_inv(dot3(velocity, velocity));
#pragma unroll
    for (int i = 0; i < 3; i++) velocity[i] *= gm;
  }
#pragma unroll
  for (int i = 0; i < 3; i++) v[i] = velocity[i];
}

// Particles::vay_pusher_single, src/particles.cpp:1152-1254, as written
__device__ __forceinline__ void vay(const GridDev &g, double q, double m, double *e, double *b,
                                    double *v) {
  const double const1 = q * g.dt / (2 * m);
  double velocity[3], vtmp[3];
#pragma unroll
  for (int i = 0; i < 3; i++) e[i] *= 2 * const1;
#pragma unroll
  for (int i = 0; i < 3; i++) b[i] *= MAGN_CONST * const1;
#pragma unroll
  for (int i = 0; i < 3; i++) velocity[i] = (fabs(v[i]) < MNZL) ? 0 : v[i];
  double gamma = get_gamma(g, dot3(velocity, velocity));
#pragma unroll
  for (int i = 0; i < 3; i++) velocity[i] *= gamma;
#pragma unroll
  for (int i = 0; i < 3; i++) vtmp[i] = velocity[i];
#pragma unroll
  for (int i = 0; i < 3; i++) b[i] *= 2 * const1;
#pragma unroll
  for (int i = 0; i < 3; i++) velocity[i] += e[i];
#pragma unroll
  for (int i = 0; i < 3; i++) b[i] *= const1;
  gamma = get_gamma_inv(dot3(vtmp, vtmp));
  velocity[0] += gamma * (vtmp[1] * b[2] - vtmp[2] * b[1]);
  velocity[1] += gamma * (vtmp[2] * b[0] - vtmp[0] * b[2]);
  velocity[2] += gamma * (vtmp[0] * b[1] - vtmp[1] * b[0]);
  gamma = get_gamma_inv(dot3(velocity, velocity));
  double alpha = 1. / gamma / gamma;
  const double B2 = dot3(b, b);
  double sg = alpha - B2;
  const double vb = dot3(velocity, b);
  const double us2 = vb * vb;  // pow(x, 2), src/particles.cpp:1231
  alpha = 1. / sqrt(0.5 * (sg + sqrt(sg * sg + 4. * (B2 + us2))));
#pragma unroll
  for (int i = 0; i < 3; i++) b[i] *= alpha;
  sg = 1. / (1. + dot3(b, b));
  alpha = dot3(velocity, b);
  vtmp[0] = sg * (velocity[0] + alpha * b[0] + b[2] * velocity[1] - b[1] * velocity[2]);
  vtmp[1] = sg * (velocity[1] + alpha * b[1] + b[0] * velocity[2] - b[2] * velocity[0]);
  vtmp[2] = sg * (velocity[2] + alpha * b[2] + b[1] * velocity[0] - b[0] * velocity[1]);
  gamma = get_gamma_inv(dot3(vtmp, vtmp));
#pragma unroll
  for (int i = 0; i < 3; i++) v[i] = vtmp[i] * gamma;
}

// Particles::azimuthal_current_distribution, src/particles.cpp:688-784
__device__ __forceinline__ void deposit_jphi(const GridDev &g, double q, double r, double z,
                                             double vphi) {
  const double dr = g.dr, dz = g.dz;
  int r_i = cell_number(r, dr), z_k = cell_number(z, dz);
  if (r_i < 0) r_i = 0;
  if (z_k < 0) z_k = 0;
  const double r1 = r - 0.5 * dr, r2 = (r_i + 0.5) * dr, r3 = r + 0.5 * dr;
  const double ro_v = q / (2. * PI * dz * dr * r);
  double v_1;
  if (r > dr)
    v_1 = PI * dz * dr * dr * 2.0 * (r_i);
  else
    v_1 = PI * (dz) * (dr) * (dr) / 4.;
  const double v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
  const double dz1 = (z_k + 0.5) * dz - (z - 0.5 * dz);
  const double dz2 = (z + 0.5 * dz) - (z_k + 0.5) * dz;
  double rho;
  rho = ro_v * PI * (dz1) * ((r2) * (r2) - (r1) * (r1)) / v_1;
  add(g, g.jphi, r_i, z_k, rho * vphi);
  rho = ro_v * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / v_2;
  add(g, g.jphi, r_i + 1, z_k, rho * vphi);
  rho = ro_v * PI * (dz2) * ((r2) * (r2) - (r1) * (r1)) / v_1;
  add(g, g.jphi, r_i, z_k + 1, rho * vphi);
  rho = ro_v * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / v_2;
  add(g, g.jphi, r_i + 1, z_k + 1, rho * vphi);
}

// include/particles.h:169-178
#define DENS_R(q, r, dr, dz, dt) ((q) / (2 * PI * (r) * (dr) * (dz) * (dt) * 2 * (dr)))
#define DENS_Z(q, r, dr, dz, dt) ((q) / (2 * PI * (r) * (dr) * (dz) * (dt) * (dz)))
#define DENS_STRICT(q, r, dr, dz, dt) ((q) / (PI * 4. * (r) * (dz) * (dz) * (dr) * (dt)))

// Particles::simple_current_distribution, src/particles.cpp:333-474
template <typename G>
__device__ __forceinline__ void simple_current(const G &g, double q, double radius_new,
                                            double longitude_new, double radius_old,
                                            double longitude_old, int i_n, int k_n) {
  const double dr = g.dr, dz = g.dz, delta_t = g.dt;
  double wj, dens;
  const double delta_r = radius_new - radius_old;
  const double delta_z = longitude_new - longitude_old;
  if ((fabs(delta_r) < MNZL) || (fabs(delta_z) < MNZL)) return;
  double k = delta_r / delta_z;
  double b = radius_old;
  if (i_n >= 1) {
    const double lg = log((k * delta_z + b) / b);
    dens = DENS_R(q, i_n * dr, dr, dz, delta_t);
    wj = dens * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b +
                 dr * dr / k * ((i_n + 0.5) * (i_n + 0.5) - 0.25) * lg);
    add(g, g.jz, i_n, k_n, wj);
    dens = DENS_R(q, (i_n + 1) * dr, dr, dz, delta_t);
    wj = dens * (k * delta_z * delta_z / 2. + delta_z * b + delta_z * dr +
                 dr * dr / k * (0.25 - (i_n + 0.5) * (i_n + 0.5)) * lg);
    add(g, g.jz, i_n + 1, k_n, wj);
  } else {
    dens = q / (2. * PI * dr / 4. * dr * dz * delta_t * dr);
    wj = dens * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b);
    add(g, g.jz, i_n, k_n, wj);
    dens = DENS_R(q, dr, dr, dz, delta_t);
    wj = dens * (k * delta_z * delta_z / 2. + delta_z * dr + delta_z * b);
    add(g, g.jz, i_n + 1, k_n, wj);
  }
  k = -delta_z / delta_r;
  const double r0 = (i_n + 0.5) * dr;
  const double r1 = radius_old;
  b = (k_n + 1.) * dz - longitude_old;
  dens = DENS_Z(q, r0, dr, dz, delta_t);
  const double lr = log((radius_old + delta_r) / radius_old);
  wj = dens * (r0 * k * delta_r + k / 2. * delta_r * (radius_old + delta_r / 2.) +
               0.5 * delta_r * (b - k * (2 * r0 + r1)) +
               delta_r * (b - k * r1) * (4 * r0 * r0 - dr * dr) /
                   (8 * radius_old * (radius_old + delta_r)) +
               (k * (r0 * r0 / 2. - dr * dr / 8.)) * lr);
  add(g, g.jr, i_n, k_n, wj);
  b = longitude_old - k_n * dz;
  wj = dens * (-r0 * k * delta_r - k / 2. * delta_r * (radius_old + delta_r / 2.) +
               0.5 * delta_r * (b + k * (2 * r0 + r1)) +
               delta_r * (b + k * r1) * (4 * r0 * r0 - dr * dr) /
                   (8 * radius_old * (radius_old + delta_r)) -
               (k * (r0 * r0 / 2. - dr * dr / 8.)) * lr);
  add(g, g.jr, i_n, k_n + 1, wj);
}

// Particles::strict_motion_weighting, src/particles.cpp:786-988 (a step with
// no radial or no axial motion), out of line
static __device__ __noinline__ void strict_motion(DepGrid64 g, double q, double radius_new,
                                                  double longitude_new, double radius_old,
                                                  double longitude_old) {
  const double dr = g.dr, dz = g.dz, delta_t = g.dt;
  int i_n = cell_number(radius_new, dr), k_n = cell_number(longitude_new, dz);
  int i_o = cell_number(radius_old, dr), k_o = cell_number(longitude_old, dz);
  if (i_n < 0) i_n = 0;
  if (k_n < 0) k_n = 0;
  if (i_o < 0) i_o = 0;
  if (k_o < 0) k_o = 0;
  if ((fabs(radius_new - radius_old) < MNZL) && (fabs(longitude_new - longitude_old) < MNZL))
    return;
  if (fabs(radius_new - radius_old) < MNZL) {
    double delta_z, wj_lower, wj_upper;
    const double value_part = 2. * PI * radius_new * dr * dz;
    const double r1 = radius_new - 0.5 * dr, r2 = (i_n + 0.5) * dr, r3 = radius_new + 0.5 * dr;
    if (i_n == 0)
      wj_lower = q / (delta_t * PI * dr * dr / 4.) * PI * (r2 * r2 - r1 * r1) / value_part;
    else
      wj_lower = q / (delta_t * 2. * PI * i_n * dr * dr) * PI * (r2 * r2 - r1 * r1) / value_part;
    wj_upper = q / (delta_t * 2 * PI * (i_n + 1) * dr * dr) * PI * (r3 * r3 - r2 * r2) / value_part;
    add(g, g.jr, i_n, k_n, 0.);
    add(g, g.jr, i_n, k_n + 1, 0.);
    switch (k_n - k_o) {
      case 0:
        delta_z = longitude_new - longitude_old;
        add(g, g.jz, i_n, k_n, wj_lower * delta_z);
        add(g, g.jz, i_n + 1, k_n, wj_upper * delta_z);
        break;
      case 1:
        delta_z = k_n * dz - longitude_old;
        add(g, g.jz, i_n, k_n - 1, wj_lower * delta_z);
        add(g, g.jz, i_n + 1, k_n - 1, wj_upper * delta_z);
        delta_z = longitude_new - k_n * dz;
        add(g, g.jz, i_n, k_n, wj_lower * delta_z);
        add(g, g.jz, i_n + 1, k_n, wj_upper * delta_z);
        break;
      case -1:
        delta_z = (k_n + 1) * dz - longitude_old;
        add(g, g.jz, i_n, k_n + 1, wj_lower * delta_z);
        add(g, g.jz, i_n + 1, k_n + 1, wj_upper * delta_z);
        delta_z = longitude_new - (k_n + 1) * dz;
        add(g, g.jz, i_n, k_n, wj_lower * delta_z);
        add(g, g.jz, i_n + 1, k_n, wj_upper * delta_z);
        break;
    }
  } else if (fabs(longitude_new - longitude_old) < MNZL) {
    double wj, delta_r, left_delta_z, right_delta_z, r0, dens;
    switch (i_n - i_o) {
      case 0:
        delta_r = radius_new - radius_old;
        left_delta_z = (k_n + 1) * dz - longitude_new;
        right_delta_z = longitude_new - k_n * dz;
        r0 = (i_n + 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / (radius_old + delta_r) + r0 * r0 / radius_old +
                     dr * dr / (4. * (radius_old + delta_r)) - dr * dr / (4. * radius_old));
        add(g, g.jr, i_n, k_n, wj * left_delta_z);
        add(g, g.jr, i_n, k_n + 1, wj * right_delta_z);
        break;
      case 1:
        delta_r = (i_n)*dr - radius_old;
        left_delta_z = (k_n + 1) * dz - longitude_new;
        right_delta_z = longitude_new - k_n * dz;
        r0 = (i_n - 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / (radius_old + delta_r) + r0 * r0 / radius_old +
                     dr * dr / (4. * (radius_old + delta_r)) - dr * dr / (4. * radius_old));
        add(g, g.jr, i_n - 1, k_n, wj * left_delta_z);
        add(g, g.jr, i_n - 1, k_n + 1, wj * right_delta_z);
        delta_r = radius_new - i_n * dr;
        r0 = (i_n + 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        // (r0*r0/i_n)*dr as the upstream expression groups it (src/particles.cpp:941)
        wj = dens * (delta_r - r0 * r0 / (i_n * dr + delta_r) + r0 * r0 / i_n * dr +
                     dr * dr / (4. * (i_n * dr + delta_r)) - dr * dr / (4. * i_n * dr));
        add(g, g.jr, i_n, k_n, wj * left_delta_z);
        add(g, g.jr, i_n, k_n + 1, wj * right_delta_z);
        break;
      case -1:
        delta_r = (i_n + 1) * dr - radius_old;
        left_delta_z = (k_n + 1) * dz - longitude_new;
        right_delta_z = longitude_new - k_n * dz;
        r0 = (i_n + 1.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / (radius_old + delta_r) + r0 * r0 / radius_old +
                     dr * dr / (4. * (radius_old + delta_r)) - dr * dr / (4. * radius_old));
        add(g, g.jr, i_n + 1, k_n, wj * left_delta_z);
        add(g, g.jr, i_n + 1, k_n + 1, wj * right_delta_z);
        delta_r = radius_new - (i_n + 1) * dr;
        r0 = (i_n + 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / ((i_n + 1) * dr + delta_r) + r0 * r0 / (i_n + 1) * dr +
                     dr * dr / (4. * ((i_n + 1) * dr + delta_r)) - dr * dr / (4. * (i_n + 1) * dr));
        add(g, g.jr, i_n, k_n, wj * left_delta_z);
        add(g, g.jr, i_n, k_n + 1, wj * right_delta_z);
        break;
    }
  }
}

// Particles::current_distribution (src/particles.cpp:476-686), the cases of a
// step that crosses one or two cell faces (2 or 3 pieces).  Out of line, as
// strict_motion is: few steps cross a face (about one in a thousand at
// thermal speeds), and the hot loop then keeps none of their code (64-ppc
// wake case: 9.57 -> 9.36 ms per particle phase, the results unchanged).
static __device__ __noinline__ void deposit_rz_cross(DepGrid64 g, double q, double r_n,
                                                     double z_n, double r_o, double z_o, int i_n,
                                                     int k_n, int i_o, int k_o, int res_cell) {
  const double dr = g.dr, dz = g.dz;
  if (res_cell == 1) {
    if ((i_n != i_o) && (k_n == k_o)) {
      if (r_o > (i_n + 1) * dr) {
        const double a = (r_o - r_n) / (z_o - z_n);
        const double r_b = (i_n + 1) * dr;
        const double d_r = r_b - r_n;
        const double z_b = z_n + d_r / a;
        simple_current(g, q, r_b, z_b, r_o, z_o, i_n + 1, k_n);
        simple_current(g, q, r_n, z_n, r_b, z_b, i_n, k_n);
      } else {
        const double a = (r_n - r_o) / (z_n - z_o);
        const double r_b = (i_n)*dr;
        const double d_r = r_b - r_o;
        const double z_b = z_o + d_r / a;
        simple_current(g, q, r_b, z_b, r_o, z_o, i_n - 1, k_n);
        simple_current(g, q, r_n, z_n, r_b, z_b, i_n, k_n);
      }
    } else if ((i_n == i_o) && (k_n != k_o)) {
      if (z_o < k_n * dz) {
        const double z_b = k_n * dz;
        const double d_z = z_b - z_o;
        const double a = (r_n - r_o) / (z_n - z_o);
        const double r_b = r_o + a * d_z;
        simple_current(g, q, r_b, z_b, r_o, z_o, i_n, k_n - 1);
        simple_current(g, q, r_n, z_n, r_b, z_b, i_n, k_n);
      } else {
        const double z_b = (k_n + 1) * dz;
        const double d_z = z_b - z_n;
        const double a = (r_o - r_n) / (z_o - z_n);
        const double r_b = r_n + a * d_z;
        simple_current(g, q, r_b, z_b, r_o, z_o, i_n, k_n + 1);
        simple_current(g, q, r_n, z_n, r_b, z_b, i_n, k_n);
      }
    }
  } else if (res_cell == 2) {
    if (i_o < i_n) {
      if (k_o < k_n) {
        const double a = (r_n - r_o) / (z_n - z_o);
        const double r1 = i_n * dr;
        const double dz1 = (r1 - r_o) / a;
        const double z1 = z_o + dz1;
        const double z2 = k_n * dz;
        const double dr2 = (z2 - z_o) * a;
        const double r2 = r_o + dr2;
        if (z1 < k_n * dz) {
          simple_current(g, q, r1, z1, r_o, z_o, i_n - 1, k_n - 1);
          simple_current(g, q, r2, z2, r1, z1, i_n, k_n - 1);
          simple_current(g, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 > k_n * dz) {
          simple_current(g, q, r2, z2, r_o, z_o, i_n - 1, k_n - 1);
          simple_current(g, q, r1, z1, r2, z2, i_n - 1, k_n);
          simple_current(g, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      } else {
        const double a = (r_n - r_o) / (z_n - z_o);
        const double r1 = i_n * dr;
        const double dz1 = (r1 - r_o) / a;
        const double z1 = z_o + dz1;
        const double z2 = (k_n + 1) * dz;
        const double dr2 = -(z_o - z2) * a;
        const double r2 = r_o + dr2;
        if (z1 > (k_n + 1) * dz) {
          simple_current(g, q, r1, z1, r_o, z_o, i_n - 1, k_n + 1);
          simple_current(g, q, r2, z2, r1, z1, i_n, k_n + 1);
          simple_current(g, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 < (k_n + 1) * dz) {
          simple_current(g, q, r2, z2, r_o, z_o, i_n - 1, k_n + 1);
          simple_current(g, q, r1, z1, r2, z2, i_n - 1, k_n);
          simple_current(g, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      }
    } else if (i_o > i_n) {
      if (k_o < k_n) {
        const double a = (r_n - r_o) / (z_n - z_o);
        const double r1 = (i_n + 1) * dr;
        const double dz1 = -(r_o - r1) / a;
        const double z1 = z_o + dz1;
        const double z2 = k_n * dz;
        const double dr2 = -(z2 - z_o) * a;
        const double r2 = r_o - dr2;
        if (z1 < (k_n)*dz) {
          simple_current(g, q, r1, z1, r_o, z_o, i_n + 1, k_n - 1);
          simple_current(g, q, r2, z2, r1, z1, i_n, k_n - 1);
          simple_current(g, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 > (k_n)*dz) {
          simple_current(g, q, r2, z2, r_o, z_o, i_n + 1, k_n - 1);
          simple_current(g, q, r1, z1, r2, z2, i_n + 1, k_n);
          simple_current(g, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      } else if (k_o > k_n) {
        const double a = (r_o - r_n) / (z_o - z_n);
        const double r1 = (i_n + 1) * dr;
        const double dz1 = (r1 - r_n) / a;
        const double z1 = z_n + dz1;
        const double z2 = (k_n + 1) * dz;
        const double dr2 = (z2 - z_n) * a;
        const double r2 = r_n + dr2;
        if (z1 > (k_n + 1) * dz) {
          simple_current(g, q, r1, z1, r_o, z_o, i_n + 1, k_n + 1);
          simple_current(g, q, r2, z2, r1, z1, i_n, k_n + 1);
          simple_current(g, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 < (k_n + 1) * dz) {
          simple_current(g, q, r2, z2, r_o, z_o, i_n + 1, k_n + 1);
          simple_current(g, q, r1, z1, r2, z2, i_n + 1, k_n);
          simple_current(g, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      }
    }
  }
}

// Particles::current_distribution, src/particles.cpp:476-686: the segment
// (r_o, z_o) -> (r_n, z_n) is split at cell faces into 1, 2 or 3 pieces.
__device__ __forceinline__ void deposit_rz(const GridDev &g, double q, double r_n, double z_n,
                                           double r_o, double z_o) {
  const double dr = g.dr, dz = g.dz;
  int i_n = cell_number(r_n, dr), k_n = cell_number(z_n, dz);
  int i_o = cell_number(r_o, dr), k_o = cell_number(z_o, dz);
  if (i_n < 0) i_n = 0;
  if (k_n < 0) k_n = 0;
  if (i_o < 0) i_o = 0;
  if (k_o < 0) k_o = 0;
  if (r_o == (i_o + 1) * dr) i_o = i_n;
  if (z_o == (k_o + 1) * dz) k_o = k_n;
  if (r_n == (i_n + 1) * dr) i_n = i_o;
  if (z_n == (k_n + 1) * dz) k_n = k_o;
  const int res_cell = abs(i_n - i_o) + abs(k_n - k_o);
  if ((fabs(r_n - r_o) < MNZL) || (fabs(z_n - z_o) < MNZL)) {
    strict_motion(DepGrid64{g.jr, g.jz, g.err, g.nr, g.nz, g.dr, g.dz, g.dt}, q, r_n, z_n, r_o,
                  z_o);
    return;
  }
  if (res_cell == 0) {
    simple_current(g, q, r_n, z_n, r_o, z_o, i_n, k_n);
  } else {
    deposit_rz_cross(DepGrid64{g.jr, g.jz, g.err, g.nr, g.nz, g.dr, g.dz, g.dt}, q, r_n, z_n, r_o,
                     z_o, i_n, k_n, i_o, k_o, res_cell);
  }
}

// The fused particle phase for one species.
// 4 CTAs of 256 threads per SM (64 registers): the kernel is latency-bound
// and gains more from residency than it loses to the few spilled registers.
// PUSHER: 0 relativistic Boris, 1 Vay, 2 classic Boris (one kernel per
// pusher, as the FP32 form has).
template <int PUSHER>
__global__ void __launch_bounds__(256, 4) k_push_deposit_f64(GridDev g, SpeciesDev s) {
  const double half_dt = g.dt / 2.;
  const double dr = g.dr, dz = g.dz;
  const double radius_wall = g.r_size - dr / 2.;
  const double longitude_wall = g.z_size - dz / 2.;
  const double half_dr = dr / 2., half_dz = dz / 2.;
  const double radius_wallX2 = radius_wall * 2., longitude_wallX2 = longitude_wall * 2.;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x) {
    if (s.alive != nullptr && !s.alive[p]) continue;
    double r = s.r[p], z = s.z[p];
    if (isnan(r) || isinf(r) || isnan(z) || isinf(z)) {
      flag(g, ERR_NAN);
      continue;
    }
    double v[3] = {s.vr[p], s.vphi[p], s.vz[p]};
    const double w = s.w[p];
    const double q = s.charge * w, m = s.mass * w;
    // gather (E at time n, H at n+1/2 from the half-time arrays)
    // The six components in one rolled loop: every component's arithmetic
    // is the same as six inlined calls, but the kernel holds one copy of it
    // (instruction-cache misses were the kernel's top stall).
    double e[3], b[3];
    {
      double g0 = 0, g1 = 0, g2 = 0, g3 = 0, g4 = 0, g5 = 0;
#pragma unroll 1
      for (int c = 0; c < 6; c++) {
        const double *f =
            c == 0 ? g.er
                   : (c == 1 ? g.ez
                             : (c == 2 ? g.ephi : (c == 3 ? g.hzh : (c == 4 ? g.hrh : g.hphih))));
        const bool rh = (c == 0) || (c == 3) || (c == 5);
        const bool zh = (c == 1) || (c == 4) || (c == 5);
        const double val = gather_one(g, f, r, z, rh, zh);
        g0 = c == 0 ? val : g0;
        g1 = c == 1 ? val : g1;
        g2 = c == 2 ? val : g2;
        g3 = c == 3 ? val : g3;
        g4 = c == 4 ? val : g4;
        g5 = c == 5 ? val : g5;
      }
      e[0] = g0;
      e[2] = g1;
      e[1] = g2;
      b[2] = g3;
      b[0] = g4;
      b[1] = g5;
    }
    if (PUSHER == 1)
      vay(g, q, m, e, b, v);
    else
      boris(g, q, m, e, b, v, PUSHER == 0);
    // dump_position_to_old + half_step_pos + back_position_to_rz
    // (src/particles.cpp:1256-1294); y is 0 on entry
    const double r_old = r, z_old = z;
    double x = r + v[0] * half_dt;
    double y = 0.0 + v[1] * half_dt;
    z = z + v[2] * half_dt;
    r = sqrt(x * x + y * y);
    // azimuthal current at the mid-step position (src/particles.cpp:688-784)
    deposit_jphi(g, q, r, z, v[1]);
    // second half move, reflection, rz rotation (src/particles.cpp:1355-1365)
    x = r + v[0] * half_dt;
    y = 0.0 + v[1] * half_dt;
    z = z + v[2] * half_dt;
    bool alive = true;
    if (s.kind == KIND_PLASMA) {  // src/particles.cpp:1318-1353
      if (x > radius_wall) { x = radius_wallX2 - x; v[0] = -v[0]; }
      if (z > longitude_wall) { z = longitude_wallX2 - z; v[2] = -v[2]; }
    } else {                      // src/bunch.cpp:126-153
      if (x > radius_wall) alive = false;
      if (z > longitude_wall) alive = false;
    }
    if (x < half_dr) { x = dr - x; v[0] = -v[0]; }
    if (z < half_dz) { z = dz - z; v[2] = -v[2]; }
    r = sqrt(x * x + y * y);
    const double sin_t = y / r;
    if (alive) {
      deposit_rz(g, q, r, z, r_old, z_old);
      // back_velocity_to_rz_single, src/particles.cpp:1005-1015
      const double cos_t = sqrt(1 - sin_t * sin_t);
      const double u2 = cos_t * v[0] - sin_t * v[1];
      const double v2 = sin_t * v[0] + cos_t * v[1];
      v[0] = u2;
      v[1] = v2;
    } else {
      s.alive[p] = 0;
    }
    s.r[p] = r;
    s.z[p] = z;
    s.vr[p] = v[0];
    s.vphi[p] = v[1];
    s.vz[p] = v[2];
  }
}

// Particles::charge_weighting, src/particles.cpp:101-226, with the per
// particle values of charge_weights (the upstream expressions, compiled here
// without FMA contraction like the rest of the FP64 form); runs of lanes on
// the same node block are summed in the warp before the FP64 atomics
// (charge_run_add), so only the summation order of rho differs from the CPU
// loop's.  The loop runs whole warps (every lane takes part in the sums).
__global__ void __launch_bounds__(256) k_charge_density_f64(GridDev g, SpeciesDev s,
                                                            double *rho) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); p0 < s.n;
       p0 += stride) {
    const long long p = p0 + (threadIdx.x & 31);
    bool live = p < s.n && (s.alive == nullptr || s.alive[p]);
    int r_i = 0, z_k = 0;
    double w[4] = {0, 0, 0, 0};
    if (live) {
      const double r = s.r[p], z = s.z[p], q = s.charge * s.w[p];
      if (isnan(r) || isinf(r) || isnan(z) || isinf(z)) {
        flag(g, ERR_NAN);
        live = false;
      } else {
        charge_weights(g, r, z, q, r_i, z_k, w);
      }
    }
    charge_run_add(g, rho, live, r_i, z_k, w);
  }
}

// Bunch::bunch_inject, src/bunch.cpp:104-122: particles [start, start+count)
// get z = dl * random_reverse(index, 11) + dz/2, v_z = v_beam, alive.
// inv_pow11[o] holds pow(11., -o) computed on the host with the same libm
// the CPU step uses.
__device__ __forceinline__ void inject_slot(const SpeciesDev &s, long long idx, double dl,
                                            double half_dz, double velocity,
                                            const double *inv_pow11) {
  // random_reverse(idx, 11), src/math/rand.cpp:40-53
  int int_vel = (int)floor((double)(unsigned)idx);
  double ost = 0, rr = 0;
  int order = 1;
  while (int_vel >= 1 && order < 40) {
    ost = int_vel % 11;
    rr = rr + ost * inv_pow11[order];
    int_vel = (int)((int_vel - ost) / 11);
    order = order + 1;
  }
  if (idx < s.n) {
    s.z[idx] = dl * rr + half_dz;
    s.vz[idx] = velocity;
    s.alive[idx] = 1;
  }
}

__global__ void k_bunch_inject(SpeciesDev s, long long start, long long count, double dl,
                               double half_dz, double velocity, const double *inv_pow11) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    inject_slot(s, start + i, dl, half_dz, velocity, inv_pow11);
}

// the same with the schedule evaluated from the device time (a captured step)
__global__ void k_bunch_inject_dev(SpeciesDev s, const double *d_t, double begin, double end,
                                   double dt, unsigned pis, double dl, double half_dz,
                                   double velocity, const double *inv_pow11) {
  long long start, count;
  if (!inject_window(*d_t, begin, end, dt, pis, (unsigned)s.n, start, count)) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    inject_slot(s, start + i, dl, half_dz, velocity, inv_pow11);
}

// the device copy of the context's time (a captured step reads and advances
// it; the host keeps its own copy with the same additions)
__global__ void k_set_time(double *d_t, double v) { *d_t = v; }
__global__ void k_advance_time(double *d_t, double dt) { *d_t = *d_t + dt; }

void launch_push_deposit_f64(const GridDev &g, const SpeciesDev &s, int pusher, int n_sm,
                             cudaStream_t st) {
  if (s.n <= 0) return;
  long long blocks = (s.n + 255) / 256;
  const long long cap = (long long)n_sm * 8;
  if (blocks > cap) blocks = cap;
  if (pusher == 1)
    k_push_deposit_f64<1><<<(int)blocks, 256, 0, st>>>(g, s);
  else if (pusher == 2)
    k_push_deposit_f64<2><<<(int)blocks, 256, 0, st>>>(g, s);
  else
    k_push_deposit_f64<0><<<(int)blocks, 256, 0, st>>>(g, s);
}

void launch_charge_density_f64(const GridDev &g, const SpeciesDev &s, double *rho,
                               cudaStream_t st) {
  if (s.n <= 0) return;
  long long blocks = (s.n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_charge_density_f64<<<(int)blocks, 256, 0, st>>>(g, s, rho);
}

void launch_bunch_inject_dev(const SpeciesDev &s, const double *d_t, double begin, double end,
                             double dt, unsigned pis, double dl, double half_dz, double velocity,
                             const double *inv_pow11, cudaStream_t st) {
  if (pis == 0) return;
  long long blocks = ((long long)pis + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  k_bunch_inject_dev<<<(int)blocks, 256, 0, st>>>(s, d_t, begin, end, dt, pis, dl, half_dz,
                                                  velocity, inv_pow11);
}

void launch_set_time(double *d_t, double v, cudaStream_t st) { k_set_time<<<1, 1, 0, st>>>(d_t, v); }

void launch_advance_time(double *d_t, double dt, cudaStream_t st) {
  k_advance_time<<<1, 1, 0, st>>>(d_t, dt);
}

void launch_bunch_inject(const SpeciesDev &s, long long start, long long count, double dl,
                         double half_dz, double velocity, const double *inv_pow11,
                         cudaStream_t st) {
  if (count <= 0) return;
  long long blocks = (count + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  k_bunch_inject<<<(int)blocks, 256, 0, st>>>(s, start, count, dl, half_dz, velocity, inv_pow11);
}

}  // namespace pdp3g
