/*
 * CPU restatement of the PDP3 per-timestep PIC loop (see pic_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU kernels, never shipped.
 *
 * Arithmetic is written in the upstream evaluation order, including the
 * order that the upstream geometry macros impose when they expand inside a
 * larger expression (include/geometry.h:33-44, include/particles.h:169-178
 * expand without outer parentheses, so for example
 *     ro_v * CYL_RNG_VOL(dz1, r1, r2) / v_1
 * evaluates as (((ro_v * PI) * dz1) * (r2*r2 - r1*r1)) / v_1).
 * Built with -O2 -ffp-contract=off and no fast-math.
 */
#define _POSIX_C_SOURCE 200809L
#include "pic_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* include/constant.h:10-27 (rounded SI values used by the upstream code) */
#define PI 3.1415926535897932
#define EPSILON0 8.85E-12
#define EL_MASS 9.1E-31
#define EL_CHARGE 1.6E-19
#define LIGHT_SPEED 3.0E8
#define MAGN_CONST 1.26E-6
#define MNZL 1e-15
/* src/lib.cpp:8 pow(LIGHT_SPEED, 2), exact in binary64 */
#define LIGHT_SPEED_POW_2 9.0e16

typedef struct {
  int n, kind;
  double charge, mass;              /* per unit weight, SI */
  double *r, *z, *vr, *vphi, *vz, *w;
  double *r_old, *z_old, *y, *sin_t;
  uint8_t *alive;
  /* bunch parameters (src/bunch.cpp:17-26) */
  double duration, bunch_number, hole_duration, density, velocity, radius;
} species_t;

typedef struct {
  int nr, nz, pusher, errors;
  double r_size, z_size, dr, dz, dt, t;
  double *g[ORC_NCOMP];
  int nsp;
  species_t sp[64];
} sim_t;

#define AT(a, i, k) (a)[(size_t)(i) * (size_t)s->nz + (size_t)(k)]

static int cell_number(double x, double dx) { return (int)ceil(x / dx) - 1; } /* geometry.h:44 */

/* ---------------------------------------------------------------- geometry */

/* Geometry::set_pml, src/geometry.cpp:56-107 */
static void set_pml(sim_t *s, double l1, double l2, double l3, double sigma1, double sigma2) {
  double *sig = s->g[ORC_SIGMA];
  int nr = s->nr, nz = s->nz;
  double dr = s->dr, dz = s->dz, r_size = s->r_size, z_size = s->z_size;
  double len_left = dz * (floor(nz * l1));
  double len_right = dz * (floor(nz * l2));
  double len_ext = dr * (floor(nr * l3));
  if ((l1 == 0) && (l2 == 0) && (l3 != 0)) {
    for (int i = 0; i < nr; i++)
      for (int k = 0; k < nz; k++)
        if (r_size - dr * i <= len_ext)
          AT(sig, i, k) = sigma1 + (sigma2 - sigma1) / pow(len_ext, 2) *
                                       pow((dr * (i + 1) - r_size + len_ext), 2);
  } else {
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nr; i++) {
        if (dz * k < len_left)
          AT(sig, i, k) = sigma1 + (sigma2 - sigma1) / pow(len_left, 2) *
                                       pow(len_left - dz * k, 2);
        if (z_size - dz * k < len_right)
          AT(sig, i, k) = sigma1 + (sigma2 - sigma1) / pow(len_right, 2) *
                                       pow(dz * (k + 1) - z_size + len_right, 2);
      }
  }
  if (l3 != 0) {
    for (int i = 0; i < nr; i++)
      for (int k = 0; k < nz; k++)
        if (r_size - dr * i <= len_ext)
          if ((r_size - dr * (i + 1) < len_ext * dz * k / len_left) &&
              (r_size - dr * i <= len_ext / len_right * (z_size - dz * k)))
            AT(sig, i, k) = sigma1 + (sigma2 - sigma1) / pow(len_ext, 2) *
                                         pow(dr * (i + 1) - r_size + len_ext, 2);
  }
}

void *orc_create(double r_size, double z_size, int n_grid_r, int n_grid_z, double dt,
                 double current_time, const double *pml, int pusher) {
  sim_t *s = (sim_t *)calloc(1, sizeof(sim_t));
  s->nr = n_grid_r;
  s->nz = n_grid_z;
  s->r_size = r_size;
  s->z_size = z_size;
  s->dr = r_size / (n_grid_r - 1); /* src/geometry.cpp:45-53 */
  s->dz = z_size / (n_grid_z - 1);
  s->dt = dt;
  s->t = current_time;
  s->pusher = pusher;
  for (int c = 0; c < ORC_NCOMP; c++)
    s->g[c] = (double *)calloc((size_t)n_grid_r * n_grid_z, sizeof(double));
  /* src/parameters.cpp:244-245 */
  if (pml && (pml[0] != 0 || pml[1] != 0 || pml[2] != 0))
    set_pml(s, pml[0], pml[1], pml[2], pml[3], pml[4]);
  return s;
}

static void free_species(species_t *p) {
  free(p->r); free(p->z); free(p->vr); free(p->vphi); free(p->vz); free(p->w);
  free(p->r_old); free(p->z_old); free(p->y); free(p->sin_t); free(p->alive);
}

void orc_destroy(void *h) {
  sim_t *s = (sim_t *)h;
  for (int c = 0; c < ORC_NCOMP; c++) free(s->g[c]);
  for (int i = 0; i < s->nsp; i++) free_species(&s->sp[i]);
  free(s);
}

static species_t *new_species(sim_t *s, int n, int kind, double charge_e, double mass_me) {
  if (s->nsp >= 64) return NULL;
  species_t *p = &s->sp[s->nsp++];
  memset(p, 0, sizeof(*p));
  p->n = n;
  p->kind = kind;
  p->charge = charge_e * EL_CHARGE; /* src/particles.cpp:30-32 */
  p->mass = mass_me * EL_MASS;
  size_t b = sizeof(double) * (size_t)(n > 0 ? n : 1);
  p->r = malloc(b); p->z = malloc(b); p->vr = malloc(b); p->vphi = malloc(b);
  p->vz = malloc(b); p->w = malloc(b); p->r_old = malloc(b); p->z_old = malloc(b);
  p->y = calloc(n > 0 ? n : 1, sizeof(double)); p->sin_t = calloc(n > 0 ? n : 1, sizeof(double));
  p->alive = calloc(n > 0 ? n : 1, 1);
  return p;
}

int orc_add_species(void *h, double charge_e, double mass_me, int n, const double *r,
                    const double *z, const double *vr, const double *vphi, const double *vz,
                    const double *w) {
  sim_t *s = (sim_t *)h;
  species_t *p = new_species(s, n, ORC_PLASMA, charge_e, mass_me);
  if (!p) return -1;
  for (int i = 0; i < n; i++) {
    p->r[i] = r[i]; p->z[i] = z[i]; p->vr[i] = vr[i]; p->vphi[i] = vphi[i]; p->vz[i] = vz[i];
    p->w[i] = w[i]; p->r_old[i] = r[i]; p->z_old[i] = z[i]; p->alive[i] = 1;
  }
  return s->nsp - 1;
}

/* src/math/rand.cpp:40-53 */
double orc_random_reverse(double x, int power) {
  int int_vel = (int)floor(x);
  double ost = 0, r = 0;
  int order = 1;
  while (int_vel >= 1) {
    ost = int_vel % power;
    r = r + ost * pow((double)power, (-order));
    int_vel = (int_vel - ost) / power;
    order = order + 1;
  }
  return r;
}

/* Bunch::Bunch in TESTMODE, src/bunch.cpp:6-80: radial positions from
   random_reverse(i, 9), weights normalised to the bunch's particle count. */
int orc_add_bunch(void *h, double charge_e, double mass_me, int n, double duration,
                  double radius, double density, double velocity, int bunch_number,
                  double hole_duration) {
  sim_t *s = (sim_t *)h;
  species_t *p = new_species(s, n, ORC_BUNCH, charge_e, mass_me);
  if (!p) return -1;
  p->duration = duration;
  p->bunch_number = bunch_number;
  p->hole_duration = hole_duration;
  p->radius = radius;
  p->density = density;
  p->velocity = velocity;
  double b_lenght = duration * velocity;
  double v_total = 0.;
  double N_total = PI * pow(radius, 2) * b_lenght * density;
  double dr = s->dr, dz = s->dz;
  for (unsigned int i = 0; i < (unsigned int)n; i++) {
    double rand_r = orc_random_reverse(i, 9);
    p->r[i] = (radius - dr) * rand_r + dr / 2;
    p->z[i] = 0.;
    p->alive[i] = 0;
    p->vr[i] = 0.; p->vphi[i] = 0.; p->vz[i] = 0.;
    if (p->r[i] > dr)
      v_total += 2 * PI * p->r[i] * dr * dz;
    else
      v_total += PI * p->r[i] * p->r[i] * dz;
  }
  double v_avg = v_total / n;
  double n_per_macro_avg = N_total / n;
  for (int i = 0; i < n; i++) {
    double norm;
    if (p->r[i] > dr / 2)
      norm = 2 * PI * p->r[i] * dr * dz / v_avg;
    else
      norm = PI * (p->r[i] * p->r[i] + p->r[i] * dr + dr * dr / 4) * dz / v_avg;
    p->w[i] = n_per_macro_avg * norm;
    p->r_old[i] = p->r[i];
    p->z_old[i] = 0.;
  }
  return s->nsp - 1;
}

/* Bunch::bunch_inject, src/bunch.cpp:87-124 (TESTMODE sequence) */
static void bunch_inject(sim_t *s, species_t *p) {
  double begin = p->duration * p->bunch_number + p->hole_duration * p->bunch_number;
  double end = begin + p->duration;
  double dl = p->velocity * s->dt;
  int steps_amount = ceil(p->duration / s->dt);
  unsigned int number = (unsigned int)p->n;
  unsigned int particles_in_step = number / steps_amount;
  int start_number = (s->t - begin) / s->dt * particles_in_step;
  double half_z_cell_size = s->dz / 2.0;
  if (s->t >= begin && s->t < end) {
    for (unsigned int i = 0; i < particles_in_step; i++) {
      double rand_z = orc_random_reverse(start_number + i, 11);
      if (i + start_number < number) {
        p->z[i + start_number] = dl * rand_z + half_z_cell_size;
        p->vz[i + start_number] = p->velocity;
        p->alive[i + start_number] = 1;
      }
    }
  }
}

/* ------------------------------------------------------------------ fields */

/* HField::calc_field, src/hField.cpp:93-157 */
void orc_field_h(void *h) {
  sim_t *s = (sim_t *)h;
  int nr = s->nr, nz = s->nz;
  double dr = s->dr, dz = s->dz, dt = s->dt;
  double *er = s->g[ORC_E_R], *ephi = s->g[ORC_E_PHI], *ez = s->g[ORC_E_Z];
  double *hr = s->g[ORC_H_R], *hphi = s->g[ORC_H_PHI], *hz = s->g[ORC_H_Z];
  double *hrh = s->g[ORC_H_R_HALF], *hphih = s->g[ORC_H_PHI_HALF], *hzh = s->g[ORC_H_Z_HALF];
  for (int k = 0; k < nz - 1; k++) {
    int i = nr - 1;
    double a = dt * (AT(ephi, i, k + 1) - AT(ephi, i, k)) / (dz * MAGN_CONST);
    AT(hrh, i, k) = AT(hr, i, k) + a / 2;
    AT(hr, i, k) = AT(hr, i, k) + a;
  }
#pragma omp parallel for
  for (int i = 0; i < nr - 1; i++)
    for (int k = 0; k < nz - 1; k++) {
      double a = dt * (AT(ephi, i, k + 1) - AT(ephi, i, k)) / (dz * MAGN_CONST);
      AT(hrh, i, k) = AT(hr, i, k) + a / 2;
      AT(hr, i, k) = AT(hr, i, k) + a;
      double b = dt * ((AT(ez, i + 1, k) - AT(ez, i, k)) / dr -
                       (AT(er, i, k + 1) - AT(er, i, k)) / dz) / MAGN_CONST;
      AT(hphih, i, k) = AT(hphi, i, k) + b / 2;
      AT(hphi, i, k) = AT(hphi, i, k) + b;
      double c = dt * ((AT(ephi, i + 1, k) + AT(ephi, i, k)) / (2.0 * dr * (i + 0.5)) +
                       (AT(ephi, i + 1, k) - AT(ephi, i, k)) / dr) / MAGN_CONST;
      AT(hzh, i, k) = AT(hz, i, k) - c / 2;
      AT(hz, i, k) = AT(hz, i, k) - c;
    }
}

/* EField::calc_field, src/eField.cpp:85-170 (epsilon == 1 everywhere,
   Geometry::set_epsilon src/geometry.cpp:33-39) */
void orc_field_e(void *h) {
  sim_t *s = (sim_t *)h;
  int nr = s->nr, nz = s->nz;
  double dr = s->dr, dz = s->dz, dt = s->dt;
  double *er = s->g[ORC_E_R], *ephi = s->g[ORC_E_PHI], *ez = s->g[ORC_E_Z];
  double *hr = s->g[ORC_H_R], *hphi = s->g[ORC_H_PHI], *hz = s->g[ORC_H_Z];
  double *jr = s->g[ORC_J_R], *jphi = s->g[ORC_J_PHI], *jz = s->g[ORC_J_Z];
  double *sig = s->g[ORC_SIGMA];
#define KOEF(i, k)                                              \
  double epsx2 = 2 * 1.0 * EPSILON0;                            \
  double sigma_t = AT(sig, i, k) * dt;                          \
  double koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);        \
  double koef_h = 2 * dt / (epsx2 + sigma_t);
  for (int k = 1; k < nz - 1; k++) {
    int i = 0;
    KOEF(i, k)
    AT(er, i, k) = AT(er, i, k) * koef_e -
                   (AT(jr, i, k) + (AT(hphi, i, k) - AT(hphi, i, k - 1)) / dz) * koef_h;
  }
  for (int k = 0; k < nz - 1; k++) {
    int i = 0;
    KOEF(i, k)
    AT(ez, i, k) = AT(ez, i, k) * koef_e - (AT(jz, i, k) - 4.0 / dr * AT(hphi, i, k)) * koef_h;
  }
#pragma omp parallel for
  for (int i = 1; i < nr - 1; i++)
    for (int k = 1; k < nz - 1; k++) {
      KOEF(i, k)
      AT(er, i, k) = AT(er, i, k) * koef_e -
                     (AT(jr, i, k) + (AT(hphi, i, k) - AT(hphi, i, k - 1)) / dz) * koef_h;
      AT(ephi, i, k) = AT(ephi, i, k) * koef_e -
                       (AT(jphi, i, k) - (AT(hr, i, k) - AT(hr, i, k - 1)) / dz +
                        (AT(hz, i, k) - AT(hz, i - 1, k)) / dr) * koef_h;
      AT(ez, i, k) = AT(ez, i, k) * koef_e -
                     (AT(jz, i, k) - (AT(hphi, i, k) - AT(hphi, i - 1, k)) / dr -
                      (AT(hphi, i, k) + AT(hphi, i - 1, k)) / (2.0 * dr * i)) * koef_h;
    }
  for (int i = 1; i < nr - 1; i++) {
    int k = 0;
    KOEF(i, k)
    AT(ez, i, k) = AT(ez, i, k) * koef_e -
                   (AT(jz, i, k) - (AT(hphi, i, k) - AT(hphi, i - 1, k)) / dr -
                    (AT(hphi, i, k) + AT(hphi, i - 1, k)) / (2.0 * dr * i)) * koef_h;
  }
#undef KOEF
}

/* -------------------------------------------------------------- gathering */

/* one staggered component: 4-node r-volume x z-linear weights.
   ishift/kshift = 1 when the component sits half a cell off the node in r/z.
   EField::get_field src/eField.cpp:204-316, HField::get_field src/hField.cpp:159-267 */
static double gather_one(const sim_t *s, const double *f, double radius, double longitude,
                         int rhalf, int zhalf) {
  double dr = s->dr, dz = s->dz;
  double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr;
  int i_r = rhalf ? cell_number(radius - 0.5 * dr, dr) : cell_number(radius, dr);
  int k_z = zhalf ? cell_number(longitude - 0.5 * dz, dz) : cell_number(longitude, dz);
  if (i_r < 0) i_r = 0;
  if (k_z < 0) k_z = 0;
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
  double acc = 0;
  acc = acc + AT(f, i_r, k_z) * PI * (dz1) * ((r2) * (r2) - (r1) * (r1)) / vol_1;
  acc = acc + AT(f, i_r + 1, k_z) * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / vol_2;
  acc = acc + AT(f, i_r, k_z + 1) * PI * (dz2) * ((r2) * (r2) - (r1) * (r1)) / vol_1;
  acc = acc + AT(f, i_r + 1, k_z + 1) * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / vol_2;
  return acc;
}

void orc_gather(void *h, double r, double z, double *e, double *b) {
  sim_t *s = (sim_t *)h;
  e[0] = gather_one(s, s->g[ORC_E_R], r, z, 1, 0);
  e[2] = gather_one(s, s->g[ORC_E_Z], r, z, 0, 1);
  e[1] = gather_one(s, s->g[ORC_E_PHI], r, z, 0, 0);
  b[2] = gather_one(s, s->g[ORC_H_Z_HALF], r, z, 1, 0);
  b[0] = gather_one(s, s->g[ORC_H_R_HALF], r, z, 0, 1);
  b[1] = gather_one(s, s->g[ORC_H_PHI_HALF], r, z, 1, 1);
}

/* ----------------------------------------------------------------- pushers */

/* tinyvec3d::tv_squared_sum / tv_dot, lib/tinyvec3d/tinyvec3d.cpp:55-62,121-124 */
static double dot3(const double *a, const double *b) {
  double res = 0;
  for (int i = 0; i < 3; i++) res += a[i] * b[i];
  return res;
}

/* lib::get_gamma, src/lib.cpp:45-70 */
static double get_gamma(double sq_velocity, int *err) {
  double beta = sq_velocity / LIGHT_SPEED_POW_2;
  if (beta > 1) {
    *err |= ORC_ERR_V_GE_C;
    return 1.0;
  }
  double gamma = 1 / sqrt(1.0 - beta);
  if (isinf(gamma)) return 1e100;
  return gamma;
}

/* lib::get_gamma_inv, src/lib.cpp:72-80 */
static double get_gamma_inv(double sq_velocity) {
  return pow(1.0 + sq_velocity / LIGHT_SPEED_POW_2, -0.5);
}

/* Particles::boris_pusher_single, src/particles.cpp:1025-1150.
   rel = 1: relativistic form (PUSHER_BORIS_RELATIVISTIC, which is also what
   the default adaptive build computes at -O2); rel = 0: PUSHER_BORIS_CLASSIC. */
static void boris(double q, double m, double dt, double *e, double *b, double *v, int rel,
                  int *err) {
  double const1 = q * dt / (2 * m);
  double velocity[3], vtmp[3];
  for (int i = 0; i < 3; i++) e[i] *= const1;
  for (int i = 0; i < 3; i++) b[i] *= MAGN_CONST * const1;
  for (int i = 0; i < 3; i++) velocity[i] = (fabs(v[i]) < MNZL) ? 0 : v[i];
  if (rel) {
    double g = get_gamma(dot3(velocity, velocity), err);
    for (int i = 0; i < 3; i++) velocity[i] *= g;
  }
  for (int i = 0; i < 3; i++) velocity[i] += e[i];
  if (rel) {
    double g = get_gamma_inv(dot3(velocity, velocity));
    for (int i = 0; i < 3; i++) b[i] *= g;
  }
  double const2 = 2. / (1. + dot3(b, b));
  for (int i = 0; i < 3; i++) vtmp[i] = velocity[i];
  velocity[0] = vtmp[0] + const2 * ((vtmp[1] - vtmp[0] * b[2] + vtmp[2] * b[0]) * b[2] -
                                    (vtmp[2] + vtmp[0] * b[1] - vtmp[1] * b[0]) * b[1]);
  velocity[1] = vtmp[1] + const2 * (-(vtmp[0] + vtmp[1] * b[2] - vtmp[2] * b[1]) * b[2] +
                                    (vtmp[2] + vtmp[0] * b[1] - vtmp[1] * b[0]) * b[0]);
  velocity[2] = vtmp[2] + const2 * ((vtmp[0] + vtmp[1] * b[2] - vtmp[2] * b[1]) * b[1] -
                                    (vtmp[1] - vtmp[0] * b[2] + vtmp[2] * b[0]) * b[0]);
  for (int i = 0; i < 3; i++) velocity[i] += e[i];
  if (rel) {
    double g = get_gamma_inv(dot3(velocity, velocity));
    for (int i = 0; i < 3; i++) velocity[i] *= g;
  }
  for (int i = 0; i < 3; i++) v[i] = velocity[i];
}

/* Particles::vay_pusher_single, src/particles.cpp:1152-1254, as written
   (the magnetic factor is multiplied by MAGN_CONST*const1, 2*const1 and
   const1 in turn). */
static void vay(double q, double m, double dt, double *e, double *b, double *v, int *err) {
  double const1 = q * dt / (2 * m);
  double velocity[3], vtmp[3];
  for (int i = 0; i < 3; i++) e[i] *= 2 * const1;
  for (int i = 0; i < 3; i++) b[i] *= MAGN_CONST * const1;
  for (int i = 0; i < 3; i++) velocity[i] = (fabs(v[i]) < MNZL) ? 0 : v[i];
  double gamma = get_gamma(dot3(velocity, velocity), err);
  for (int i = 0; i < 3; i++) velocity[i] *= gamma;
  for (int i = 0; i < 3; i++) vtmp[i] = velocity[i];
  for (int i = 0; i < 3; i++) b[i] *= 2 * const1;
  for (int i = 0; i < 3; i++) velocity[i] += e[i];
  for (int i = 0; i < 3; i++) b[i] *= const1;
  gamma = get_gamma_inv(dot3(vtmp, vtmp));
  velocity[0] += gamma * (vtmp[1] * b[2] - vtmp[2] * b[1]);
  velocity[1] += gamma * (vtmp[2] * b[0] - vtmp[0] * b[2]);
  velocity[2] += gamma * (vtmp[0] * b[1] - vtmp[1] * b[0]);
  gamma = get_gamma_inv(dot3(velocity, velocity));
  double alpha = 1. / gamma / gamma;
  double B2 = dot3(b, b);
  double sg = alpha - B2;
  double us2 = pow(dot3(velocity, b), 2);
  alpha = 1. / sqrt(0.5 * (sg + sqrt(sg * sg + 4. * (B2 + us2))));
  for (int i = 0; i < 3; i++) b[i] *= alpha;
  sg = 1. / (1. + dot3(b, b));
  alpha = dot3(velocity, b);
  vtmp[0] = sg * (velocity[0] + alpha * b[0] + b[2] * velocity[1] - b[1] * velocity[2]);
  vtmp[1] = sg * (velocity[1] + alpha * b[1] + b[0] * velocity[2] - b[2] * velocity[0]);
  vtmp[2] = sg * (velocity[2] + alpha * b[2] + b[1] * velocity[0] - b[0] * velocity[1]);
  gamma = get_gamma_inv(dot3(vtmp, vtmp));
  for (int i = 0; i < 3; i++) v[i] = vtmp[i] * gamma;
}

/* ------------------------------------------------------------- deposition */

static inline void inc(sim_t *s, int comp, int i, int k, double v) {
  AT(s->g[comp], i, k) += v;
}

/* Particles::azimuthal_current_distribution, src/particles.cpp:688-784 */
static void deposit_jphi(sim_t *s, double q, double r, double z, double vphi) {
  double dr = s->dr, dz = s->dz;
  int r_i = cell_number(r, dr), z_k = cell_number(z, dz);
  if (r_i < 0) r_i = 0;
  if (z_k < 0) z_k = 0;
  double r1 = r - 0.5 * dr, r2 = (r_i + 0.5) * dr, r3 = r + 0.5 * dr;
  double ro_v = q / (2. * PI * dz * dr * r);
  double v_1, v_2;
  if (r > dr)
    v_1 = PI * dz * dr * dr * 2.0 * (r_i);
  else
    v_1 = PI * (dz) * (dr) * (dr) / 4.;
  v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
  double dz1 = (z_k + 0.5) * dz - (z - 0.5 * dz);
  double dz2 = (z + 0.5 * dz) - (z_k + 0.5) * dz;
  double rho;
  rho = ro_v * PI * (dz1) * ((r2) * (r2) - (r1) * (r1)) / v_1;
  inc(s, ORC_J_PHI, r_i, z_k, rho * vphi);
  rho = ro_v * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / v_2;
  inc(s, ORC_J_PHI, r_i + 1, z_k, rho * vphi);
  rho = ro_v * PI * (dz2) * ((r2) * (r2) - (r1) * (r1)) / v_1;
  inc(s, ORC_J_PHI, r_i, z_k + 1, rho * vphi);
  rho = ro_v * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / v_2;
  inc(s, ORC_J_PHI, r_i + 1, z_k + 1, rho * vphi);
}

/* SOME_SHIT_DENSITY_R/Z/STRICT, include/particles.h:169-178 */
#define DENS_R(q, r, dr, dz, dt) ((q) / (2 * PI * (r) * (dr) * (dz) * (dt) * 2 * (dr)))
#define DENS_Z(q, r, dr, dz, dt) ((q) / (2 * PI * (r) * (dr) * (dz) * (dt) * (dz)))
#define DENS_STRICT(q, r, dr, dz, dt) ((q) / (PI * 4. * (r) * (dz) * (dz) * (dr) * (dt)))

/* Particles::simple_current_distribution, src/particles.cpp:333-474 */
static void simple_current(sim_t *s, double q, double radius_new, double longitude_new,
                           double radius_old, double longitude_old, int i_n, int k_n) {
  double dr = s->dr, dz = s->dz, delta_t = s->dt, wj, dens;
  double delta_r = radius_new - radius_old;
  double delta_z = longitude_new - longitude_old;
  if ((fabs(delta_r) < MNZL) || (fabs(delta_z) < MNZL)) return;
  double k = delta_r / delta_z;
  double b = radius_old;
  if (i_n >= 1) {
    dens = DENS_R(q, i_n * dr, dr, dz, delta_t);
    wj = dens * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b +
                 dr * dr / k * ((i_n + 0.5) * (i_n + 0.5) - 0.25) * log((k * delta_z + b) / b));
    inc(s, ORC_J_Z, i_n, k_n, wj);
    dens = DENS_R(q, (i_n + 1) * dr, dr, dz, delta_t);
    wj = dens * (k * delta_z * delta_z / 2. + delta_z * b + delta_z * dr +
                 dr * dr / k * (0.25 - (i_n + 0.5) * (i_n + 0.5)) * log((k * delta_z + b) / b));
    inc(s, ORC_J_Z, i_n + 1, k_n, wj);
  } else {
    dens = q / (2. * PI * dr / 4. * dr * dz * delta_t * dr);
    wj = dens * (dr * delta_z - k * delta_z * delta_z / 2. - delta_z * b);
    inc(s, ORC_J_Z, i_n, k_n, wj);
    dens = DENS_R(q, dr, dr, dz, delta_t);
    wj = dens * (k * delta_z * delta_z / 2. + delta_z * dr + delta_z * b);
    inc(s, ORC_J_Z, i_n + 1, k_n, wj);
  }
  /* j_r part: the same expressions in both upstream branches
     (src/particles.cpp:386-412 and :444-472) */
  k = -delta_z / delta_r;
  double r0 = (i_n + 0.5) * dr;
  double r1 = radius_old;
  b = (k_n + 1.) * dz - longitude_old;
  dens = DENS_Z(q, r0, dr, dz, delta_t);
  wj = dens * (r0 * k * delta_r + k / 2. * delta_r * (radius_old + delta_r / 2.) +
               0.5 * delta_r * (b - k * (2 * r0 + r1)) +
               delta_r * (b - k * r1) * (4 * r0 * r0 - dr * dr) /
                   (8 * radius_old * (radius_old + delta_r)) +
               (k * (r0 * r0 / 2. - dr * dr / 8.)) * log((radius_old + delta_r) / radius_old));
  inc(s, ORC_J_R, i_n, k_n, wj);
  b = longitude_old - k_n * dz;
  wj = dens * (-r0 * k * delta_r - k / 2. * delta_r * (radius_old + delta_r / 2.) +
               0.5 * delta_r * (b + k * (2 * r0 + r1)) +
               delta_r * (b + k * r1) * (4 * r0 * r0 - dr * dr) /
                   (8 * radius_old * (radius_old + delta_r)) -
               (k * (r0 * r0 / 2. - dr * dr / 8.)) * log((radius_old + delta_r) / radius_old));
  inc(s, ORC_J_R, i_n, k_n + 1, wj);
}

/* Particles::strict_motion_weighting, src/particles.cpp:786-988 */
static void strict_motion(sim_t *s, double q, double radius_new, double longitude_new,
                          double radius_old, double longitude_old) {
  double dr = s->dr, dz = s->dz, delta_t = s->dt;
  int i_n = cell_number(radius_new, dr), k_n = cell_number(longitude_new, dz);
  int i_o = cell_number(radius_old, dr), k_o = cell_number(longitude_old, dz);
  if (i_n < 0) i_n = 0;
  if (k_n < 0) k_n = 0;
  if (i_o < 0) i_o = 0;
  if (k_o < 0) k_o = 0;
  if ((fabs(radius_new - radius_old) < MNZL) && (fabs(longitude_new - longitude_old) < MNZL))
    return;
  if (fabs(radius_new - radius_old) < MNZL) {
    /* motion along z only */
    double delta_z, wj, wj_lower, wj_upper;
    double value_part = 2. * PI * radius_new * dr * dz;
    double r1 = radius_new - 0.5 * dr, r2 = (i_n + 0.5) * dr, r3 = radius_new + 0.5 * dr;
    if (i_n == 0)
      wj_lower = q / (delta_t * PI * dr * dr / 4.) * PI * (r2 * r2 - r1 * r1) / value_part;
    else
      wj_lower = q / (delta_t * 2. * PI * i_n * dr * dr) * PI * (r2 * r2 - r1 * r1) / value_part;
    wj_upper = q / (delta_t * 2 * PI * (i_n + 1) * dr * dr) * PI * (r3 * r3 - r2 * r2) / value_part;
    inc(s, ORC_J_R, i_n, k_n, 0.);
    inc(s, ORC_J_R, i_n, k_n + 1, 0.);
    switch (k_n - k_o) {
      case 0:
        delta_z = longitude_new - longitude_old;
        inc(s, ORC_J_Z, i_n, k_n, wj_lower * delta_z);
        inc(s, ORC_J_Z, i_n + 1, k_n, wj_upper * delta_z);
        break;
      case 1:
        delta_z = k_n * dz - longitude_old;
        inc(s, ORC_J_Z, i_n, k_n - 1, wj_lower * delta_z);
        inc(s, ORC_J_Z, i_n + 1, k_n - 1, wj_upper * delta_z);
        delta_z = longitude_new - k_n * dz;
        inc(s, ORC_J_Z, i_n, k_n, wj_lower * delta_z);
        inc(s, ORC_J_Z, i_n + 1, k_n, wj_upper * delta_z);
        break;
      case -1:
        delta_z = (k_n + 1) * dz - longitude_old;
        inc(s, ORC_J_Z, i_n, k_n + 1, wj_lower * delta_z);
        inc(s, ORC_J_Z, i_n + 1, k_n + 1, wj_upper * delta_z);
        delta_z = longitude_new - (k_n + 1) * dz;
        inc(s, ORC_J_Z, i_n, k_n, wj_lower * delta_z);
        inc(s, ORC_J_Z, i_n + 1, k_n, wj_upper * delta_z);
        break;
    }
    (void)wj;
  } else if (fabs(longitude_new - longitude_old) < MNZL) {
    /* motion along r only */
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
        inc(s, ORC_J_R, i_n, k_n, wj * left_delta_z);
        inc(s, ORC_J_R, i_n, k_n + 1, wj * right_delta_z);
        break;
      case 1:
        delta_r = (i_n)*dr - radius_old;
        left_delta_z = (k_n + 1) * dz - longitude_new;
        right_delta_z = longitude_new - k_n * dz;
        r0 = (i_n - 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / (radius_old + delta_r) + r0 * r0 / radius_old +
                     dr * dr / (4. * (radius_old + delta_r)) - dr * dr / (4. * radius_old));
        inc(s, ORC_J_R, i_n - 1, k_n, wj * left_delta_z);
        inc(s, ORC_J_R, i_n - 1, k_n + 1, wj * right_delta_z);
        delta_r = radius_new - i_n * dr;
        r0 = (i_n + 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        /* "r0 * r0 / i_n * dr" is (r0*r0/i_n)*dr upstream (src/particles.cpp:941) */
        wj = dens * (delta_r - r0 * r0 / (i_n * dr + delta_r) + r0 * r0 / i_n * dr +
                     dr * dr / (4. * (i_n * dr + delta_r)) - dr * dr / (4. * i_n * dr));
        inc(s, ORC_J_R, i_n, k_n, wj * left_delta_z);
        inc(s, ORC_J_R, i_n, k_n + 1, wj * right_delta_z);
        break;
      case -1:
        delta_r = (i_n + 1) * dr - radius_old;
        left_delta_z = (k_n + 1) * dz - longitude_new;
        right_delta_z = longitude_new - k_n * dz;
        r0 = (i_n + 1.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / (radius_old + delta_r) + r0 * r0 / radius_old +
                     dr * dr / (4. * (radius_old + delta_r)) - dr * dr / (4. * radius_old));
        inc(s, ORC_J_R, i_n + 1, k_n, wj * left_delta_z);
        inc(s, ORC_J_R, i_n + 1, k_n + 1, wj * right_delta_z);
        delta_r = radius_new - (i_n + 1) * dr;
        r0 = (i_n + 0.5) * dr;
        dens = DENS_STRICT(q, r0, dr, dz, delta_t);
        wj = dens * (delta_r - r0 * r0 / ((i_n + 1) * dr + delta_r) + r0 * r0 / (i_n + 1) * dr +
                     dr * dr / (4. * ((i_n + 1) * dr + delta_r)) - dr * dr / (4. * (i_n + 1) * dr));
        inc(s, ORC_J_R, i_n, k_n, wj * left_delta_z);
        inc(s, ORC_J_R, i_n, k_n + 1, wj * right_delta_z);
        break;
    }
  }
}

/* Particles::current_distribution, src/particles.cpp:476-686: the move
   (r_o, z_o) -> (r_n, z_n) is split at cell faces into 1-3 straight segments. */
static void deposit_rz(sim_t *s, double q, double r_n, double z_n, double r_o, double z_o) {
  double dr = s->dr, dz = s->dz;
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
  int res_cell = abs(i_n - i_o) + abs(k_n - k_o);
  if ((fabs(r_n - r_o) < MNZL) || (fabs(z_n - z_o) < MNZL)) {
    strict_motion(s, q, r_n, z_n, r_o, z_o);
    return;
  }
  if (res_cell == 0) {
    simple_current(s, q, r_n, z_n, r_o, z_o, i_n, k_n);
  } else if (res_cell == 1) {
    if ((i_n != i_o) && (k_n == k_o)) {
      if (r_o > (i_n + 1) * dr) {
        double a = (r_o - r_n) / (z_o - z_n);
        double r_b = (i_n + 1) * dr;
        double d_r = r_b - r_n;
        double z_b = z_n + d_r / a;
        simple_current(s, q, r_b, z_b, r_o, z_o, i_n + 1, k_n);
        simple_current(s, q, r_n, z_n, r_b, z_b, i_n, k_n);
      } else {
        double a = (r_n - r_o) / (z_n - z_o);
        double r_b = (i_n)*dr;
        double d_r = r_b - r_o;
        double z_b = z_o + d_r / a;
        simple_current(s, q, r_b, z_b, r_o, z_o, i_n - 1, k_n);
        simple_current(s, q, r_n, z_n, r_b, z_b, i_n, k_n);
      }
    } else if ((i_n == i_o) && (k_n != k_o)) {
      if (z_o < k_n * dz) {
        double z_b = k_n * dz;
        double d_z = z_b - z_o;
        double a = (r_n - r_o) / (z_n - z_o);
        double r_b = r_o + a * d_z;
        simple_current(s, q, r_b, z_b, r_o, z_o, i_n, k_n - 1);
        simple_current(s, q, r_n, z_n, r_b, z_b, i_n, k_n);
      } else {
        double z_b = (k_n + 1) * dz;
        double d_z = z_b - z_n;
        double a = (r_o - r_n) / (z_o - z_n);
        double r_b = r_n + a * d_z;
        simple_current(s, q, r_b, z_b, r_o, z_o, i_n, k_n + 1);
        simple_current(s, q, r_n, z_n, r_b, z_b, i_n, k_n);
      }
    }
  } else if (res_cell == 2) {
    if (i_o < i_n) {
      if (k_o < k_n) {
        double a = (r_n - r_o) / (z_n - z_o);
        double r1 = i_n * dr;
        double dz1 = (r1 - r_o) / a;
        double z1 = z_o + dz1;
        double z2 = k_n * dz;
        double dr2 = (z2 - z_o) * a;
        double r2 = r_o + dr2;
        if (z1 < k_n * dz) {
          simple_current(s, q, r1, z1, r_o, z_o, i_n - 1, k_n - 1);
          simple_current(s, q, r2, z2, r1, z1, i_n, k_n - 1);
          simple_current(s, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 > k_n * dz) {
          simple_current(s, q, r2, z2, r_o, z_o, i_n - 1, k_n - 1);
          simple_current(s, q, r1, z1, r2, z2, i_n - 1, k_n);
          simple_current(s, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      } else {
        double a = (r_n - r_o) / (z_n - z_o);
        double r1 = i_n * dr;
        double dz1 = (r1 - r_o) / a;
        double z1 = z_o + dz1;
        double z2 = (k_n + 1) * dz;
        double dr2 = -(z_o - z2) * a;
        double r2 = r_o + dr2;
        if (z1 > (k_n + 1) * dz) {
          simple_current(s, q, r1, z1, r_o, z_o, i_n - 1, k_n + 1);
          simple_current(s, q, r2, z2, r1, z1, i_n, k_n + 1);
          simple_current(s, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 < (k_n + 1) * dz) {
          simple_current(s, q, r2, z2, r_o, z_o, i_n - 1, k_n + 1);
          simple_current(s, q, r1, z1, r2, z2, i_n - 1, k_n);
          simple_current(s, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      }
    } else if (i_o > i_n) {
      if (k_o < k_n) {
        double a = (r_n - r_o) / (z_n - z_o);
        double r1 = (i_n + 1) * dr;
        double dz1 = -(r_o - r1) / a;
        double z1 = z_o + dz1;
        double z2 = k_n * dz;
        double dr2 = -(z2 - z_o) * a;
        double r2 = r_o - dr2;
        if (z1 < (k_n)*dz) {
          simple_current(s, q, r1, z1, r_o, z_o, i_n + 1, k_n - 1);
          simple_current(s, q, r2, z2, r1, z1, i_n, k_n - 1);
          simple_current(s, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 > (k_n)*dz) {
          simple_current(s, q, r2, z2, r_o, z_o, i_n + 1, k_n - 1);
          simple_current(s, q, r1, z1, r2, z2, i_n + 1, k_n);
          simple_current(s, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      } else if (k_o > k_n) {
        double a = (r_o - r_n) / (z_o - z_n);
        double r1 = (i_n + 1) * dr;
        double dz1 = (r1 - r_n) / a;
        double z1 = z_n + dz1;
        double z2 = (k_n + 1) * dz;
        double dr2 = (z2 - z_n) * a;
        double r2 = r_n + dr2;
        if (z1 > (k_n + 1) * dz) {
          simple_current(s, q, r1, z1, r_o, z_o, i_n + 1, k_n + 1);
          simple_current(s, q, r2, z2, r1, z1, i_n, k_n + 1);
          simple_current(s, q, r_n, z_n, r2, z2, i_n, k_n);
        } else if (z1 < (k_n + 1) * dz) {
          simple_current(s, q, r2, z2, r_o, z_o, i_n + 1, k_n + 1);
          simple_current(s, q, r1, z1, r2, z2, i_n + 1, k_n);
          simple_current(s, q, r_n, z_n, r1, z1, i_n, k_n);
        }
      }
    }
  }
}

/* ------------------------------------------------------------------- step */

static int bad_number(double x) { return isnan(x) || isinf(x); }

/* Particles::step_v, src/particles.cpp:1296-1316, with
   dump_position_to_old_single :1256-1260, half_step_pos_single :1270-1284,
   back_position_to_rz_single :1286-1294 */
static void species_push(sim_t *s, species_t *p) {
  double half_dt = s->dt / 2.;
  int err = 0;
#pragma omp parallel for reduction(| : err)
  for (int i = 0; i < p->n; i++) {
    if (!p->alive[i]) continue;
    if (bad_number(p->r[i]) || bad_number(p->z[i])) {
      err |= ORC_ERR_NAN;
      continue;
    }
    double e[3], b[3], v[3] = {p->vr[i], p->vphi[i], p->vz[i]};
    orc_gather(s, p->r[i], p->z[i], e, b);
    double q = p->charge * p->w[i], m = p->mass * p->w[i];
    if (s->pusher == ORC_VAY)
      vay(q, m, s->dt, e, b, v, &err);
    else
      boris(q, m, s->dt, e, b, v, s->pusher == ORC_BORIS_REL, &err);
    p->vr[i] = v[0]; p->vphi[i] = v[1]; p->vz[i] = v[2];
    p->r_old[i] = p->r[i];
    p->z_old[i] = p->z[i];
    p->r[i] = p->r[i] + p->vr[i] * half_dt;
    p->y[i] = p->y[i] + p->vphi[i] * half_dt;
    p->z[i] = p->z[i] + p->vz[i] * half_dt;
    double r = sqrt(p->r[i] * p->r[i] + p->y[i] * p->y[i]);
    p->sin_t[i] = p->y[i] / r;
    p->r[i] = r;
    p->y[i] = 0;
  }
  s->errors |= err;
}

/* Particles::reflection_single src/particles.cpp:1318-1353 (plasma: mirror)
   and Bunch::reflection_single src/bunch.cpp:126-153 (bunch: outer walls kill) */
static void reflect(const sim_t *s, species_t *p, int i) {
  double dr = s->dr, dz = s->dz;
  double radius_wall = s->r_size - dr / 2.;
  double longitude_wall = s->z_size - dz / 2.;
  double half_dr = dr / 2., half_dz = dz / 2.;
  if (p->kind == ORC_PLASMA) {
    double radius_wallX2 = radius_wall * 2., longitude_wallX2 = longitude_wall * 2.;
    if (p->r[i] > radius_wall) { p->r[i] = radius_wallX2 - p->r[i]; p->vr[i] = -p->vr[i]; }
    if (p->z[i] > longitude_wall) { p->z[i] = longitude_wallX2 - p->z[i]; p->vz[i] = -p->vz[i]; }
  } else {
    if (p->r[i] > radius_wall) p->alive[i] = 0;
    if (p->z[i] > longitude_wall) p->alive[i] = 0;
  }
  if (p->r[i] < half_dr) { p->r[i] = dr - p->r[i]; p->vr[i] = -p->vr[i]; }
  if (p->z[i] < half_dz) { p->z[i] = dz - p->z[i]; p->vz[i] = -p->vz[i]; }
}

/* Particles::full_current_distribution, src/particles.cpp:1367-1373 */
static void species_current(sim_t *s, species_t *p) {
  double half_dt = s->dt / 2.;
  for (int i = 0; i < p->n; i++)
    if (p->alive[i]) deposit_jphi(s, p->charge * p->w[i], p->r[i], p->z[i], p->vphi[i]);
  /* move_half_reflect, src/particles.cpp:1355-1365 */
#pragma omp parallel for
  for (int i = 0; i < p->n; i++) {
    if (!p->alive[i]) continue;
    p->r[i] = p->r[i] + p->vr[i] * half_dt;
    p->y[i] = p->y[i] + p->vphi[i] * half_dt;
    p->z[i] = p->z[i] + p->vz[i] * half_dt;
    reflect(s, p, i);
    double r = sqrt(p->r[i] * p->r[i] + p->y[i] * p->y[i]);
    p->sin_t[i] = p->y[i] / r;
    p->r[i] = r;
    p->y[i] = 0;
  }
  for (int i = 0; i < p->n; i++)
    if (p->alive[i]) deposit_rz(s, p->charge * p->w[i], p->r[i], p->z[i], p->r_old[i], p->z_old[i]);
  /* back_velocity_to_rz, src/particles.cpp:1005-1023 */
#pragma omp parallel for
  for (int i = 0; i < p->n; i++) {
    if (!p->alive[i]) continue;
    double st = p->sin_t[i];
    double ct = sqrt(1 - st * st);
    double u2 = ct * p->vr[i] - st * p->vphi[i];
    double v2 = st * p->vr[i] + ct * p->vphi[i];
    p->vr[i] = u2;
    p->vphi[i] = v2;
  }
}

/* LoadInitParam::run loop body, src/loadInitParam.cpp:471-587 (probes off) */
int orc_step(void *h) {
  sim_t *s = (sim_t *)h;
  for (int i = 0; i < s->nsp; i++)
    if (s->sp[i].kind == ORC_BUNCH) bunch_inject(s, &s->sp[i]);
  orc_field_h(s);
  size_t ng = (size_t)s->nr * s->nz;
  memset(s->g[ORC_J_R], 0, ng * sizeof(double));
  memset(s->g[ORC_J_PHI], 0, ng * sizeof(double));
  memset(s->g[ORC_J_Z], 0, ng * sizeof(double));
  for (int i = 0; i < s->nsp; i++) species_push(s, &s->sp[i]);
  for (int i = 0; i < s->nsp; i++) species_current(s, &s->sp[i]);
  orc_field_e(s);
  int sched = (int)(s->t / s->dt);
  s->t = s->t + s->dt;
  return sched;
}

int orc_errors(void *h) { return ((sim_t *)h)->errors; }
double orc_time(void *h) { return ((sim_t *)h)->t; }
int orc_species_n(void *h, int idx) { return ((sim_t *)h)->sp[idx].n; }

int orc_get_grid(void *h, int comp, double *out) {
  sim_t *s = (sim_t *)h;
  if (comp < 0 || comp >= ORC_NCOMP) return -1;
  memcpy(out, s->g[comp], sizeof(double) * (size_t)s->nr * s->nz);
  return 0;
}

int orc_set_grid(void *h, int comp, const double *in) {
  sim_t *s = (sim_t *)h;
  if (comp < 0 || comp >= ORC_NCOMP) return -1;
  memcpy(s->g[comp], in, sizeof(double) * (size_t)s->nr * s->nz);
  return 0;
}

int orc_get_species(void *h, int idx, double *r, double *z, double *vr, double *vphi,
                    double *vz, double *w, uint8_t *alive) {
  sim_t *s = (sim_t *)h;
  if (idx < 0 || idx >= s->nsp) return -1;
  species_t *p = &s->sp[idx];
  size_t b = sizeof(double) * (size_t)p->n;
  if (r) memcpy(r, p->r, b);
  if (z) memcpy(z, p->z, b);
  if (vr) memcpy(vr, p->vr, b);
  if (vphi) memcpy(vphi, p->vphi, b);
  if (vz) memcpy(vz, p->vz, b);
  if (w) memcpy(w, p->w, b);
  if (alive) memcpy(alive, p->alive, (size_t)p->n);
  return 0;
}

int orc_set_species(void *h, int idx, const double *r, const double *z, const double *vr,
                    const double *vphi, const double *vz, const uint8_t *alive) {
  sim_t *s = (sim_t *)h;
  if (idx < 0 || idx >= s->nsp) return -1;
  species_t *p = &s->sp[idx];
  size_t b = sizeof(double) * (size_t)p->n;
  if (r) memcpy(p->r, r, b);
  if (z) memcpy(p->z, z, b);
  if (vr) memcpy(p->vr, vr, b);
  if (vphi) memcpy(p->vphi, vphi, b);
  if (vz) memcpy(p->vz, vz, b);
  if (alive) memcpy(p->alive, alive, (size_t)p->n);
  return 0;
}

/* Particles::charge_weighting, src/particles.cpp:101-226 */
void orc_charge_density(void *h, uint32_t mask, double *out) {
  sim_t *s = (sim_t *)h;
  double dr = s->dr, dz = s->dz;
  memset(out, 0, sizeof(double) * (size_t)s->nr * s->nz);
  for (int sp = 0; sp < s->nsp; sp++) {
    if (!(mask & (1u << sp))) continue;
    species_t *p = &s->sp[sp];
    for (int i = 0; i < p->n; i++) {
      if (!p->alive[i]) continue;
      double r = p->r[i], z = p->z[i], q = p->charge * p->w[i];
      int r_i = cell_number(r, dr), z_k = cell_number(z, dz);
      if (r_i < 0) r_i = 0;
      if (z_k < 0) z_k = 0;
      double r1, r2, r3, ro_v, v_1, v_2, dz1, dz2;
      if (r > dr) {
        r1 = r - 0.5 * dr; r2 = (r_i + 0.5) * dr; r3 = r + 0.5 * dr;
        ro_v = q / (2. * PI * dz * dr * r);
        v_1 = PI * dz * dr * dr * 2.0 * (r_i);
        v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
        dz1 = (z_k + 0.5) * dz - (z - 0.5 * dz);
        dz2 = (z + 0.5 * dz) - (z_k + 0.5) * dz;
        AT(out, r_i, z_k) += ro_v * PI * (dz1) * ((r2) * (r2) - (r1) * (r1)) / v_1;
        AT(out, r_i + 1, z_k) += ro_v * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / v_2;
        AT(out, r_i, z_k + 1) += ro_v * PI * (dz2) * ((r2) * (r2) - (r1) * (r1)) / v_1;
        AT(out, r_i + 1, z_k + 1) += ro_v * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / v_2;
      } else if (r <= dr / 2.) {
        r_i = 0;
        r1 = 0.; r2 = (r_i + 0.5) * dr; r3 = r + 0.5 * dr;
        dz1 = (z_k + 0.5) * dz - (z - 0.5 * dz);
        dz2 = (z + 0.5 * dz) - (z_k + 0.5) * dz;
        ro_v = q / (PI * dz * (2. * r * r + dr * dr / 2.));
        v_1 = PI * (dz) * (dr) * (dr) / 4.;
        v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
        AT(out, r_i, z_k) += ro_v * PI * dz1 * (dr * dr / 2. - r * dr + r * r) / v_1;
        AT(out, r_i + 1, z_k) += ro_v * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / v_2;
        AT(out, r_i, z_k + 1) += ro_v * PI * dz2 * (dr * dr / 2. - r * dr + r * r) / v_1;
        AT(out, r_i + 1, z_k + 1) += ro_v * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / v_2;
      } else {
        r1 = r - 0.5 * dr; r2 = (r_i + 0.5) * dr; r3 = r + 0.5 * dr;
        dz1 = (z_k + 0.5) * dz - (z - 0.5 * dz);
        dz2 = (z + 0.5 * dz) - (z_k + 0.5) * dz;
        ro_v = q / (2. * PI * dz * dr * r);
        v_1 = PI * (dz) * (dr) * (dr) / 4.;
        v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
        AT(out, r_i, z_k) += ro_v * PI * (dz1) * ((r2) * (r2) - (r1) * (r1)) / v_1;
        AT(out, r_i + 1, z_k) += ro_v * PI * (dz1) * ((r3) * (r3) - (r2) * (r2)) / v_2;
        AT(out, r_i, z_k + 1) += ro_v * PI * (dz2) * ((r2) * (r2) - (r1) * (r1)) / v_1;
        AT(out, r_i + 1, z_k + 1) += ro_v * PI * (dz2) * ((r3) * (r3) - (r2) * (r2)) / v_2;
      }
    }
  }
}
