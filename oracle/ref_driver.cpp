// Test-infrastructure driver for the upstream PDP3 hot-path classes.
//
// ORACLE ONLY: this file is compiled together with the unmodified upstream
// sources (oracle/Makefile) into oracle/_ref/libpdp3ref_*.so.  Only tests/,
// the smoke check and bench.py's CPU-baseline leg load it, as a checker and
// as the timed CPU reference.  The GPU product never links it.
//
// The upstream main loop lives in LoadInitParam (src/loadInitParam.cpp),
// which cannot be linked here because its Parameters dependency needs the
// un-vendored tinyxml2.  This driver therefore re-creates the sequence that
// LoadInitParam::LoadInitParam / init_fields / init_particles / init_beam /
// run perform, calling the upstream classes directly:
//   ctor:          src/loadInitParam.cpp:10-128 (fields, particles, no probes)
//   init_fields:   src/loadInitParam.cpp:250-260
//   init_particles src/loadInitParam.cpp:134-166
//   init_beam:     src/loadInitParam.cpp:168-248 (bunch erasure not needed:
//                  dead bunches carry no alive particle and change nothing)
//   run() body:    src/loadInitParam.cpp:471-587
// and exposes it through a plain C ABI for ctypes.

#include <chrono>
#include <cstring>
#include <cstdlib>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "geometry.h"
#include "pdp3Time.h"
#include "eField.h"
#include "hField.h"
#include "current.h"
#include "chargeDensity.h"
#include "particles.h"
#include "particlesList.h"
#include "bunch.h"
#include "particlesDensity.h"
#include "poissonDirichlet.h"
#include "temperatureClassic.h"

namespace {

struct BeamParams {
  bool enabled = false;
  double charge_e = -1, mass_me = 1;
  int number_macro = 0;
  double bunch_length = 0, radius = 0, density = 0, velocity = 0;
  int number_bunches = 0;
  double bunches_distance = 0;
};

struct RefSim {
  Geometry *geom = nullptr;
  Time *time = nullptr;
  EField *efield = nullptr;
  HField *hfield = nullptr;
  Current *current = nullptr;
  ChargeDensity *rho_new = nullptr, *rho_old = nullptr, *rho_bunch = nullptr;
  ParticlesList *plist = nullptr;
  std::vector<Bunch *> bunches;
  BeamParams beam;
  int current_bunch_number = 0;
  std::vector<char *> names;
  TemperatureClassic *temperature = nullptr;  // LoadInitParam's diagnostics
  ParticlesDensity *density = nullptr;
};

// The upstream diagnostics index CELL_NUMBER(r), CELL_NUMBER(z) (and +1)
// unchecked: a particle at r <= 0 or z <= 0, or beyond the grid, would write
// outside their arrays.  The driver refuses such species instead.
bool cells_inside(RefSim *s, Particles *p) {
  const double dr = s->geom->dr, dz = s->geom->dz;
  for (unsigned int i = 0; i < p->number; i++) {
    const int ri = CELL_NUMBER(p->pos[i][0], dr), zk = CELL_NUMBER(p->pos[i][2], dz);
    if (ri < 0 || zk < 0 || ri + 1 >= (int)s->geom->n_grid_r || zk + 1 >= (int)s->geom->n_grid_z)
      return false;
  }
  return true;
}

char *keep_name(RefSim *s, const char *name) {
  char *c = strdup(name ? name : "species");
  s->names.push_back(c);
  return c;
}

void init_beam(RefSim *s) {
  // src/loadInitParam.cpp:168-248
  const BeamParams &b = s->beam;
  if (!b.enabled) return;
  double duration = b.bunch_length / b.velocity;
  double hole_duration = b.bunches_distance / b.velocity;
  double bunch_inject_time = s->current_bunch_number * (duration + hole_duration);
  if (s->time->current_time >= bunch_inject_time &&
      s->current_bunch_number < b.number_bunches) {
    char buf[64];
    snprintf(buf, sizeof(buf), "Beam#%d", s->current_bunch_number);
    Bunch *prtls = new Bunch(keep_name(s, buf), b.charge_e, b.mass_me, b.number_macro,
                             s->geom, duration, b.radius, b.density, b.velocity,
                             s->current_bunch_number, hole_duration);
    s->plist->part_list.push_back(prtls);
    s->bunches.push_back(prtls);
    ++s->current_bunch_number;
  }
  for (auto *bn : s->bunches) bn->bunch_inject(s->time);
}

void copy_rows(double **src, int rows, int cols, int ngz, double *out) {
  for (int i = 0; i < rows; i++)
    for (int k = 0; k < cols; k++) out[(size_t)i * ngz + k] = src[i][k];
}

}  // namespace

extern "C" {

void ref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int ref_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// pml: {comparative_l_1, comparative_l_2, comparative_l_3, sigma_1, sigma_2}
void *ref_create(double r_size, double z_size, int n_grid_r, int n_grid_z,
                 double dt, double current_time, double end_time, const double *pml) {
  RefSim *s = new RefSim();
  s->geom = new Geometry(r_size, z_size, n_grid_r, n_grid_z);
  s->geom->set_epsilon();
  // src/parameters.cpp:244-245: set_pml only when some comparative length is non-zero
  if (pml && (pml[0] != 0 || pml[1] != 0 || pml[2] != 0))
    s->geom->set_pml(pml[0], pml[1], pml[2], pml[3], pml[4]);
  s->time = new Time(current_time, 0.0, 0.0, end_time, dt);
  // init_fields: src/loadInitParam.cpp:250-260
  s->efield = new EField(s->geom);
  s->hfield = new HField(s->geom);
  s->efield->boundary_conditions();
  s->efield->set_homogeneous_efield(0., 0., 0.);
  s->hfield->set_homogeneous_h(0.0, 0., 0.);
  s->efield->set_fi_on_z();
  // init_particles: src/loadInitParam.cpp:142-150
  s->plist = new ParticlesList();
  s->rho_new = new ChargeDensity(s->geom);
  s->rho_old = new ChargeDensity(s->geom);
  s->rho_bunch = new ChargeDensity(s->geom);
  s->current = new Current(s->geom);
  // Current's constructor only zeroes [0, n-1) x [0, n-1); reset_j clears all.
  s->current->reset_j();
  return s;
}

// Species whose state is given explicitly (identical arrays go to the GPU).
// charge_array = charge * w and mass_array = mass * w, as the upstream
// initialisation computes them (src/particles.cpp:328-329).
int ref_add_species(void *h, const char *name, double charge_e, double mass_me, int n,
                    const double *r, const double *z, const double *vr,
                    const double *vphi, const double *vz, const double *w) {
  RefSim *s = (RefSim *)h;
  Particles *p = new Particles(keep_name(s, name), charge_e, mass_me, n, s->geom);
  for (int i = 0; i < n; i++) {
    p->pos[i][0] = r[i];
    p->pos[i][1] = 0.0;
    p->pos[i][2] = z[i];
    p->pos_old[i][0] = r[i];
    p->pos_old[i][1] = 0.0;
    p->pos_old[i][2] = z[i];
    p->vel[i][0] = vr[i];
    p->vel[i][1] = vphi[i];
    p->vel[i][2] = vz[i];
    p->charge_array[i] = p->charge * w[i];
    p->mass_array[i] = p->mass * w[i];
    p->is_alive[i] = true;
  }
  s->plist->part_list.push_back(p);
  return (int)s->plist->part_list.size() - 1;
}

// Species initialised by the upstream routines themselves (TESTMODE build:
// deterministic random_reverse sequences), src/loadInitParam.cpp:152-165.
int ref_add_species_upstream_init(void *h, const char *name, double charge_e, double mass_me,
                                  int n, double left_density, double right_density,
                                  double temperature) {
  RefSim *s = (RefSim *)h;
  Particles *p = new Particles(keep_name(s, name), charge_e, mass_me, n, s->geom);
  p->load_cylindrical_spatial_distribution(left_density, right_density, 0);
  p->velocity_distribution(temperature);
  for (int i = 0; i < n; i++) {
    p->pos_old[i][0] = p->pos[i][0];
    p->pos_old[i][1] = 0.0;
    p->pos_old[i][2] = p->pos[i][2];
  }
  s->plist->part_list.push_back(p);
  return (int)s->plist->part_list.size() - 1;
}

void ref_set_beam(void *h, double charge_e, double mass_me, int number_macro,
                  double bunch_length, double radius, double density, double velocity,
                  int number_bunches, double bunches_distance) {
  RefSim *s = (RefSim *)h;
  s->beam.enabled = true;
  s->beam.charge_e = charge_e;
  s->beam.mass_me = mass_me;
  s->beam.number_macro = number_macro;
  s->beam.bunch_length = bunch_length;
  s->beam.radius = radius;
  s->beam.density = density;
  s->beam.velocity = velocity;
  s->beam.number_bunches = number_bunches;
  s->beam.bunches_distance = bunches_distance;
}

// One pass of the upstream main loop body (src/loadInitParam.cpp:471-587),
// without the probe output.  Returns (int)(t/dt) evaluated before t += dt,
// the value the upstream dump schedule tests (src/loadInitParam.cpp:329).
int ref_step(void *h) {
  RefSim *s = (RefSim *)h;
  init_beam(s);
  s->hfield->calc_field(s->efield, s->time);
  s->current->reset_j();
  s->rho_old->reset_rho();
  s->rho_bunch->reset_rho();
  s->plist->step_v(s->efield, s->hfield, s->time);
  s->plist->full_current_distribution(s->current, s->time);
  s->efield->calc_field(s->hfield, s->time, s->current);
  s->rho_new->reset_rho();
  for (auto *b : s->bunches) b->charge_weighting(s->rho_bunch);
  int sched = (int)(s->time->current_time / s->time->delta_t);
  s->time->current_time = s->time->current_time + s->time->delta_t;
  return sched;
}

// Runs n steps and returns the wall time of the loop in seconds
// (steady_clock, loop only).
double ref_run(void *h, int n) {
  auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < n; i++) ref_step(h);
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double>(t1 - t0).count();
}

double ref_current_time(void *h) { return ((RefSim *)h)->time->current_time; }
int ref_species_count(void *h) { return (int)((RefSim *)h)->plist->part_list.size(); }
int ref_species_number(void *h, int idx) {
  return (int)((RefSim *)h)->plist->part_list[idx]->number;
}

// Component ids: 0 E_r, 1 E_phi, 2 E_z, 3 H_r, 4 H_phi, 5 H_z,
// 6 H_r half, 7 H_phi half, 8 H_z half, 9 J_r, 10 J_phi, 11 J_z,
// 12 rho_bunch (as left by the last step), 13 rho_beam as the upstream probe
// writes it (one more charge_weighting of every bunch, src/loadInitParam.cpp:361-366).
// out is [n_grid_r * n_grid_z] row-major; cells outside an array's allocation are 0.
int ref_get_field(void *h, int comp, double *out) {
  RefSim *s = (RefSim *)h;
  int nr = s->geom->n_grid_r, nz = s->geom->n_grid_z;
  memset(out, 0, sizeof(double) * (size_t)nr * nz);
  switch (comp) {
    case 0: copy_rows(s->efield->field_r, nr, nz, nz, out); break;
    case 1: copy_rows(s->efield->field_phi, nr, nz, nz, out); break;
    case 2: copy_rows(s->efield->field_z, nr, nz, nz, out); break;
    case 3: copy_rows(s->hfield->field_r, nr, nz, nz, out); break;
    case 4: copy_rows(s->hfield->field_phi, nr, nz, nz, out); break;
    case 5: copy_rows(s->hfield->field_z, nr, nz, nz, out); break;
    case 6: copy_rows(s->hfield->field_r_half_time, nr, nz - 1, nz, out); break;
    case 7: copy_rows(s->hfield->field_phi_half_time, nr - 1, nz - 1, nz, out); break;
    case 8: copy_rows(s->hfield->field_z_half_time, nr - 1, nz - 1, nz, out); break;
    case 9: copy_rows(s->current->get_j_r(), nr, nz, nz, out); break;
    case 10: copy_rows(s->current->get_j_phi(), nr, nz, nz, out); break;
    case 11: copy_rows(s->current->get_j_z(), nr, nz, nz, out); break;
    case 12: copy_rows(s->rho_bunch->get_rho(), nr, nz, nz, out); break;
    case 13:
      for (auto *b : s->bunches) b->charge_weighting(s->rho_bunch);
      copy_rows(s->rho_bunch->get_rho(), nr, nz, nz, out);
      break;
    default: return -1;
  }
  return 0;
}

// Overwrites a field component (used to seed non-zero fields in parity cases).
int ref_set_field(void *h, int comp, const double *in) {
  RefSim *s = (RefSim *)h;
  int nr = s->geom->n_grid_r, nz = s->geom->n_grid_z;
  double **dst = nullptr;
  int rows = nr, cols = nz;
  switch (comp) {
    case 0: dst = s->efield->field_r; break;
    case 1: dst = s->efield->field_phi; break;
    case 2: dst = s->efield->field_z; break;
    case 3: dst = s->hfield->field_r; break;
    case 4: dst = s->hfield->field_phi; break;
    case 5: dst = s->hfield->field_z; break;
    case 6: dst = s->hfield->field_r_half_time; cols = nz - 1; break;
    case 7: dst = s->hfield->field_phi_half_time; rows = nr - 1; cols = nz - 1; break;
    case 8: dst = s->hfield->field_z_half_time; rows = nr - 1; cols = nz - 1; break;
    default: return -1;
  }
  for (int i = 0; i < rows; i++)
    for (int k = 0; k < cols; k++) dst[i][k] = in[(size_t)i * nz + k];
  return 0;
}

// Particle state of list entry idx (plasma species first, then bunches).
int ref_get_species(void *h, int idx, double *r, double *z, double *vr, double *vphi,
                    double *vz, double *q, double *m, unsigned char *alive) {
  RefSim *s = (RefSim *)h;
  if (idx < 0 || idx >= (int)s->plist->part_list.size()) return -1;
  Particles *p = s->plist->part_list[idx];
  for (unsigned int i = 0; i < p->number; i++) {
    if (r) r[i] = p->pos[i][0];
    if (z) z[i] = p->pos[i][2];
    if (vr) vr[i] = p->vel[i][0];
    if (vphi) vphi[i] = p->vel[i][1];
    if (vz) vz[i] = p->vel[i][2];
    if (q) q[i] = p->charge_array[i];
    if (m) m[i] = p->mass_array[i];
    if (alive) alive[i] = p->is_alive[i] ? 1 : 0;
  }
  return 0;
}

// Upstream charge weighting of every species into a fresh grid
// (src/particles.cpp:101-226, src/particlesList.cpp:14-18).
void ref_charge_density(void *h, double *out) {
  RefSim *s = (RefSim *)h;
  s->rho_new->reset_rho();
  s->plist->charge_weighting(s->rho_new);
  int nr = s->geom->n_grid_r, nz = s->geom->n_grid_z;
  copy_rows(s->rho_new->get_rho(), nr, nz, nz, out);
}

// The dump_data diagnostics (src/loadInitParam.cpp:369-390) of list entry
// idx: TemperatureClassic reset/calc_t/normalize (t: [n_grid_r-1][n_grid_z-1])
// and ParticlesDensity reset/calc_density (density, rows i <= n_grid_r-1,
// columns k <= n_grid_z-1 as written).  Both constructors size their arrays
// one row and one column short of what reset() and the weighting write; the
// handle keeps one instance of each and the tests use grids whose
// n_grid_r - 1 and n_grid_z - 1 are even, where glibc's 16-byte chunk
// rounding leaves the extra element inside each allocation.
int ref_temperature(void *h, int idx, double *out) {
  RefSim *s = (RefSim *)h;
  if (idx < 0 || idx >= (int)s->plist->part_list.size()) return -1;
  Particles *p = s->plist->part_list[idx];
  if (!cells_inside(s, p)) return -2;
  if (!s->temperature) s->temperature = new TemperatureClassic(s->geom);
  s->temperature->reset();
  s->temperature->calc_t(p);
  s->temperature->normalize(p);
  const int nr = s->geom->n_grid_r, nz = s->geom->n_grid_z;
  copy_rows(s->temperature->t, nr - 1, nz - 1, nz - 1, out);
  return 0;
}

int ref_density(void *h, int idx, double *out) {
  RefSim *s = (RefSim *)h;
  if (idx < 0 || idx >= (int)s->plist->part_list.size()) return -1;
  Particles *p = s->plist->part_list[idx];
  if (!cells_inside(s, p)) return -2;
  if (!s->density) s->density = new ParticlesDensity(s->geom);
  s->density->reset();
  s->density->calc_density(p);
  const int nr = s->geom->n_grid_r, nz = s->geom->n_grid_z;
  copy_rows(s->density->density, nr, nz, nz, out);
  return 0;
}

// PoissonDirichlet::poisson_solve(efield, rho) with rho given
// ([n_grid_r][n_grid_z]); returns phi, E_r and E_z after the solve.
int ref_poisson_dirichlet(void *h, const double *rho, double *fi, double *er, double *ez) {
  RefSim *s = (RefSim *)h;
  const int nr = s->geom->n_grid_r, nz = s->geom->n_grid_z;
  double **r = s->rho_new->get_rho();
  for (int i = 0; i < nr; i++)
    for (int k = 0; k < nz; k++) r[i][k] = rho[(size_t)i * nz + k];
  PoissonDirichlet solver(s->geom);
  solver.poisson_solve(s->efield, s->rho_new);
  copy_rows(s->efield->fi, nr, nz, nz, fi);
  copy_rows(s->efield->field_r, nr, nz, nz, er);
  copy_rows(s->efield->field_z, nr, nz, nz, ez);
  return 0;
}

double ref_sigma(void *h, int i, int k) { return ((RefSim *)h)->geom->sigma[i][k]; }

void ref_destroy(void *h) {
  RefSim *s = (RefSim *)h;
  // The upstream destructors free row by row with mismatched bounds
  // (src/field.cpp:28-35, src/hField.cpp:49-62); the process-lifetime leak of
  // a test handle is preferred to running them.
  for (char *c : s->names) free(c);
  delete s;
}

}  // extern "C"
