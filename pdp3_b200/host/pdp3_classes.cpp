// Upstream-style C++ classes over the pdp3g C ABI (see pdp3_classes.h).
#include "pdp3_classes.h"

#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <stdexcept>
#include <memory>

namespace pdp3gpu {

namespace {
constexpr double EL_CHARGE = 1.6E-19;  // include/constant.h:10-27
constexpr double EL_MASS = 9.1E-31;
constexpr double PI = 3.1415926535897932;

std::map<Geometry *, std::unique_ptr<Device>> &registry() {
  static std::map<Geometry *, std::unique_ptr<Device>> r;
  return r;
}

Time *g_last_time = nullptr;  // the run's Time, remembered for lazily created contexts
}  // namespace

void check(pdp3g_status st, pdp3g_ctx *ctx, const char *what) {
  if (st == PDP3G_OK) return;
  std::string msg = std::string(what) + ": " + pdp3g_status_string(st);
  if (ctx) {
    const char *e = pdp3g_last_error(ctx);
    if (e && *e) msg += std::string(" (") + e + ")";
  }
  throw Error(st, msg);
}

Device &Device::of(Geometry *geom) {
  auto &r = registry();
  auto it = r.find(geom);
  if (it == r.end()) {
    auto d = std::make_unique<Device>();
    d->geom_ = geom;
    it = r.emplace(geom, std::move(d)).first;
  }
  return *it->second;
}

pdp3g_ctx *Device::ctx(Time *time) {
  if (time) g_last_time = time;
  if (ctx_) return ctx_;
  Time *t = time ? time : g_last_time;
  if (!t) throw Error(PDP3G_INVALID_ARG, "pdp3gpu: no Time known when the device is first used");
  pdp3g_config cfg = {};
  cfg.r_size = geom_->r_size;
  cfg.z_size = geom_->z_size;
  cfg.n_grid_r = geom_->n_grid_r;
  cfg.n_grid_z = geom_->n_grid_z;
  cfg.dt = t->delta_t;
  cfg.current_time = t->current_time;
  cfg.pml_l1 = geom_->pml[0];
  cfg.pml_l2 = geom_->pml[1];
  cfg.pml_l3 = geom_->pml[2];
  cfg.pml_sigma1 = geom_->pml[3];
  cfg.pml_sigma2 = geom_->pml[4];
  cfg.pusher = pusher;
  cfg.precision = precision;
  cfg.device = device;
  check(pdp3g_create(&cfg, &ctx_), nullptr, "pdp3g_create");
  return ctx_;
}

Device::~Device() {
  if (ctx_) pdp3g_destroy(ctx_);
}

// ------------------------------------------------------------------ Geometry

Geometry::Geometry(double rs, double zs, int ngr, int ngz)
    : r_size(rs), z_size(zs), n_grid_r(ngr), n_grid_z(ngz) {
  dr = get_dr();
  dz = get_dz();
}

void Geometry::set_pml(double l1, double l2, double l3, double sigma1, double sigma2) {
  pml[0] = l1;
  pml[1] = l2;
  pml[2] = l3;
  pml[3] = sigma1;
  pml[4] = sigma2;
}

Geometry::~Geometry() { registry().erase(this); }

// --------------------------------------------------------------------- grids

static double **make_rows(double *base, int nr, int nz) {
  double **r = new double *[nr];
  for (int i = 0; i < nr; i++) r[i] = base + (size_t)i * nz;
  return r;
}

Field::Field(Geometry *g) : geom1(g) {
  const size_t ng = (size_t)g->n_grid_r * g->n_grid_z;
  store_.assign(3 * ng, 0.0);
  field_r = make_rows(store_.data(), g->n_grid_r, g->n_grid_z);
  field_phi = make_rows(store_.data() + ng, g->n_grid_r, g->n_grid_z);
  field_z = make_rows(store_.data() + 2 * ng, g->n_grid_r, g->n_grid_z);
}

Field::~Field() {
  delete[] field_r;
  delete[] field_phi;
  delete[] field_z;
}

void Field::fetch(int comp, double **dst) {
  pdp3g_ctx *c = Device::of(geom1).ctx(nullptr);
  check(pdp3g_get_field(c, comp, dst[0]), c, "pdp3g_get_field");
}

void EField::calc_field(HField *, Time *t, Current *) {
  pdp3g_ctx *c = Device::of(geom1).ctx(t);
  check(pdp3g_calc_e(c), c, "EField::calc_field");
}

void EField::download() {
  fetch(PDP3G_E_R, field_r);
  fetch(PDP3G_E_PHI, field_phi);
  fetch(PDP3G_E_Z, field_z);
}

// E gather on the host mirrors (EField::get_field, src/eField.cpp:204-316);
// the GPU step gathers on the device, this serves host-side probes.
double *EField::get_field(double radius, double longitude) {
  const double dr = geom1->dr, dz = geom1->dz;
  auto cell = [](double x, double d) { int c = (int)std::ceil(x / d) - 1; return c < 0 ? 0 : c; };
  auto one = [&](double **f, bool rhalf, bool zhalf) {
    const double r1 = radius - 0.5 * dr, r3 = radius + 0.5 * dr;
    const int i = rhalf ? cell(radius - 0.5 * dr, dr) : cell(radius, dr);
    const int k = zhalf ? cell(longitude - 0.5 * dz, dz) : cell(longitude, dz);
    double v1, v2, r2;
    if (rhalf) {
      v1 = PI * dz * dr * dr * 2.0 * (i + 1);
      v2 = PI * dz * dr * dr * 2.0 * (i + 3);
      r2 = (i + 1) * dr;
    } else {
      v1 = radius > dr ? PI * dz * dr * dr * 2.0 * i : PI * dz * dr * dr / 4.;
      v2 = PI * dz * dr * dr * 2.0 * (i + 2);
      r2 = (i + 0.5) * dr;
    }
    const double dz1 = zhalf ? (k + 1.5) * dz - longitude : (k + 1) * dz - longitude;
    const double dz2 = zhalf ? longitude - (k + 0.5) * dz : longitude - k * dz;
    double a = 0;
    a = a + f[i][k] * PI * dz1 * (r2 * r2 - r1 * r1) / v1;
    a = a + f[i + 1][k] * PI * dz1 * (r3 * r3 - r2 * r2) / v2;
    a = a + f[i][k + 1] * PI * dz2 * (r2 * r2 - r1 * r1) / v1;
    a = a + f[i + 1][k + 1] * PI * dz2 * (r3 * r3 - r2 * r2) / v2;
    return a;
  };
  double *out = new double[3];
  out[0] = one(field_r, true, false);
  out[1] = one(field_phi, false, false);
  out[2] = one(field_z, false, true);
  return out;
}

HField::HField(Geometry *g) : Field(g) {
  const size_t ng = (size_t)g->n_grid_r * g->n_grid_z;
  half_.assign(3 * ng, 0.0);
  field_r_half_time = make_rows(half_.data(), g->n_grid_r, g->n_grid_z);
  field_phi_half_time = make_rows(half_.data() + ng, g->n_grid_r, g->n_grid_z);
  field_z_half_time = make_rows(half_.data() + 2 * ng, g->n_grid_r, g->n_grid_z);
}

HField::~HField() {
  delete[] field_r_half_time;
  delete[] field_phi_half_time;
  delete[] field_z_half_time;
}

void HField::calc_field(EField *, Time *t) {
  pdp3g_ctx *c = Device::of(geom1).ctx(t);
  check(pdp3g_calc_h(c), c, "HField::calc_field");
}

void HField::download() {
  fetch(PDP3G_H_R, field_r);
  fetch(PDP3G_H_PHI, field_phi);
  fetch(PDP3G_H_Z, field_z);
  fetch(PDP3G_H_R_HALF, field_r_half_time);
  fetch(PDP3G_H_PHI_HALF, field_phi_half_time);
  fetch(PDP3G_H_Z_HALF, field_z_half_time);
}

Current::Current(Geometry *g) : geom1(g) {
  const size_t ng = (size_t)g->n_grid_r * g->n_grid_z;
  store_.assign(3 * ng, 0.0);
  j_r = make_rows(store_.data(), g->n_grid_r, g->n_grid_z);
  j_phi = make_rows(store_.data() + ng, g->n_grid_r, g->n_grid_z);
  j_z = make_rows(store_.data() + 2 * ng, g->n_grid_r, g->n_grid_z);
}

Current::~Current() {
  delete[] j_r;
  delete[] j_phi;
  delete[] j_z;
}

static double **current_fetch(Geometry *g, int comp, double **dst) {
  pdp3g_ctx *c = Device::of(g).ctx(nullptr);
  check(pdp3g_get_field(c, comp, dst[0]), c, "Current::get_j");
  return dst;
}

double **Current::get_j_r() { return current_fetch(geom1, PDP3G_J_R, j_r); }
double **Current::get_j_phi() { return current_fetch(geom1, PDP3G_J_PHI, j_phi); }
double **Current::get_j_z() { return current_fetch(geom1, PDP3G_J_Z, j_z); }

void Current::reset_j() {
  pdp3g_ctx *c = Device::of(geom1).ctx(nullptr);
  check(pdp3g_reset_j(c), c, "Current::reset_j");
}

ChargeDensity::ChargeDensity(Geometry *g) : geom1(g) {
  store_.assign((size_t)g->n_grid_r * g->n_grid_z, 0.0);
  rho = make_rows(store_.data(), g->n_grid_r, g->n_grid_z);
}

ChargeDensity::~ChargeDensity() { delete[] rho; }

void ChargeDensity::reset_rho() { std::fill(store_.begin(), store_.end(), 0.0); }

// ----------------------------------------------------------------- particles

Particles::Particles(const char *p_name, double p_charge, double p_mass, int p_number,
                     Geometry *geom)
    : geom1(geom) {
  name = strdup(p_name ? p_name : "species");
  charge = p_charge * EL_CHARGE;  // src/particles.cpp:30-32
  mass = p_mass * EL_MASS;
  number = (unsigned)p_number;
  charge_array = new double[number];
  mass_array = new double[number];
  is_alive = new bool[number];
  pos_store_.assign(3 * (size_t)number, 0.0);
  vel_store_.assign(3 * (size_t)number, 0.0);
  pos = new double *[number];
  vel = new double *[number];
  for (unsigned i = 0; i < number; i++) {
    pos[i] = pos_store_.data() + 3 * (size_t)i;
    vel[i] = vel_store_.data() + 3 * (size_t)i;
    is_alive[i] = true;
    charge_array[i] = 0;
    mass_array[i] = 0;
  }
  Device::of(geom).pending.push_back(this);
}

Particles::~Particles() {
  free(name);
  delete[] charge_array;
  delete[] mass_array;
  delete[] is_alive;
  delete[] pos;
  delete[] vel;
}

void Particles::load_cylindrical_spatial_distribution(double n1, double n2,
                                                      double left_plasma_boundary) {
  spatial_set_ = true;
  init_n1_ = n1;
  init_n2_ = n2;
  init_left_ = left_plasma_boundary;
}

void Particles::velocity_distribution(double tempr_ev) {
  velocity_set_ = true;
  init_tempr_ = tempr_ev;
}

void Particles::upload(pdp3g_ctx *ctx) {
  if (spatial_set_ || velocity_set_) {
    if (!(spatial_set_ && velocity_set_))
      throw std::runtime_error(std::string(name) +
                               ": load_cylindrical_spatial_distribution and "
                               "velocity_distribution are generated together");
    int32_t sid = -1;
    check(pdp3g_add_species_upstream(ctx, charge / EL_CHARGE, mass / EL_MASS, number, init_n1_,
                                     init_n2_, init_left_, init_tempr_, &sid),
          ctx, "pdp3g_add_species_upstream");
    id = sid;
    download();
    return;
  }
  std::vector<double> r(number), z(number), vr(number), vp(number), vz(number), w(number);
  std::vector<uint8_t> alive(number);
  bool all_alive = true;
  for (unsigned i = 0; i < number; i++) {
    r[i] = pos[i][0];
    z[i] = pos[i][2];
    vr[i] = vel[i][0];
    vp[i] = vel[i][1];
    vz[i] = vel[i][2];
    w[i] = charge_array[i] / charge;  // the weight charge_array = charge * w
    alive[i] = is_alive[i] ? 1 : 0;
    all_alive = all_alive && is_alive[i];
  }
  int32_t sid = -1;
  check(pdp3g_add_species(ctx, charge / EL_CHARGE, mass / EL_MASS, number, r.data(), z.data(),
                          vr.data(), vp.data(), vz.data(), w.data(),
                          all_alive ? nullptr : alive.data(), &sid),
        ctx, "pdp3g_add_species");
  id = sid;
}

void Particles::download() {
  if (id < 0) return;
  pdp3g_ctx *c = Device::of(geom1).ctx(nullptr);
  std::vector<double> r(number), z(number), vr(number), vp(number), vz(number), w(number);
  std::vector<uint8_t> alive(number);
  check(pdp3g_get_species(c, id, r.data(), z.data(), vr.data(), vp.data(), vz.data(), w.data(),
                          alive.data()),
        c, "pdp3g_get_species");
  for (unsigned i = 0; i < number; i++) {
    pos[i][0] = r[i];
    pos[i][1] = 0.0;
    pos[i][2] = z[i];
    vel[i][0] = vr[i];
    vel[i][1] = vp[i];
    vel[i][2] = vz[i];
    charge_array[i] = charge * w[i];
    mass_array[i] = mass * w[i];
    is_alive[i] = alive[i] != 0;
  }
}

void Particles::charge_weighting(ChargeDensity *ro1) {
  if (id < 0) return;
  pdp3g_ctx *c = Device::of(geom1).ctx(nullptr);
  std::vector<double> tmp((size_t)geom1->n_grid_r * geom1->n_grid_z);
  check(pdp3g_charge_density(c, 1u << id, tmp.data()), c, "charge_weighting");
  for (size_t j = 0; j < tmp.size(); j++) ro1->store_[j] += tmp[j];
}

Bunch::Bunch(char *p_name, double p_charge, double p_mass, int p_number, Geometry *geom,
             double b_duration, double b_radius, double b_density, double b_init_velocity,
             int b_number, double h_duration)
    : Particles(p_name, p_charge, p_mass, p_number, geom),
      duration(b_duration),
      bunch_number(b_number),
      hole_duration(h_duration),
      density(b_density),
      velocity(b_init_velocity),
      radius(b_radius) {
  for (unsigned i = 0; i < number; i++) is_alive[i] = false;
}

void Bunch::upload(pdp3g_ctx *ctx) {
  int32_t sid = -1;
  check(pdp3g_add_bunch(ctx, charge / EL_CHARGE, mass / EL_MASS, number, duration, radius, density,
                        velocity, (int32_t)bunch_number, hole_duration, &sid),
        ctx, "pdp3g_add_bunch");
  id = sid;
}

static void upload_pending(Geometry *g, Time *t) {
  Device &d = Device::of(g);
  pdp3g_ctx *c = d.ctx(t);
  for (Particles *p : d.pending) p->upload(c);
  d.pending.clear();
}

void Bunch::bunch_inject(Time *time) {
  // one device call injects every bunch for the current time; the upstream
  // loop calls this once per bunch per step (src/loadInitParam.cpp:246-247)
  static double last_time = -1.0;
  static pdp3g_ctx *last_ctx = nullptr;
  upload_pending(geom1, time);
  pdp3g_ctx *c = Device::of(geom1).ctx(time);
  if (c == last_ctx && time->current_time == last_time) return;
  check(pdp3g_set_time(c, time->current_time), c, "pdp3g_set_time");
  check(pdp3g_inject(c), c, "Bunch::bunch_inject");
  last_time = time->current_time;
  last_ctx = c;
}

void ParticlesList::step_v(EField *e, HField *, Time *t) {
  // gather + push + first half move run inside the fused kernel launched by
  // full_current_distribution; here the species are made resident
  upload_pending(e->geom1, t);
}

void ParticlesList::full_current_distribution(Current *current, Time *t) {
  upload_pending(current->geom1, t);
  pdp3g_ctx *c = Device::of(current->geom1).ctx(t);
  check(pdp3g_set_time(c, t->current_time), c, "pdp3g_set_time");
  check(pdp3g_push_deposit(c), c, "full_current_distribution");
  check(pdp3g_sync(c), c, "full_current_distribution");
}

void ParticlesList::charge_weighting(ChargeDensity *rho) {
  for (Particles *p : part_list) p->charge_weighting(rho);
}

void BoundaryMaxwellConditions::specify_initial_field(Geometry *cyl_geom, double E_fi_upper,
                                                      double E_fi_left, double E_fi_right) {
  pdp3g_ctx *c = Device::of(cyl_geom).ctx(nullptr);
  e_fld->download();
  const int n1 = cyl_geom->n_grid_r, n2 = cyl_geom->n_grid_z;
  for (int i = 0; i < n1; i++) {
    e_fld->field_phi[i][0] = E_fi_left;
    e_fld->field_phi[i][n2 - 1] = E_fi_right;
  }
  for (int k = 0; k < n2; k++) e_fld->field_phi[n1 - 1][k] = E_fi_upper;
  check(pdp3g_set_field(c, PDP3G_E_PHI, e_fld->field_phi[0]), c, "specify_initial_field");
}



// ------------------------------------------------------------------ probes

namespace {

void make_directory(const std::string &path) {  // lib::make_directory (mkdir -p)
  std::string cur;
  for (size_t i = 0; i <= path.size(); i++) {
    if (i == path.size() || path[i] == '/') {
      if (!cur.empty()) mkdir(cur.c_str(), 0755);
    }
    if (i < path.size()) cur += path[i];
  }
}

}  // namespace

ProbePlain::ProbePlain(const char *c_path, const char *c_component, int c_type, int c_start_r,
                       int c_start_z, int c_end_r, int c_end_z, bool c_compress,
                       int c_compress_level, int c_schedule, const char *c_specie) {
  snprintf(path, sizeof(path), "%s", c_path);
  snprintf(component, sizeof(component), "%s", c_component);
  snprintf(specie, sizeof(specie), "%s", c_specie);
  type = c_type;
  start_r = c_start_r;
  start_z = c_start_z;
  end_r = c_end_r;
  end_z = c_end_z;
  schedule = c_schedule;
  compress = c_compress;
  compress_level = c_compress_level;
  if (compress) std::cerr << "WARNING! compression is not supported by plaintext backend" << std::endl;
  std::string result_component = c_component;
  if (strcmp(c_specie, "none") != 0) result_component += std::string("/") + c_specie;
  char buf[512];
  switch (type) {
    case 0:
      snprintf(buf, sizeof(buf), "%s/%s/frame_%d:%d_%d:%d", c_path, result_component.c_str(),
               c_start_r, c_start_z, c_end_r, c_end_z);
      break;
    case 1:
      snprintf(buf, sizeof(buf), "%s/%s/col_%d", c_path, result_component.c_str(), c_start_z);
      break;
    case 2:
      snprintf(buf, sizeof(buf), "%s/%s/row_%d", c_path, result_component.c_str(), c_start_r);
      break;
    case 3:
      snprintf(buf, sizeof(buf), "%s/%s/dot_%d_%d", c_path, result_component.c_str(), c_start_r,
               c_start_z);
      break;
    default:
      snprintf(buf, sizeof(buf), "%s/%s/mpframe_%d:%d_%d:%d", c_path, result_component.c_str(),
               c_start_r, c_start_z, c_end_r, c_end_z);
      break;
  }
  path_result_ = buf;
  make_directory(path_result_);
}

std::string ProbePlain::get_data_path(const char *name) const {
  return path_result_ + "/" + name + ".dat";
}

static int probe_component(const char *c) {
  static const char *names[] = {"E_r", "E_phi", "E_z", "H_r", "H_phi", "H_z"};
  for (int i = 0; i < 6; i++)
    if (strcmp(c, names[i]) == 0) return PDP3G_E_R + i;
  if (strcmp(c, "J_r") == 0) return PDP3G_J_R;
  if (strcmp(c, "J_phi") == 0) return PDP3G_J_PHI;
  if (strcmp(c, "J_z") == 0) return PDP3G_J_Z;
  if (strcmp(c, "rho_beam") == 0) return PDP3G_PROBE_RHO_BEAM;
  return -1;
}

void ProbePlain::write(const char *name, pdp3g_ctx *ctx, int species_id) {
  const bool is_t = strcmp(component, "T") == 0, is_density = strcmp(component, "density") == 0;
  const bool per_species = is_t || is_density;
  const int comp = is_t ? PDP3G_PROBE_T : is_density ? PDP3G_PROBE_DENSITY : probe_component(component);
  if (comp < 0) {
    std::cerr << "WARNING! probe for component ``" << component << "'' does not exist. Skipping"
              << std::endl;
    return;
  }
  long long cap = 1;
  if (type == 0) cap = (long long)(end_r - start_r) * (end_z - start_z);
  if (type == 1) cap = end_r - start_r;
  if (type == 2) cap = end_z - start_z;
  std::vector<double> v((size_t)std::max<long long>(cap, 1));
  int64_t n = 0;
  if (per_species)
    check(pdp3g_probe_read_species(ctx, comp, species_id, type, start_r, start_z, end_r, end_z,
                                   v.data(), (int64_t)v.size(), &n),
          ctx, "probe_read_species");
  else
    check(pdp3g_probe_read(ctx, comp, type, start_r, start_z, end_r, end_z, v.data(),
                           (int64_t)v.size(), &n),
          ctx, "probe_read");
  std::ofstream out_file(get_data_path(name), std::ios::app);
  for (int64_t i = 0; i < n; i++) out_file << v[(size_t)i] << " ";
}

void ProbePlain::mpwrite(const char *name, pdp3g_ctx *ctx, int species_id) {
  const int64_t cap = pdp3g_species_size(ctx, species_id);
  std::vector<double> a[5];
  for (auto &x : a) x.resize((size_t)std::max<int64_t>(cap, 1));
  int64_t n = 0;
  check(pdp3g_probe_particles(ctx, species_id, start_r, start_z, end_r, end_z, a[0].data(),
                              a[1].data(), a[2].data(), a[3].data(), a[4].data(), cap, &n),
        ctx, "probe_particles");
  static const char *suffix[5] = {"_pos_r", "_pos_z", "_vel_r", "_vel_phi", "_vel_z"};
  for (int c = 0; c < 5; c++) {
    std::ofstream f(get_data_path((std::string(name) + suffix[c]).c_str()), std::ios::app);
    for (int64_t i = 0; i < n; i++) f << a[c][(size_t)i] << " ";
  }
}

void dump_probes(std::vector<ProbePlain *> &probes, pdp3g_ctx *ctx, Time *time,
                 int frames_per_file, const std::vector<std::string> &species_names) {
  for (ProbePlain *w : probes) {
    if ((int)(time->current_time / time->delta_t) % w->schedule != 0) continue;
    char file_name[64];
    snprintf(file_name, sizeof(file_name), "%d", (int)floor(w->step_number / frames_per_file));
    if (w->type == 4) {
      // mpframes are named by their step number (no frames per file)
      snprintf(file_name, sizeof(file_name), "%d", w->step_number);
      for (size_t s = 0; s < species_names.size(); s++)
        if (species_names[s] == w->component) w->mpwrite(file_name, ctx, (int)s);
    } else if (strcmp(w->component, "T") == 0 || strcmp(w->component, "density") == 0) {
      // TemperatureClassic / ParticlesDensity of the species the probe names
      for (size_t s = 0; s < species_names.size(); s++)
        if (species_names[s] == w->specie) w->write(file_name, ctx, (int)s);
    } else {
      w->write(file_name, ctx);
    }
    ++w->step_number;
  }
}

}  // namespace pdp3gpu
