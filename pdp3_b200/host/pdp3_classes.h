// C++ host layer with the upstream PDP3 class interfaces, running the step
// on a B200 through the pdp3g C ABI (include/pdp3g.h).
//
// The classes carry the upstream names, constructors, public members and
// methods of the hot path (include/geometry.h, pdp3Time.h, eField.h,
// hField.h, current.h, chargeDensity.h, particles.h, particlesList.h,
// bunch.h, boundaryMaxwellConditions.h), so LoadInitParam::run's loop body
// (src/loadInitParam.cpp:471-587) compiles against them unchanged:
//
//   init_beam();                                        -> Bunch::bunch_inject
//   hfield->calc_field(efield, time);                   -> pdp3g_calc_h
//   c_current->reset_j();                               -> pdp3g_reset_j
//   p_list->step_v(efield, hfield, time);               -> (fused below)
//   p_list->full_current_distribution(c_current, time); -> pdp3g_push_deposit
//   efield->calc_field(hfield, time, c_current);        -> pdp3g_calc_e
//   time->current_time += time->delta_t;                (host; read by injection)
//
// State lives on the GPU.  The public double** arrays are host mirrors,
// refreshed by download() (fields, currents, particles) — the upstream
// probes read them directly, so a host calls download() before dump_data.
// Errors that upstream turns into exit(1) raise pdp3gpu::Error.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "pdp3g.h"

namespace pdp3gpu {

struct Error : std::runtime_error {
  pdp3g_status status;
  Error(pdp3g_status st, const std::string &what) : std::runtime_error(what), status(st) {}
};

class Geometry;
class Time;
class EField;
class HField;
class Current;
class ChargeDensity;
class Particles;
class ParticlesList;

// One device simulation shared by the objects of a run (the upstream objects
// share a Geometry*); created on first use from the Geometry and Time.
class Device {
 public:
  static Device &of(Geometry *geom);
  pdp3g_ctx *ctx(Time *time);
  pdp3g_ctx *ctx_if_created() const { return ctx_; }
  int pusher = PDP3G_PUSHER_BORIS;
  int precision = PDP3G_FP64;
  int device = 0;
  std::vector<Particles *> pending;  // species not yet uploaded
  ~Device();

 private:
  Geometry *geom_ = nullptr;
  pdp3g_ctx *ctx_ = nullptr;
};

void check(pdp3g_status st, pdp3g_ctx *ctx, const char *what);

// Geometry, include/geometry.h:5-29
class Geometry {
 public:
  double r_size, z_size;
  int n_grid_r, n_grid_z;
  double dr, dz;
  double pml[5] = {0, 0, 0, 0, 0};
  Geometry(double rs, double zs, int ngr, int ngz);
  double get_dr() { return r_size / (n_grid_r - 1); }
  double get_dz() { return z_size / (n_grid_z - 1); }
  void set_epsilon() {}  // epsilon is 1 everywhere (src/geometry.cpp:33-39)
  void set_pml(double l1, double l2, double l3, double sigma1, double sigma2);
  ~Geometry();
};

// Time, include/pdp3Time.h:3-16
class Time {
 public:
  double current_time, start_time, relaxation_time, end_time, delta_t;
  Time(double ct, double st, double rt, double et, double dt)
      : current_time(ct), start_time(st), relaxation_time(rt), end_time(et), delta_t(dt) {}
};

// Field, include/field.h: three [n_grid_r][n_grid_z] host mirrors
class Field {
 public:
  Geometry *geom1;
  double **field_r, **field_phi, **field_z;
  explicit Field(Geometry *g);
  virtual ~Field();

 protected:
  std::vector<double> store_;
  double **rows(double *base);
  void fetch(int comp, double **dst);
};

class EField : public Field {
 public:
  explicit EField(Geometry *g) : Field(g) {}
  void calc_field(HField *h, Time *t, Current *j);  // src/eField.cpp:85-170
  void boundary_conditions() {}                     // device grids start at zero
  void set_homogeneous_efield(double, double, double) {}
  void set_fi_on_z() {}
  double *get_field(double radius, double longitude);  // caller deletes (upstream contract)
  void download();
};

class HField : public Field {
 public:
  double **field_r_half_time, **field_phi_half_time, **field_z_half_time;
  explicit HField(Geometry *g);
  ~HField() override;
  void calc_field(EField *e, Time *t);  // src/hField.cpp:93-157
  void set_homogeneous_h(double, double, double) {}
  void download();

 private:
  std::vector<double> half_;
};

class Current {
 public:
  Geometry *geom1;
  explicit Current(Geometry *g);
  ~Current();
  double **get_j_r();    // downloads
  double **get_j_phi();
  double **get_j_z();
  void reset_j();        // src/current.cpp:125-135

 private:
  std::vector<double> store_;
  double **j_r, **j_phi, **j_z;
};

class ChargeDensity {
 public:
  Geometry *geom1;
  explicit ChargeDensity(Geometry *g);
  ~ChargeDensity();
  double **get_rho() const { return rho; }
  void inc_rho(int i, int k, double value) { rho[i][k] += value; }
  void reset_rho();

 private:
  std::vector<double> store_;
  double **rho;
  friend class Particles;
};

// Particles, include/particles.h:34-165
class Particles {
 public:
  char *name;
  double charge, mass;          // SI, per physical particle
  unsigned int number;
  double *charge_array, *mass_array;
  double **pos, **vel;          // [number][3]
  bool *is_alive;
  Geometry *geom1;
  int id = -1;                  // species index on the device (-1: not uploaded)

  Particles(const char *p_name, double p_charge, double p_mass, int p_number, Geometry *geom);
  virtual ~Particles();
  void charge_weighting(ChargeDensity *ro1);  // src/particles.cpp:101-226
  // src/particles.cpp:278-331 and :228-276: recorded here and generated on
  // the device when the species is uploaded (pdp3g_add_species_upstream);
  // pos, vel, charge_array and mass_array are filled from the device then.
  void load_cylindrical_spatial_distribution(double n1, double n2, double left_plasma_boundary);
  void velocity_distribution(double tempr_ev);
  void download();                             // refresh pos/vel/is_alive
  virtual void upload(pdp3g_ctx *ctx);

 protected:
  std::vector<double> pos_store_, vel_store_;
  bool spatial_set_ = false, velocity_set_ = false;
  double init_n1_ = 0, init_n2_ = 0, init_left_ = 0, init_tempr_ = 0;
};

// Bunch, include/bunch.h:4-36
class Bunch : public Particles {
 public:
  double duration, bunch_number, hole_duration, density, velocity, radius;
  Bunch(char *p_name, double p_charge, double p_mass, int p_number, Geometry *geom,
        double b_duration, double b_radius, double b_density, double b_init_velocity, int b_number,
        double h_duration);
  void bunch_inject(Time *time);  // src/bunch.cpp:87-124
  void upload(pdp3g_ctx *ctx) override;
};

// ParticlesList, include/particlesList.h:9-26
class ParticlesList {
 public:
  std::vector<Particles *> part_list;
  void step_v(EField *e, HField *h, Time *t);
  void full_current_distribution(Current *current, Time *t);
  void charge_weighting(ChargeDensity *rho);
};

// ProbePlain, include/probePlain.h:7-33 and src/probePlain.cpp:1-224: the
// plain-text probe.  Files and formats are the upstream's: the result path
// <path>/<component>[/<specie>]/{frame_R0:Z0_R1:Z1, col_Z, row_R, dot_R_Z,
// mpframe_R0:Z0_R1:Z1}/<name>.dat, values printed with the stream's default
// format and a trailing space, appended per dump.  write() reads only the
// probe's region from the GPU (pdp3g_probe_read) instead of a host grid.
class ProbePlain {
 public:
  char path[256];
  char component[16];
  char specie[100];
  int type;  // 0 frame, 1 col, 2 row, 3 dot, 4 mpframe
  int start_r, start_z, end_r, end_z;
  bool compress;
  int compress_level;
  int schedule;
  int step_number = 0;
  ProbePlain(const char *c_path, const char *c_component, int c_type, int c_start_r,
             int c_start_z, int c_end_r, int c_end_z, bool c_compress, int c_compress_level,
             int c_schedule, const char *c_specie = "none");
  std::string get_data_path(const char *name) const;
  // types 0-3; species_id: the species of a per-species component (T, density)
  void write(const char *name, pdp3g_ctx *ctx, int species_id = -1);
  void mpwrite(const char *name, pdp3g_ctx *ctx, int species_id);  // type 4
  const std::string &result_path() const { return path_result_; }

 private:
  std::string path_result_;
};

// LoadInitParam::dump_data's probe loop (src/loadInitParam.cpp:319-398) for
// the grid components and mpframes: each probe whose schedule divides
// (int)(t / dt) writes file floor(step_number / frames_per_file).
// species_names: the species of the device context in order (mpframe probes
// name one as their component).
void dump_probes(std::vector<ProbePlain *> &probes, pdp3g_ctx *ctx, Time *time,
                 int frames_per_file, const std::vector<std::string> &species_names);

// BoundaryMaxwellConditions, include/boundaryMaxwellConditions.h:6-16
// (never instantiated by the upstream loop; kept for interface parity)
class BoundaryMaxwellConditions {
 public:
  EField *e_fld;
  explicit BoundaryMaxwellConditions(EField *e) : e_fld(e) {}
  // sets E_phi on the z = 0, z = Z and r = R walls (src/boundaryMaxwellConditions.cpp:17-38)
  void specify_initial_field(Geometry *cyl_geom, double E_fi_upper, double E_fi_left,
                             double E_fi_right);
};

}  // namespace pdp3gpu
