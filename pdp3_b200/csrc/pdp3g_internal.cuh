// Internal declarations shared by the pdp3g CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pdp3g {

// include/constant.h:10-27 (the upstream rounded SI constants)
constexpr double PI = 3.1415926535897932;
constexpr double EPSILON0 = 8.85E-12;
constexpr double EL_MASS = 9.1E-31;
constexpr double EL_CHARGE = 1.6E-19;
constexpr double LIGHT_SPEED = 3.0E8;
constexpr double MAGN_CONST = 1.26E-6;
constexpr double MNZL = 1e-15;
constexpr double LIGHT_SPEED_POW_2 = 9.0e16;  // pow(3e8, 2), exact in binary64

// device error flags (the upstream code calls exit(1) in these cases)
enum : unsigned { ERR_NAN = 1u, ERR_V_GE_C = 2u, ERR_OUT_OF_GRID = 4u };

enum { KIND_PLASMA = 0, KIND_BUNCH = 1 };

// Grid view passed by value to kernels.  All component arrays are
// [nr][nz] row-major doubles in one allocation.
struct GridDev {
  int nr, nz;
  double r_size, z_size, dr, dz, dt;
  double *er, *ephi, *ez;
  double *hr, *hphi, *hz;
  double *hrh, *hphih, *hzh;
  double *jr, *jphi, *jz;
  const double *sigma;
  unsigned *err;
};

// FP64 structure-of-arrays species (the plain form).
struct SpeciesDev {
  double *r, *z, *vr, *vphi, *vz;
  const double *w;
  uint8_t *alive;      // nullptr: every particle alive
  long long n;
  double charge, mass; // per unit weight (charge_e*e, mass_me*m_e)
  int kind;
};

// host-side launchers (fields.cu, particles_f64.cu, diag.cu)
void launch_yee_h(const GridDev &g, cudaStream_t st);
void launch_yee_e(const GridDev &g, cudaStream_t st);
void launch_push_deposit_f64(const GridDev &g, const SpeciesDev &s, int pusher, int n_sm,
                             cudaStream_t st);
void launch_charge_density_f64(const GridDev &g, const SpeciesDev &s, double *rho,
                               cudaStream_t st);
int diag_blocks();
void launch_grid_diag(const GridDev &g, const double *rho, const double *rho0, double *partials,
                      double *out, cudaStream_t st);
void launch_rho_norm(const GridDev &g, const double *rho, double *partials, double *out,
                     cudaStream_t st);
void launch_kinetic_f64(const SpeciesDev &s, double *partials, double *out, cudaStream_t st);
void launch_bunch_inject(const SpeciesDev &s, long long start, long long count, double dl,
                         double half_dz, double velocity, const double *inv_pow11,
                         cudaStream_t st);

}  // namespace pdp3g
