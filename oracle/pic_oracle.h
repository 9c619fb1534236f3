/*
 * CPU restatement of the PDP3 per-timestep particle-in-cell loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU kernels are compared
 * with; it is never linked into the product.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it (through ctypes).
 *
 * Every routine restates an upstream routine with the same floating-point
 * operation order (compiled without contraction or fast-math), so that on
 * identical inputs it reproduces the upstream FP64 step.  The upstream
 * file:line each routine follows is given beside its definition.
 *
 * Layout: every grid is one contiguous row-major [n_grid_r][n_grid_z] array
 * of doubles (upstream allocates row by row); particles are structure-of-
 * arrays.  Cells of an array that the upstream code never allocates or never
 * writes are kept at zero.
 */
#ifndef PDP3_PIC_ORACLE_H
#define PDP3_PIC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_BORIS_REL = 0, ORC_VAY = 1, ORC_BORIS_CLASSIC = 2 };
enum { ORC_PLASMA = 0, ORC_BUNCH = 1 };
/* error bits (upstream calls exit(1) in these cases) */
enum { ORC_ERR_NAN = 1, ORC_ERR_V_GE_C = 2 };

/* grid component ids */
enum {
  ORC_E_R = 0, ORC_E_PHI, ORC_E_Z, ORC_H_R, ORC_H_PHI, ORC_H_Z,
  ORC_H_R_HALF, ORC_H_PHI_HALF, ORC_H_Z_HALF, ORC_J_R, ORC_J_PHI, ORC_J_Z,
  ORC_SIGMA, ORC_NCOMP
};

void *orc_create(double r_size, double z_size, int n_grid_r, int n_grid_z, double dt,
                 double current_time, const double *pml /* l1,l2,l3,sigma1,sigma2 */,
                 int pusher);
void orc_destroy(void *sim);

/* plasma species: explicit state, charge/mass per particle = q_s*w, m_s*w */
int orc_add_species(void *sim, double charge_e, double mass_me, int n, const double *r,
                    const double *z, const double *vr, const double *vphi, const double *vz,
                    const double *w);
/* electron bunch (upstream Bunch, TESTMODE initialisation, src/bunch.cpp:6-80) */
int orc_add_bunch(void *sim, double charge_e, double mass_me, int n, double duration,
                  double radius, double density, double velocity, int bunch_number,
                  double hole_duration);

int orc_step(void *sim);          /* returns (int)(t/dt) before t += dt */
int orc_errors(void *sim);
double orc_time(void *sim);
int orc_species_n(void *sim, int idx);

int orc_get_grid(void *sim, int comp, double *out);
int orc_set_grid(void *sim, int comp, const double *in);
int orc_get_species(void *sim, int idx, double *r, double *z, double *vr, double *vphi,
                    double *vz, double *w, uint8_t *alive);
int orc_set_species(void *sim, int idx, const double *r, const double *z, const double *vr,
                    const double *vphi, const double *vz, const uint8_t *alive);
/* charge weighting (src/particles.cpp:101-226) of the species selected by
   mask (bit s = species s) into a fresh grid */
void orc_charge_density(void *sim, uint32_t species_mask, double *out);

/* standalone pieces (parity cases for single kernels) */
void orc_field_h(void *sim);
void orc_field_e(void *sim);
void orc_gather(void *sim, double r, double z, double *e3, double *h3);

/* upstream pseudo-random sequence (src/math/rand.cpp:40-53) */
double orc_random_reverse(double x, int power);

#ifdef __cplusplus
}
#endif
#endif
