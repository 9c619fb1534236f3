// Internal declarations shared by the pdp3g CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>

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

// particles per CTA chunk of the FP32 particle phase (particles_f32.cuh)
constexpr int F32_CHUNK = 1024;

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
  // FP32 contexts only (else null): FP32 copies of E (3 grids) and of the
  // half-step H (3 grids, right after them), written by the Yee updates
  // beside the FP64 values
  float *e32, *hh32;
  // FP32 contexts only: the same 6 components per cell, q32[c * ncells +
  // i * (nz - 1) + k] = (f[i][k], f[i+1][k], f[i][k+1], f[i+1][k+1]) for the
  // cell (i, k), packed from e32/hh32 before each particle phase
  // (launch_pack_quads), so that the FP32 particle kernel gathers a
  // component with one 16-byte load
  const float4 *q32;
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

// FP32 cell-local species (particles_f32.cu).
struct SpeciesF32 {
  int *cell;           // i * (nz - 1) + k
  float *fr, *fz;      // in-cell offsets in (0, 1]
  float *ur, *uphi, *uz;  // gamma v / c
  const float *w;
  uint8_t *alive;      // bunch species only
  long long n;
  int kind;
  // species constants (FP32)
  float ke;     // charge dt / (2 mass c):  du per V/m (Boris)
  float kb;     // mu0 charge dt / (2 mass): rotation vector per A/m (Boris)
  float cr, cz; // c dt / (2 dr), c dt / (2 dz): half-step move per unit v/c, in cells
  float kphi;   // charge c / (2 pi dz dr^2): j_phi per (w u_phi/gamma x weight)
  float kz;     // charge / (4 pi dr^2 dt)
  float kr;     // charge / (2 pi dr dz dt)
  float vay_e;  // charge dt / mass (upstream Vay: e * 2 const1)
  float vay_b;  // 2 mu0 const1^3 (upstream Vay: b * mu0 const1 * 2 const1 * const1)
  float inv_c2; // 1 / c^2
};

// Where the FP32 particle phase writes its result: the input arrays (the
// step in place) or another state of the same species (the adjoint's
// recompute writes step s+1's state next to step s's; then particles the
// step skips, dead or not yet injected, are copied across).
struct SpeciesOut {
  int *cell;
  float *fr, *fz, *ur, *uphi, *uz;
  uint8_t *alive;
};

__host__ __device__ inline SpeciesOut in_place(const SpeciesF32 &s) {
  return SpeciesOut{s.cell, s.fr, s.fz, s.ur, s.uphi, s.uz, s.alive};
}

// Particles::charge_weighting per particle, src/particles.cpp:101-226: the
// node block (r_i, z_k) and the 4 values (nodes (r_i, z_k), (r_i+1, z_k),
// (r_i, z_k+1), (r_i+1, z_k+1)) of charge q at (r, z) with the upstream
// volume weights.
__device__ __forceinline__ void charge_weights(const GridDev &g, double r, double z, double q,
                                               int &r_i, int &z_k, double w[4]) {
  const double dr = g.dr, dz = g.dz;
  r_i = (int)ceil(r / dr) - 1;
  z_k = (int)ceil(z / dz) - 1;
  if (r_i < 0) r_i = 0;
  if (z_k < 0) z_k = 0;
  double r1, r2, r3, ro_v, v_1, v_2;
  const double dz1 = (z_k + 0.5) * dz - (z - 0.5 * dz);
  const double dz2 = (z + 0.5 * dz) - (z_k + 0.5) * dz;
  if (r > dr) {
    r1 = r - 0.5 * dr; r2 = (r_i + 0.5) * dr; r3 = r + 0.5 * dr;
    ro_v = q / (2. * PI * dz * dr * r);
    v_1 = PI * dz * dr * dr * 2.0 * (r_i);
    v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
    w[0] = ro_v * PI * dz1 * (r2 * r2 - r1 * r1) / v_1;
    w[1] = ro_v * PI * dz1 * (r3 * r3 - r2 * r2) / v_2;
    w[2] = ro_v * PI * dz2 * (r2 * r2 - r1 * r1) / v_1;
    w[3] = ro_v * PI * dz2 * (r3 * r3 - r2 * r2) / v_2;
  } else if (r <= dr / 2.) {
    r_i = 0;
    r2 = (r_i + 0.5) * dr; r3 = r + 0.5 * dr;
    ro_v = q / (PI * dz * (2. * r * r + dr * dr / 2.));
    v_1 = PI * dz * dr * dr / 4.;
    v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
    w[0] = ro_v * PI * dz1 * (dr * dr / 2. - r * dr + r * r) / v_1;
    w[1] = ro_v * PI * dz1 * (r3 * r3 - r2 * r2) / v_2;
    w[2] = ro_v * PI * dz2 * (dr * dr / 2. - r * dr + r * r) / v_1;
    w[3] = ro_v * PI * dz2 * (r3 * r3 - r2 * r2) / v_2;
  } else {
    r1 = r - 0.5 * dr; r2 = (r_i + 0.5) * dr; r3 = r + 0.5 * dr;
    ro_v = q / (2. * PI * dz * dr * r);
    v_1 = PI * dz * dr * dr / 4.;
    v_2 = PI * dz * dr * dr * 2.0 * (r_i + 1);
    w[0] = ro_v * PI * dz1 * (r2 * r2 - r1 * r1) / v_1;
    w[1] = ro_v * PI * dz1 * (r3 * r3 - r2 * r2) / v_2;
    w[2] = ro_v * PI * dz2 * (r2 * r2 - r1 * r1) / v_1;
    w[3] = ro_v * PI * dz2 * (r3 * r3 - r2 * r2) / v_2;
  }
}

// Segmented sum over runs of consecutive lanes with the same key: every lane
// of the warp calls it; afterwards the last lane of each run (returns true)
// holds the run's totals.  Particles sorted by cell form long runs, so the
// FP64 atomics that follow are one per run and node instead of one per
// particle and node on the same few addresses.  A lane that must not merge
// with its neighbours passes a key of its own (e.g. -2 - lane).
template <int N>
__device__ __forceinline__ bool warp_run_sum_f64(int key, double (&v)[N]) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int prev = __shfl_up_sync(FULL, key, 1);
  const int next = __shfl_down_sync(FULL, key, 1);
  const bool head = lane == 0 || prev != key;
  const bool tail = lane == 31 || next != key;
  const unsigned heads = __ballot_sync(FULL, head);
  const unsigned le = lane == 31 ? FULL : ((2u << lane) - 1u);
  const int seg_start = 31 - __clz(heads & le);
#pragma unroll
  for (int j = 0; j < N; j++) {
    double x = v[j];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const double y = __shfl_up_sync(FULL, x, off);
      if (lane >= seg_start + off) x += y;
    }
    v[j] = x;
  }
  return tail;
}

// rho += the charge weights of a warp's particles (charge_weights), one run
// sum per node block (r_i, z_k).  live: this lane holds a particle.  Blocks
// that reach outside the grid are not merged (their lanes raise
// ERR_OUT_OF_GRID for the nodes outside, as one particle would).
__device__ __forceinline__ void charge_run_add(const GridDev &g, double *rho, bool live, int r_i,
                                               int z_k, double (&w)[4]) {
  const bool inside = r_i <= g.nr - 2 && z_k <= g.nz - 2;
  const int key = !live ? -1 : (inside ? r_i * g.nz + z_k : -2 - (int)(threadIdx.x & 31));
  if (!warp_run_sum_f64<4>(key, w) || !live) return;
  const int ii[4] = {r_i, r_i + 1, r_i, r_i + 1}, kk[4] = {z_k, z_k, z_k + 1, z_k + 1};
#pragma unroll
  for (int j = 0; j < 4; j++) {
    if ((unsigned)ii[j] >= (unsigned)g.nr || (unsigned)kk[j] >= (unsigned)g.nz) {
      atomicOr(g.err, ERR_OUT_OF_GRID);
      continue;
    }
    atomicAdd(rho + (size_t)ii[j] * g.nz + kk[j], w[j]);
  }
}

// batched ensemble (ensemble.cu)
struct EnsRun {
  GridDev g;
  double t;
  long long h_begin, e_begin, j_begin, chunk_begin;  // prefixes of the index spaces
  int pusher;
};

struct EnsSpecies {
  SpeciesF32 s;
  int run;
  long long chunk_begin;
  int is_bunch;
  double duration, bunch_number, hole_duration, velocity;
  float uz_beam;
};

struct EnsembleDev {
  EnsRun *runs;
  int nruns;
  EnsSpecies *species;
  int nspecies;
  long long total_h, total_e, total_j, total_chunks;
  const double *inv_pow11;
  volatile int *cancel;  // host-mapped
  int *status;           // [0] steps done, [1] stop (0 run, 1 cancelled, 2 budget),
                         // [2] steps to run (set before each launch)
  const long long *budget_cycles;  // device: 0 = none (read at launch, so graphs see updates)
};

// pusher: the pusher every run uses, or -1 when they differ
int ensemble_max_blocks_per_sm(int pusher);
cudaError_t ensemble_launch(const EnsembleDev &E, int blocks, int pusher, cudaStream_t st);
// graph mode: injection of every bunch, and t += dt of every run (both from
// and into device memory)
cudaError_t ensemble_inject_all(const EnsembleDev &E, cudaStream_t st);
cudaError_t ensemble_advance(const EnsembleDev &E, cudaStream_t st);

// byte offsets of the radix sort's scratch (sort.cu)
struct SortLayout {
  long long nsub, m, nb;
  size_t keys_a, keys_b, idx_a, idx_b, H, bs, tmp, total;
};
// state bytes per particle that the gather stages (FP64: r, z, vr, vphi,
// vz, w; FP32: cell, fr, fz, ur, uphi, uz, w)
constexpr size_t SORT_STATE_F64 = 6 * 8, SORT_STATE_F32 = 7 * 4;
SortLayout sort_layout(long long n, size_t state_bytes);
int sort_species_f64(const GridDev &g, SpeciesDev &s, char *scratch, cudaStream_t st);
int sort_species_f32(const GridDev &g, SpeciesF32 &s, char *scratch, cudaStream_t st);

// host-side launchers (fields.cu, particles_f64.cu, particles_f32.cu, diag.cu)
void launch_to_f32(const double *src, float *dst, size_t n, cudaStream_t st);
// packs GridDev::q32 (at q, 6 * (nr-1) * (nz-1) entries) from e32/hh32
void launch_pack_quads(const GridDev &g, float4 *q, cudaStream_t st);
void launch_yee_h(const GridDev &g, cudaStream_t st);
void launch_yee_e(const GridDev &g, cudaStream_t st);
void launch_push_deposit_f64(const GridDev &g, const SpeciesDev &s, int pusher, int n_sm,
                             cudaStream_t st);
void launch_charge_density_f64(const GridDev &g, const SpeciesDev &s, double *rho,
                               cudaStream_t st);
int diag_blocks();
void launch_finalize(const double *partials, int nblocks, int nv, double *out, cudaStream_t st);
void launch_push_deposit_f32(const GridDev &g, const SpeciesF32 &s, int pusher, int n_sm,
                             int blocks_per_sm, cudaStream_t st);
void launch_push_deposit_f32_to(const GridDev &g, const SpeciesF32 &s, const SpeciesOut &o,
                                int pusher, int n_sm, int blocks_per_sm, cudaStream_t st);
// the step-graph forms of the injection: the schedule is evaluated on the
// device from *d_t (inject_window); grid sized for pis slots
void launch_bunch_inject_f32_dev(const SpeciesF32 &s, const double *d_t, double begin,
                                 double end, double dt, unsigned pis, double dl, double half_dz,
                                 double dz, int ncz, float uz, const double *inv_pow11,
                                 cudaStream_t st);
void launch_bunch_inject_dev(const SpeciesDev &s, const double *d_t, double begin, double end,
                             double dt, unsigned pis, double dl, double half_dz, double velocity,
                             const double *inv_pow11, cudaStream_t st);
// *d_t = v, and *d_t = *d_t + dt (t += dt, src/loadInitParam.cpp:586)
void launch_set_time(double *d_t, double v, cudaStream_t st);
void launch_advance_time(double *d_t, double dt, cudaStream_t st);
void launch_bunch_inject_f32(const SpeciesF32 &s, long long start, long long count, double dl,
                             double half_dz, double dz, int ncz, float uz,
                             const double *inv_pow11, cudaStream_t st);
void launch_charge_density_f32(const GridDev &g, const SpeciesF32 &s, double charge,
                               double *rho, cudaStream_t st);
void launch_cell_to_f64(const SpeciesF32 &s, double dr, double dz, int ncz, double *r, double *z,
                        double *vr, double *vphi, double *vz, double *w_out, cudaStream_t st);
void launch_f64_to_cell(const SpeciesF32 &s, const double *r, const double *z, const double *vr,
                        const double *vphi, const double *vz, const double *w_in, double dr,
                        double dz, int nr, int nz, unsigned *err, cudaStream_t st);
void launch_kinetic_f32(const SpeciesF32 &s, double mass, double *partials, double *out,
                        cudaStream_t st);
void launch_grid_diag(const GridDev &g, const double *rho, const double *rho0, double *partials,
                      double *out, cudaStream_t st);
void launch_rho_norm(const GridDev &g, const double *rho, double *partials, double *out,
                     cudaStream_t st);
void launch_kinetic_f64(const SpeciesDev &s, double *partials, double *out, cudaStream_t st);
void launch_bunch_inject(const SpeciesDev &s, long long start, long long count, double dl,
                         double half_dz, double velocity, const double *inv_pow11,
                         cudaStream_t st);

// Adjoint (adjoint.cu): FP64 adjoint grids of one context and the adjoint
// particle state of one FP32 species.
struct AdjGrids {
  double *lEr, *lEphi, *lEz;     // adjoint of E
  double *lHr, *lHphi, *lHz;     // adjoint of H
  double *lHhr, *lHhphi, *lHhz;  // adjoint of the half-step H of the current step
  float *lJr, *lJphi, *lJz;      // adjoint of the current step's J (read by the FP32
                                 // particle reverse only, so stored in FP32)
};

struct AdjSpeciesDev {
  SpeciesF32 st;  // stored input state of the particle phase of the step
  float *la, *lb, *lur, *luphi, *luz;  // adjoints of fr, fz, ur, uphi, uz
  double *lw;                          // adjoint of w (accumulated over steps)
};

// PoissonDirichlet (poisson.cu)
int poisson_check(int nz);
cudaError_t launch_poisson(const GridDev &g, const double *rho, double *t, double *fi,
                           double *alpha, double *beta, const double *b_mode, double *er,
                           double *ez, cudaStream_t st);

// upstream initial state (init.cu)
void launch_init_species(unsigned n, double r_size, double z_size, double dr, double dz,
                         double n1, double n2, double left, double temperature, double mass,
                         const double *inv_pow, double *r, double *z, double *vr, double *vphi,
                         double *vz, double *w, double *scratch_vol, double *d_sum, unsigned *err,
                         cudaStream_t st);
void init_inv_pow_table(double *host);
int init_inv_pow_count();

// TemperatureClassic and ParticlesDensity (species_diag.cu)
void launch_density_f64(const GridDev &g, const SpeciesDev &s, double *out, cudaStream_t st);
void launch_density_f32(const GridDev &g, const SpeciesF32 &s, double mass, double *out,
                        cudaStream_t st);
void launch_temperature_f64(const GridDev &g, const SpeciesDev &s, double *acc, cudaStream_t st);
void launch_temperature_f32(const GridDev &g, const SpeciesF32 &s, double *acc, cudaStream_t st);
void launch_temperature_normalize(const GridDev &g, const double *acc, double mass, double charge,
                                  double *t_out, cudaStream_t st);

// probes (probe.cu)
struct MpArrays {
  const double *src[5];  // r, z, v_r, v_phi, v_z of every slot
  double *dst[5];        // the selected slots, compacted in slot order
};
void launch_probe_gather(const double *f, int nz, int type, int r0, int z0, int r1, int z1,
                         long long n, double *out, cudaStream_t st);
long long mp_blocks(long long n);
void launch_mp_count(const double *r, const double *z, long long n, double dr, double dz, int r0,
                     int z0, int r1, int z1, unsigned *counts, cudaStream_t st);
void launch_mp_write(const MpArrays &arr, long long n, double dr, double dz, int r0, int z0,
                     int r1, int z1, const unsigned long long *offsets, cudaStream_t st);

void adj_launch_e(const GridDev &g, const AdjGrids &A, cudaStream_t st);
void adj_launch_h(const GridDev &g, const AdjGrids &A, cudaStream_t st);
// per cell: 1 when an adjoint of J within reach of its particles is nonzero
void adj_launch_active(const GridDev &g, const AdjGrids &A, uint8_t *active, cudaStream_t st);
// Q: the step's per-cell quads of E and the half-step H (GridDev::q32
// layout); active: adj_launch_active's flags of the step
void adj_launch_particles(const GridDev &g, const float4 *Q, const AdjSpeciesDev &S,
                          const AdjGrids &A, const uint8_t *active, int face, float face_h,
                          cudaStream_t st);
void adj_launch_inject(const AdjSpeciesDev &S, long long start, long long count, double dt,
                       double dz, double velocity, const double *inv_pow11, double *lv,
                       cudaStream_t st);
void adj_launch_seed(const GridDev &g, const AdjGrids &A, int r0, int r1, int z0, int z1,
                     double *loss, cudaStream_t st);

#ifdef __CUDACC__
// Bunch::bunch_inject's schedule at time t (src/bunch.cpp:87-124): the slots
// [start, start + count) injected in the step, from the host-computed window
// [begin, end) and particles per step.  The one operation done here,
// (t - begin) / dt * pis, is the host's (no contraction is possible), so the
// device schedule of a captured step equals the host's.
__device__ __forceinline__ bool inject_window(double t, double begin, double end, double dt,
                                              unsigned pis, unsigned number, long long &start,
                                              long long &count) {
  start = 0;
  count = 0;
  if (!(t >= begin && t < end) || pis == 0) return false;
  const int start_number = (t - begin) / dt * pis;
  start = (long long)(unsigned)start_number;
  count = pis;
  if (start >= (long long)number) count = 0;
  else if (start + count > (long long)number) count = (long long)number - start;
  return count > 0;
}

// L2 prefetch of [ptr, ptr + bytes) by the bulk-copy unit (bytes a multiple
// of 16; skipped unless ptr is 16-byte aligned).  A hint: nothing waits on
// it.  The particle kernels let one thread per CTA ask for the CTA's next
// chunk while its warps step the current one.
__device__ __forceinline__ void prefetch_l2(const void *ptr, unsigned bytes) {
  if ((reinterpret_cast<unsigned long long>(ptr) & 15ull) != 0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ptr), "r"(bytes) : "memory");
}
#endif

}  // namespace pdp3g
