/*
 * pdp3g: B200 (sm_100a) implementation of the PDP3 per-timestep
 * particle-in-cell loop, behind a plain C ABI.
 *
 * The upstream code has no plugin or FFI layer; its seam is a set of C++
 * classes driven by LoadInitParam::run (src/loadInitParam.cpp:471-587).
 * Each entry point below names the upstream interface it stands in for.
 * The library owns all device memory; host pointers are borrowed for the
 * duration of a call.  Calls on one context are not thread-safe; separate
 * contexts may be used from separate threads.  No entry point calls exit():
 * every failure is a status code (upstream: exit(1) / exit(78) / abort()).
 *
 * Units are SI with the upstream constants (include/constant.h:10-27).
 * Grids are [n_grid_r][n_grid_z] row-major doubles (upstream: double** rows,
 * src/field.cpp:10-25).  Particles are given as structure-of-arrays.
 */
#ifndef PDP3G_H
#define PDP3G_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PDP3G_OK = 0,
  PDP3G_INVALID_ARG = 1,
  PDP3G_CUDA_ERROR = 2,
  PDP3G_NAN_DETECTED = 3,   /* upstream: exit(1), src/particles.cpp:1046-1053 */
  PDP3G_V_GE_C = 4,         /* upstream: exit(1), src/lib.cpp:54-59 */
  PDP3G_OUT_OF_GRID = 5,    /* a particle reached a cell outside the grid */
  PDP3G_TIMEOUT = 6,
  PDP3G_NOT_SUPPORTED = 7,
  PDP3G_NO_MEMORY = 8
} pdp3g_status;

typedef enum {
  PDP3G_PUSHER_BORIS = 0,         /* relativistic Boris (PUSHER_BORIS_RELATIVISTIC; also
                                     what the default adaptive build computes at -O2) */
  PDP3G_PUSHER_VAY = 1,           /* PUSHER_VAY, src/particles.cpp:1152-1254 */
  PDP3G_PUSHER_BORIS_CLASSIC = 2  /* PUSHER_BORIS_CLASSIC */
} pdp3g_pusher;

typedef enum {
  PDP3G_FP64 = 0,       /* plain form: FP64 throughout, upstream operation order */
  PDP3G_FP32_CELL = 1   /* int cell + FP32 offset/momentum, FP64 grid accumulation */
} pdp3g_precision;

/* grid components (upstream public members, include/eField.h, hField.h, current.h) */
typedef enum {
  PDP3G_E_R = 0, PDP3G_E_PHI, PDP3G_E_Z,
  PDP3G_H_R, PDP3G_H_PHI, PDP3G_H_Z,
  PDP3G_H_R_HALF, PDP3G_H_PHI_HALF, PDP3G_H_Z_HALF,
  PDP3G_J_R, PDP3G_J_PHI, PDP3G_J_Z,
  PDP3G_SIGMA,
  PDP3G_NCOMP
} pdp3g_comp;

typedef struct {
  /* Geometry(r_size, z_size, n_grid_r, n_grid_z), src/geometry.cpp:8-31 */
  double r_size, z_size;
  int32_t n_grid_r, n_grid_z;
  /* Time(current_time, ..., delta_t), src/pdp3Time.cpp:11-18 */
  double dt, current_time;
  /* Geometry::set_pml(l1, l2, l3, sigma1, sigma2), src/geometry.cpp:56-107;
     applied only when one of l1..l3 is non-zero (src/parameters.cpp:244-245) */
  double pml_l1, pml_l2, pml_l3, pml_sigma1, pml_sigma2;
  int32_t pusher;       /* pdp3g_pusher */
  int32_t precision;    /* pdp3g_precision */
  int32_t device;       /* CUDA device ordinal (PDP3G_INVALID_ARG past the last one) */
  int32_t sort_interval;/* particles re-sorted by cell every N steps (0: never) */
} pdp3g_config;

/* FP64 reductions over the current state (no upstream counterpart; the
   upstream code prints no energy or residual diagnostics). */
typedef struct {
  double field_energy;      /* 1/2 sum (eps0 E^2 + mu0 H^2) dV over node volumes */
  double kinetic_energy;    /* sum m_i c^2 (gamma_i - 1) over alive particles */
  double gauss_residual;    /* ||eps0 div E - (rho - rho_0)||_2 over the nodes
                               2 <= i <= nr-3, 2 <= k <= nz-3 whose divergence
                               stencil is undamped: sigma == 0 at (i,k), (i-1,k)
                               and (i,k-1) (where the update conserves it) */
  double gauss_norm;        /* sqrt(sum over species ||rho_s||_2^2), same nodes:
                               the charge-density scale the residual is relative to */
  double charge_total;      /* sum rho dV */
  int64_t alive;            /* alive macroparticles */
} pdp3g_diag;

typedef struct {
  double ms_step_total;     /* device time of all launches, summed */
  double ms_particles;      /* push + deposition kernels */
  double ms_fields;         /* Yee H and E kernels */
  double ms_sort;           /* counting sort */
  double ms_other;          /* injection, clears */
  int64_t launches;         /* kernels launched since the last reset */
  int64_t particle_launches;
  int64_t steps;
  int64_t particle_steps;   /* alive macroparticles pushed, summed over steps */
} pdp3g_timing;

typedef struct pdp3g_ctx pdp3g_ctx;

/* Geometry + Time + EField/HField/Current construction and
   LoadInitParam::init_fields (src/loadInitParam.cpp:250-260): all grids 0. */
pdp3g_status pdp3g_create(const pdp3g_config *cfg, pdp3g_ctx **out);
void pdp3g_destroy(pdp3g_ctx *ctx);

/* Particles(name, charge_e, mass_me, n, geom) with its public pos/vel arrays
   filled (include/particles.h:34-100): charge_array = charge_e*e*w,
   mass_array = mass_me*m_e*w (src/particles.cpp:328-329).  alive may be NULL
   (all alive).  *id receives the species index (ParticlesList order). */
pdp3g_status pdp3g_add_species(pdp3g_ctx *ctx, double charge_e, double mass_me, int64_t n,
                               const double *r, const double *z, const double *vr,
                               const double *vphi, const double *vz, const double *w,
                               const uint8_t *alive, int32_t *id);
/* The same with the six FP64 arrays in device memory of the context's
   device (e.g. generated there), all particles alive.  The call first waits
   for all work on the device (the arrays may come from any stream) and has
   read the arrays when it returns.  No upstream counterpart (the upstream
   fills its host arrays in place). */
pdp3g_status pdp3g_add_species_device(pdp3g_ctx *ctx, double charge_e, double mass_me,
                                      int64_t n, const double *r, const double *z,
                                      const double *vr, const double *vphi, const double *vz,
                                      const double *w, int32_t *id);
/* LoadInitParam::init_particles for one species (src/loadInitParam.cpp:
   157-164): Particles(name, charge_e, mass_me, n, geom),
   load_cylindrical_spatial_distribution(left_density, right_density,
   left_plasma_boundary) (src/particles.cpp:278-331) and
   velocity_distribution(temperature) (src/particles.cpp:228-276, TESTMODE
   random_reverse sequences, Maxwell-Juttner sampler) generated on the device.
   Positions and weights equal the upstream's bit for bit; velocities agree to
   about 1e-13 relative (device log/exp/pow, sampler tables computed from
   their definition).  n < 2^30.  PDP3G_TIMEOUT if the sampler's rejection
   loop exceeds 100000 draws for a particle. */
pdp3g_status pdp3g_add_species_upstream(pdp3g_ctx *ctx, double charge_e, double mass_me,
                                        int64_t n, double left_density, double right_density,
                                        double left_plasma_boundary, double temperature,
                                        int32_t *id);

/* Bunch(name, charge, mass, n, geom, duration, radius, density, velocity,
   bunch_number, hole_duration), src/bunch.cpp:6-80 (TESTMODE radial
   sequence), injected progressively by Bunch::bunch_inject
   (src/bunch.cpp:87-124) at the start of each step. */
pdp3g_status pdp3g_add_bunch(pdp3g_ctx *ctx, double charge_e, double mass_me, int64_t n,
                             double duration, double radius, double density, double velocity,
                             int32_t bunch_number, double hole_duration, int32_t *id);

/* nsteps passes of the LoadInitParam::run loop body (src/loadInitParam.cpp:
   481-527, 586): bunch injection, HField::calc_field, Current::reset_j,
   ParticlesList::step_v + full_current_distribution, EField::calc_field,
   t += dt.  Asynchronous on the context's stream.  With timing off
   (pdp3g_set_timing) each step is one launch of a graph captured on the
   first call (the injection schedule and t += dt evaluated on the device,
   with the host's arithmetic), recaptured when species are added; re-sort
   steps and timed steps launch their kernels one by one.  The context's
   stream must not be under a caller's stream capture (the call then falls
   back to one-by-one launches). */
pdp3g_status pdp3g_step(pdp3g_ctx *ctx, int32_t nsteps);

/* The phases of pdp3g_step, one per upstream call of the loop body, for
   hosts that keep the upstream call sequence (asynchronous, context stream):
     pdp3g_inject        LoadInitParam::init_beam / Bunch::bunch_inject
                         (src/loadInitParam.cpp:481, src/bunch.cpp:87-124)
     pdp3g_calc_h        HField::calc_field (src/hField.cpp:93-157)
     pdp3g_reset_j       Current::reset_j (src/current.cpp:125-135)
     pdp3g_push_deposit  ParticlesList::step_v + full_current_distribution
                         (src/particlesList.cpp:20-24, 50-54), fused
     pdp3g_calc_e        EField::calc_field (src/eField.cpp:85-170)
     pdp3g_advance_time  t += dt (src/loadInitParam.cpp:586) */
pdp3g_status pdp3g_inject(pdp3g_ctx *ctx);
pdp3g_status pdp3g_calc_h(pdp3g_ctx *ctx);
pdp3g_status pdp3g_reset_j(pdp3g_ctx *ctx);
pdp3g_status pdp3g_push_deposit(pdp3g_ctx *ctx);
pdp3g_status pdp3g_calc_e(pdp3g_ctx *ctx);
pdp3g_status pdp3g_advance_time(pdp3g_ctx *ctx);
/* Time::current_time assignment (the upstream loop advances it directly,
   src/loadInitParam.cpp:586); the bunch injection schedule reads it. */
pdp3g_status pdp3g_set_time(pdp3g_ctx *ctx, double current_time);

/* Stable sort of every plasma species by cell index (an integer LSD radix
   sort of (cell, index) pairs; the permutation equals a stable sort of the
   cell keys).  No upstream counterpart: upstream particles stay in creation
   order.  Bunch species keep their slot order.  pdp3g_step also sorts
   before the particle phase of every step whose count since the context's
   creation is a multiple of cfg.sort_interval (timing resets do not change
   that count).  The first sort allocates the context's sort scratch, kept
   until pdp3g_destroy: for the largest plasma species, 16 B per particle
   for keys and indices plus a staging copy of its state (28 B per particle
   in the FP32 form, 48 B in the FP64 form). */
pdp3g_status pdp3g_sort(pdp3g_ctx *ctx);

/* Waits for the stream and reports device-side error flags. */
pdp3g_status pdp3g_sync(pdp3g_ctx *ctx);

/* EField/HField public arrays and Current::get_j_* (src/current.cpp:88-102):
   copies one component into host memory [n_grid_r*n_grid_z]. */
pdp3g_status pdp3g_get_field(pdp3g_ctx *ctx, int32_t comp, double *host_out);
pdp3g_status pdp3g_set_field(pdp3g_ctx *ctx, int32_t comp, const double *host_in);

/* Particles public state (pos[i][0], pos[i][2], vel[i][0..2], is_alive);
   any pointer may be NULL. */
pdp3g_status pdp3g_get_species(pdp3g_ctx *ctx, int32_t id, double *r, double *z, double *vr,
                               double *vphi, double *vz, double *w, uint8_t *alive);
/* The species' state out to host arrays and the next state in, in one call:
   the device->host and host->device copies run concurrently in chunks (both
   PCIe directions at once; use pinned host memory for the overlap).  out_*
   receive what pdp3g_get_species returns; in_* are then loaded as
   pdp3g_set_species loads them (with the same checks).  in may equal out: a
   chunk is read back in only after it was written out.  No counterpart in
   the upstream, whose particles live in host memory; it serves a host that
   keeps the authoritative particle state across steps.  alive arrays may be
   NULL (out: all 1 when the species has no alive flags). */
pdp3g_status pdp3g_exchange_species(pdp3g_ctx *ctx, int32_t id, double *out_r, double *out_z,
                                    double *out_vr, double *out_vphi, double *out_vz,
                                    uint8_t *out_alive, const double *in_r, const double *in_z,
                                    const double *in_vr, const double *in_vphi,
                                    const double *in_vz, const uint8_t *in_alive);
/* pdp3g_exchange_species for several species in one call, for a host that
   holds every species' state (ParticlesList::part_list, particlesList.h:9-26):
   the copies of all items run as one pipeline (species after species on
   each PCIe direction, with no gap at a species boundary) and the FP32
   form's conversions to and from the FP64 host layout run on a third stream
   beside them.  Each species at most once; returns when every copy is done.
   Same arrays, checks and in == out rule as pdp3g_exchange_species. */
typedef struct {
  int32_t id;
  double *out_r, *out_z, *out_vr, *out_vphi, *out_vz;
  uint8_t *out_alive;
  const double *in_r, *in_z, *in_vr, *in_vphi, *in_vz;
  const uint8_t *in_alive;
} pdp3g_exchange_item;
pdp3g_status pdp3g_exchange_all(pdp3g_ctx *ctx, const pdp3g_exchange_item *items,
                                int32_t n_items);
pdp3g_status pdp3g_set_species(pdp3g_ctx *ctx, int32_t id, const double *r, const double *z,
                               const double *vr, const double *vphi, const double *vz,
                               const uint8_t *alive);
int64_t pdp3g_species_size(pdp3g_ctx *ctx, int32_t id);

/* ParticlesList::charge_weighting / Particles::charge_weighting
   (src/particlesList.cpp:14-18, src/particles.cpp:101-226) of the species in
   species_mask (bit s = species s) into a fresh grid, copied to host. */
pdp3g_status pdp3g_charge_density(pdp3g_ctx *ctx, uint32_t species_mask, double *host_out);

/* Records rho_0 for the Gauss residual (call after adding species). */
pdp3g_status pdp3g_mark_initial_charge(pdp3g_ctx *ctx);
pdp3g_status pdp3g_diagnostics(pdp3g_ctx *ctx, pdp3g_diag *out);

/* ---- Probes (ProbePlain, src/probePlain.cpp:80-224; LoadInitParam::dump_data,
   src/loadInitParam.cpp:319-398).  pdp3g_probe_read copies one probe's values
   of a component, in the order ProbePlain::write prints them:
     type 0 frame  rows start_r..end_r-1, each start_z..end_z-1
     type 1 col    start_r..end_r-1 at start_z
     type 2 row    start_z..end_z-1 at start_r
     type 3 dot    (start_r, start_z)
   comp is a grid component (PDP3G_E_R .. PDP3G_SIGMA) or
   PDP3G_PROBE_RHO_BEAM (the charge weighting of every bunch, as dump_data's
   rho_beam).  *count receives the number of values (at most capacity).
   pdp3g_probe_particles is ProbePlain::mpwrite's selection (type 4): the
   slots of species id, in slot order, whose cell (CELL_NUMBER of r and z)
   lies in [start_r, end_r] x [start_z, end_z] (inclusive, as upstream),
   alive or not; positions and velocities in the upstream units.  When more
   than capacity match, *count receives the number needed and the call
   returns PDP3G_INVALID_ARG. */
#define PDP3G_PROBE_RHO_BEAM 100
#define PDP3G_PROBE_T 101        /* per species: pdp3g_probe_read_species */
#define PDP3G_PROBE_DENSITY 102  /* per species: pdp3g_probe_read_species */
pdp3g_status pdp3g_probe_read(pdp3g_ctx *ctx, int32_t comp, int32_t type, int32_t start_r,
                              int32_t start_z, int32_t end_r, int32_t end_z, double *host_out,
                              int64_t capacity, int64_t *count);
/* dump_data's per-species components (src/loadInitParam.cpp:369-390):
   comp PDP3G_PROBE_T: TemperatureClassic, src/temperatureClassic.cpp:57-159,
   in eV, empty cells NaN as upstream; comp PDP3G_PROBE_DENSITY:
   ParticlesDensity::calc_density, src/particlesDensity.cpp:45-257. */
pdp3g_status pdp3g_probe_read_species(pdp3g_ctx *ctx, int32_t comp, int32_t id, int32_t type,
                                      int32_t start_r, int32_t start_z, int32_t end_r,
                                      int32_t end_z, double *host_out, int64_t capacity,
                                      int64_t *count);
/* TemperatureClassic::calc_t + normalize of species id: [n_grid_r][n_grid_z]
   host grid, values for i < n_grid_r-1, k < n_grid_z-1 (the rest 0). */
pdp3g_status pdp3g_temperature(pdp3g_ctx *ctx, int32_t id, double *host_out);
/* ParticlesDensity::calc_density of species id: [n_grid_r][n_grid_z] host
   grid (mass_array / EL_MASS per m^3 over the four nodes of each particle). */
pdp3g_status pdp3g_density(pdp3g_ctx *ctx, int32_t id, double *host_out);

/* PoissonDirichlet::poisson_solve(EField*, ChargeDensity*)
   (src/poissonDirichlet.cpp:23-98): phi from rho by a sine transform along
   z, a radial sweep per mode and the inverse transform, then E_r (rows
   i < n_grid_r-1) and E_z (columns k < n_grid_z-1) from phi; the other E
   values are kept.  host_rho: [n_grid_r][n_grid_z] charge density, or NULL
   for the charge weighting of every species.  host_fi (optional) receives
   phi.  Needs 2 n_grid_z + 2 a power of two <= 8192 (the upstream's radix-2
   transform has the same restriction).  Not bit-identical: the transform's
   twiddle factors come from the device sin/cos (about 1e-13 relative). */
pdp3g_status pdp3g_poisson_solve(pdp3g_ctx *ctx, const double *host_rho, double *host_fi);
pdp3g_status pdp3g_probe_particles(pdp3g_ctx *ctx, int32_t id, int32_t start_r, int32_t start_z,
                                   int32_t end_r, int32_t end_z, double *r, double *z, double *vr,
                                   double *vphi, double *vz, int64_t capacity, int64_t *count);

/* Per-kernel device timing with CUDA events on the context's stream. */
pdp3g_status pdp3g_set_timing(pdp3g_ctx *ctx, int32_t enabled);
pdp3g_status pdp3g_get_timing(pdp3g_ctx *ctx, pdp3g_timing *out);
pdp3g_status pdp3g_reset_timing(pdp3g_ctx *ctx);

/* Allocation-free grid diagnostics, for callers that cannot allocate device
   memory (code running during CUDA graph capture, hosts whose caching
   allocator owns all device memory, embedders that forbid cudaMalloc after
   start-up).  No counterpart in the upstream code.
   Inputs are device pointers to [n_grid_r][n_grid_z] grids (rho0 may be
   NULL for a zero initial charge); out is a device pointer to 3 doubles:
   {field energy, Gauss residual, total charge}, defined as the same fields
   of pdp3g_diagnostics.  Work goes to `stream` (a cudaStream_t, NULL for the
   default stream) on the calling thread's current device.
   Scratch: a static 96 KiB device array (4096 chunks of 4096 nodes) that each
   GPU loading the library holds until exit; grids above 16,777,216 nodes are
   rejected with PDP3G_INVALID_ARG.  Every call shares that array and no
   entry needs clearing (each call overwrites the slots it reads), but calls
   that overlap on the GPU race on it: serialise them.  The first call on a
   device (and the first after the current context changes, e.g. after a
   cudaDeviceReset) looks up the array's device address; make that first
   call before any stream capture.  A CUDA error already pending on the
   calling thread is reported as PDP3G_CUDA_ERROR and left in place, and
   nothing is launched.  Calls no cudaMalloc/cudaFree. */
pdp3g_status pdp3g_field_diagnostics_noalloc(
    const double *e_r, const double *e_phi, const double *e_z, const double *h_r,
    const double *h_phi, const double *h_z, const double *rho, const double *rho0,
    const double *sigma, int32_t n_grid_r, int32_t n_grid_z, double r_size, double z_size,
    double *out, void *stream);

/* ---- Batched ensemble (no upstream counterpart: the upstream runs one
   simulation per process).  Independent runs, each a context created with
   precision PDP3G_FP32_CELL on the same device (different grids, species
   and bunches allowed), are advanced together by one persistent cooperative
   kernel per pdp3g_ensemble_run call, replayed from a captured CUDA graph
   (a direct cooperative launch if the capture is refused).  Each run's
   state stays in its context (pdp3g_get_field etc. work as usual).  The
   kernel checks a host-mapped cancel flag and a time budget once per step
   and returns PDP3G_TIMEOUT when either stops it; the steps done are
   reported by pdp3g_ensemble_info and added to every run's time.
   A second mode (PDP3G_ENS_STEP_GRAPH) replays one captured CUDA graph per
   step in which every run's own step kernels (those of pdp3g_step) sit on
   parallel branches, with the bunch injection and the time advance done on
   the device; its cancel flag and budget are checked between steps (at most
   eight steps in flight).  pdp3g_ensemble_autotune times both modes. */
typedef struct pdp3g_ensemble pdp3g_ensemble;
enum { PDP3G_ENS_PERSISTENT = 0, PDP3G_ENS_STEP_GRAPH = 1 };
typedef struct {
  int32_t runs, blocks_per_sm, blocks, used_graph;
  double last_ms;            /* device time of the last run call */
  int64_t last_steps_done;
  int64_t particles;         /* macroparticle slots over all runs */
  int32_t mode;              /* PDP3G_ENS_PERSISTENT or PDP3G_ENS_STEP_GRAPH */
  int32_t graph_blocks_per_sm; /* CTAs per SM of the runs' particle kernels in the
                                  step graph (0: each context's own) */
} pdp3g_ensemble_stats;
pdp3g_status pdp3g_ensemble_create(pdp3g_ctx *const *runs, int32_t n_runs, pdp3g_ensemble **out);
pdp3g_status pdp3g_ensemble_run(pdp3g_ensemble *e, int32_t nsteps);
/* times the persistent kernel at every feasible CTAs-per-SM count and the
   step graph with the runs' particle kernels at 2, 4 and 8 CTAs per SM,
   steps_per_trial steps each (the trial steps advance the runs), and keeps
   the fastest; *blocks_per_sm receives the persistent kernel's count, or 0
   when the step graph won (its count: pdp3g_ensemble_info) */
pdp3g_status pdp3g_ensemble_autotune(pdp3g_ensemble *e, int32_t steps_per_trial,
                                     int32_t *blocks_per_sm);
/* PDP3G_ENS_PERSISTENT (the default) or PDP3G_ENS_STEP_GRAPH */
pdp3g_status pdp3g_ensemble_set_mode(pdp3g_ensemble *e, int32_t mode);
pdp3g_status pdp3g_ensemble_set_budget(pdp3g_ensemble *e, double max_ms);  /* 0: none */
/* re-sort every run's plasma species by cell every `steps` steps (between
   persistent launches); default: the smallest positive sort_interval of the
   runs' configs; 0: never */
pdp3g_status pdp3g_ensemble_set_sort_interval(pdp3g_ensemble *e, int32_t steps);
pdp3g_status pdp3g_ensemble_cancel(pdp3g_ensemble *e, int32_t cancel);     /* any thread */
pdp3g_status pdp3g_ensemble_info(pdp3g_ensemble *e, pdp3g_ensemble_stats *out);
const char *pdp3g_ensemble_last_error(pdp3g_ensemble *e);
void pdp3g_ensemble_destroy(pdp3g_ensemble *e);

/* ---- Adjoint window (no upstream counterpart: the upstream has no
   derivatives).  A forward/backward vector-Jacobian pair over window_steps
   steps of a PDP3G_FP32_CELL context with the relativistic Boris pusher.
   Loss: sum over the probe nodes i in [probe_r0, probe_r1), k in
   [probe_z0, probe_z1) of E_z(i, k)^2 V_i after the window, with V_i the
   node's ring volume 2 pi i dr^2 dz (pi dr^2 dz / 4 on the axis).
   pdp3g_forward_window steps the context window_steps steps from its
   current state (no re-sorting, so every particle keeps its slot), storing
   E, H and the particle state every checkpoint_interval steps and at the
   end, and returns the loss; a second call starts a new window from where
   the first ended and replaces its checkpoints.
   pdp3g_backward_window recomputes each interval from its checkpoint
   (storing every step's particle-phase input) and runs the hand-written
   reverse of each step, last to first; it leaves the context in the state
   that the forward ended in.  The forward stores the particle-phase inputs
   of its last interval as it runs them, so the first backward after a
   forward recomputes every interval but the last (a second backward after
   the same forward recomputes them all).  Results, all with respect to the state at the
   start of the forward window: per particle dL/dr and dL/dz (per metre),
   dL/du for u = gamma v / c (r, phi, z) and dL/dw (weight); per grid node
   dL/dE and dL/dH; per bunch dL/dv for the beam velocity through the
   injected z offsets and u_z. */
typedef struct pdp3g_adjoint pdp3g_adjoint;
pdp3g_status pdp3g_adjoint_create(pdp3g_ctx *ctx, int32_t window_steps,
                                  int32_t checkpoint_interval, int32_t probe_r0,
                                  int32_t probe_r1, int32_t probe_z0, int32_t probe_z1,
                                  pdp3g_adjoint **out);
pdp3g_status pdp3g_forward_window(pdp3g_adjoint *a, double *loss);
pdp3g_status pdp3g_backward_window(pdp3g_adjoint *a);
/* any output pointer may be NULL */
pdp3g_status pdp3g_adjoint_species(pdp3g_adjoint *a, int32_t id, double *l_r, double *l_z,
                                   double *l_ur, double *l_uphi, double *l_uz, double *l_w);
/* comp in PDP3G_E_R .. PDP3G_H_Z */
pdp3g_status pdp3g_adjoint_field(pdp3g_adjoint *a, int32_t comp, double *host_out);
pdp3g_status pdp3g_adjoint_bunch_velocity(pdp3g_adjoint *a, int32_t id, double *l_v);
/* The upstream radial gather weights jump at cell faces (node-centred
   components) and cell middles (half-node components), and a wall
   reflection flips u_r or u_z of the particles whose end point lies beyond
   the wall, so the loss of a many-particle run moves with the particles'
   density at those jumps, which a per-particle (pathwise) derivative does
   not see.  PDP3G_ADJ_MEAN_FIELD (the default) adds each particle's expected
   share of the jump terms of PDP3G_ADJ_DEFAULT_JUMPS; PDP3G_ADJ_PATHWISE
   gives the exact derivative of the particles' piecewise-smooth
   trajectories. */
enum { PDP3G_ADJ_MEAN_FIELD = 0, PDP3G_ADJ_PATHWISE = 1 };
pdp3g_status pdp3g_adjoint_set_mode(pdp3g_adjoint *a, int32_t mode);
/* The mean-field terms one by one (a bit mask; 0 = pathwise):
   PDP3G_ADJ_GATHER_JUMPS  the gather weights' jumps, for a particle density
                           uniform inside each cell;
   PDP3G_ADJ_WALL_JUMPS    the momentum jumps of the wall reflections;
   PDP3G_ADJ_WALL_CELLS    the walls leave the axis cell's and the last
                           radial cell's particles in the half next to the
                           other cells (r >= dr/2, r <= r_max - dr/2), twice
                           as dense; without it those cells count as full.
                           Applies to the uniform jump density (face width
                           0): the box kernel counts the particles that are
                           there. */
enum { PDP3G_ADJ_GATHER_JUMPS = 1, PDP3G_ADJ_WALL_JUMPS = 2, PDP3G_ADJ_WALL_CELLS = 4,
       PDP3G_ADJ_DEFAULT_JUMPS = PDP3G_ADJ_GATHER_JUMPS };
pdp3g_status pdp3g_adjoint_set_jump_terms(pdp3g_adjoint *a, uint32_t terms);
/* The density the gather jump terms use: 0 takes it uniform inside each
   cell; half_width in (0, 0.5] (cells) estimates it at each jump from the
   particles within half_width of it (a box kernel), which follows densities
   that are not uniform inside a cell.  Default 1/8 cell. */
#define PDP3G_ADJ_DEFAULT_FACE_WIDTH 0.125
pdp3g_status pdp3g_adjoint_set_face_width(pdp3g_adjoint *a, double half_width);
/* device time of the last forward and backward calls */
pdp3g_status pdp3g_adjoint_timing(pdp3g_adjoint *a, double *forward_ms, double *backward_ms);
int64_t pdp3g_adjoint_bytes(pdp3g_adjoint *a);
void pdp3g_adjoint_destroy(pdp3g_adjoint *a);

/* The CUDA stream (cudaStream_t) every launch of this context goes to, so a
   caller can order its own work or CUDA events against the step. */
void *pdp3g_stream(pdp3g_ctx *ctx);

/* Time::current_time */
double pdp3g_current_time(pdp3g_ctx *ctx);
/* device memory held by the context, bytes */
int64_t pdp3g_device_bytes(pdp3g_ctx *ctx);
const char *pdp3g_status_string(pdp3g_status st);
const char *pdp3g_last_error(pdp3g_ctx *ctx);
/* 1 when a CUDA device is usable from this process */
int32_t pdp3g_device_available(void);

#ifdef __cplusplus
}
#endif
#endif
