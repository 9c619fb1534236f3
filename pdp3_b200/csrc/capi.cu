// C-ABI of the pdp3g library: context, device memory, the step sequence of
// LoadInitParam::run (src/loadInitParam.cpp:471-587) on one CUDA stream, and
// host <-> device copies for the upstream-style public state.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pdp3g.h"
#include "pdp3g_internal.cuh"

using namespace pdp3g;

namespace {

struct Species {
  SpeciesDev dev{};      // FP64 plain form
  SpeciesF32 f32{};      // FP32 cell-local form
  bool fp32 = false;
  bool is_bunch = false;
  double charge_si = 0, mass_si = 0;  // per unit weight
  // Bunch parameters (src/bunch.cpp:17-26)
  double duration = 0, radius = 0, density = 0, velocity = 0, hole_duration = 0;
  double bunch_number = 0;
};

struct StepEvents {
  cudaEvent_t ev[7];
};

}  // namespace

struct pdp3g_ctx {
  pdp3g_config cfg{};
  int device = 0;
  int n_sm = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t stream_up = nullptr;  // pdp3g_exchange_species' host->device copies
  // the particle phase steps species 1, 3, ... on stream_side beside the
  // others on stream (fork and join events on stream)
  cudaStream_t stream_side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_chunk = nullptr, ev_up = nullptr;
  // pdp3g_exchange_all: FP64 staging of every FP32 item, and 2 events per item
  double *d_xstage = nullptr;
  size_t xstage_n = 0;
  std::vector<cudaEvent_t> xev;
  double dr = 0, dz = 0, t = 0;
  double *grid_mem = nullptr;
  float *mirror = nullptr;       // FP32 contexts: E and half-step H in FP32 (6 grids)
  float4 *quads = nullptr;       // FP32 contexts: the same per cell (GridDev::q32)
  GridDev g{};
  unsigned *d_err = nullptr;
  double *d_inv_pow11 = nullptr;
  double *d_rho0 = nullptr;
  double *d_scratch = nullptr;   // one grid (charge density)
  double *d_scratch2 = nullptr;  // one grid (per-species charge density)
  double *d_temp_acc = nullptr;  // 5 grids: the temperature probe's sums
  double *d_poisson = nullptr;   // the Poisson solve's t, phi, alpha, beta grids + modes
  double *d_partials = nullptr;  // per-block reduction partials
  double *d_red = nullptr;       // reduction results
  char *d_sort = nullptr;        // radix-sort scratch
  double *d_stage = nullptr;     // FP64 staging for the cell-local layout's conversions
  size_t stage_n = 0;
  size_t sort_bytes = 0;
  int64_t sorts = 0;
  size_t scratch_bytes = 0;
  bool has_rho0 = false;
  std::vector<Species> species;
  // timing
  bool timing = false;
  std::vector<StepEvents> step_events;
  size_t events_used = 0;
  pdp3g_timing acc{};
  int64_t launches = 0, particle_launches = 0, steps = 0;  // since the last timing reset
  int64_t sim_steps = 0;  // steps since creation: the re-sort schedule (not reset by timing)
  std::string last_error;
  int64_t bytes = 0;
  int f32_blocks_per_sm = 0;  // CTAs per SM for the FP32 particle kernel (0: its default)
  // pdp3g_step without timing replays one captured graph per step; the graph
  // reads and advances the device copy of t.  Recaptured when the species or
  // the particle kernel's launch shape change.
  double *d_time = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  size_t graph_nsp = 0;
  int graph_bpsm = -1;
  int64_t graph_launches = 0, graph_particle_launches = 0;
  bool graph_off = false;  // a capture failed: eager steps from then on
};

namespace {

pdp3g_status fail(pdp3g_ctx *ctx, pdp3g_status st, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return st;
}

pdp3g_status cuda_fail(pdp3g_ctx *ctx, cudaError_t e, const char *where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  if (ctx) ctx->last_error = m;
  return e == cudaErrorMemoryAllocation ? PDP3G_NO_MEMORY : PDP3G_CUDA_ERROR;
}

#define CK(call)                                            \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
  } while (0)

template <typename T>
cudaError_t dalloc(pdp3g_ctx *ctx, T **p, size_t count) {
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (count ? count : 1));
  if (e == cudaSuccess) ctx->bytes += (int64_t)(sizeof(T) * count);
  return e;
}

// Geometry::set_pml, src/geometry.cpp:56-107, evaluated on the host in the
// upstream order so sigma is bit-identical.
void host_set_pml(std::vector<double> &sig, int nr, int nz, double dr, double dz, double r_size,
                  double z_size, double l1, double l2, double l3, double sigma1, double sigma2) {
  auto AT = [&](int i, int k) -> double & { return sig[(size_t)i * nz + k]; };
  double len_left = dz * (std::floor(nz * l1));
  double len_right = dz * (std::floor(nz * l2));
  double len_ext = dr * (std::floor(nr * l3));
  if ((l1 == 0) && (l2 == 0) && (l3 != 0)) {
    for (int i = 0; i < nr; i++)
      for (int k = 0; k < nz; k++)
        if (r_size - dr * i <= len_ext)
          AT(i, k) = sigma1 + (sigma2 - sigma1) / std::pow(len_ext, 2) *
                                  std::pow((dr * (i + 1) - r_size + len_ext), 2);
  } else {
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nr; i++) {
        if (dz * k < len_left)
          AT(i, k) = sigma1 + (sigma2 - sigma1) / std::pow(len_left, 2) *
                                  std::pow(len_left - dz * k, 2);
        if (z_size - dz * k < len_right)
          AT(i, k) = sigma1 + (sigma2 - sigma1) / std::pow(len_right, 2) *
                                  std::pow(dz * (k + 1) - z_size + len_right, 2);
      }
  }
  if (l3 != 0) {
    for (int i = 0; i < nr; i++)
      for (int k = 0; k < nz; k++)
        if (r_size - dr * i <= len_ext)
          if ((r_size - dr * (i + 1) < len_ext * dz * k / len_left) &&
              (r_size - dr * i <= len_ext / len_right * (z_size - dz * k)))
            AT(i, k) = sigma1 + (sigma2 - sigma1) / std::pow(len_ext, 2) *
                                    std::pow(dr * (i + 1) - r_size + len_ext, 2);
  }
}

double *comp_ptr(pdp3g_ctx *ctx, int comp) {
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  if (comp < 0 || comp >= PDP3G_NCOMP) return nullptr;
  return ctx->grid_mem + (size_t)comp * ng;
}

// keeps the FP32 copy of a gathered component (E, half-step H) equal to the
// FP64 grid after the grid was written outside the Yee updates
void refresh_mirror(pdp3g_ctx *ctx, int comp) {
  if (!ctx->mirror) return;
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  int slot = -1;
  if (comp >= PDP3G_E_R && comp <= PDP3G_E_Z) slot = comp - PDP3G_E_R;
  if (comp >= PDP3G_H_R_HALF && comp <= PDP3G_H_Z_HALF) slot = 3 + comp - PDP3G_H_R_HALF;
  if (slot < 0) return;
  launch_to_f32(comp_ptr(ctx, comp), ctx->mirror + (size_t)slot * ng, ng, ctx->stream);
}

// random_reverse(i, 9), src/math/rand.cpp:40-53 (host libm)
double random_reverse(double x, int power) {
  int int_vel = (int)std::floor(x);
  double ost = 0, r = 0;
  int order = 1;
  while (int_vel >= 1) {
    ost = int_vel % power;
    r = r + ost * std::pow((double)power, (-order));
    int_vel = (int_vel - ost) / power;
    order = order + 1;
  }
  return r;
}

StepEvents *next_events(pdp3g_ctx *ctx) {
  if (ctx->events_used == ctx->step_events.size()) {
    StepEvents se;
    for (auto &e : se.ev) cudaEventCreate(&e);
    ctx->step_events.push_back(se);
  }
  return &ctx->step_events[ctx->events_used++];
}

pdp3g_status harvest_timing(pdp3g_ctx *ctx) {
  if (ctx->events_used == 0) return PDP3G_OK;
  CK(cudaStreamSynchronize(ctx->stream));
  for (size_t s = 0; s < ctx->events_used; s++) {
    float ms[6];
    for (int j = 0; j < 6; j++)
      CK(cudaEventElapsedTime(&ms[j], ctx->step_events[s].ev[j], ctx->step_events[s].ev[j + 1]));
    // ev0..1 injection, 1..2 H update, 2..3 J clear, 3..4 re-sort, 4..5 particles,
    // 5..6 E update
    ctx->acc.ms_other += ms[0] + ms[2];
    ctx->acc.ms_fields += ms[1] + ms[5];
    ctx->acc.ms_sort += ms[3];
    ctx->acc.ms_particles += ms[4];
    ctx->acc.ms_step_total += ms[0] + ms[1] + ms[2] + ms[3] + ms[4] + ms[5];
  }
  ctx->events_used = 0;
  return PDP3G_OK;
}

}  // namespace

extern "C" {

const char *pdp3g_status_string(pdp3g_status st) {
  switch (st) {
    case PDP3G_OK: return "ok";
    case PDP3G_INVALID_ARG: return "invalid argument";
    case PDP3G_CUDA_ERROR: return "CUDA error";
    case PDP3G_NAN_DETECTED: return "particle position is NaN or Inf";
    case PDP3G_V_GE_C: return "particle velocity reached the speed of light";
    case PDP3G_OUT_OF_GRID: return "particle outside the grid";
    case PDP3G_TIMEOUT: return "timeout";
    case PDP3G_NOT_SUPPORTED: return "not supported";
    case PDP3G_NO_MEMORY: return "out of device memory";
  }
  return "unknown status";
}

const char *pdp3g_last_error(pdp3g_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int32_t pdp3g_device_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n > 0 ? 1 : 0;
}

pdp3g_status pdp3g_create(const pdp3g_config *cfg, pdp3g_ctx **out) {
  if (!cfg || !out) return PDP3G_INVALID_ARG;
  *out = nullptr;
  if (cfg->n_grid_r < 3 || cfg->n_grid_z < 3 || !(cfg->r_size > 0) || !(cfg->z_size > 0) ||
      !(cfg->dt > 0) || cfg->pusher < 0 || cfg->pusher > 2 ||
      (cfg->precision != PDP3G_FP64 && cfg->precision != PDP3G_FP32_CELL))
    return PDP3G_INVALID_ARG;
  // the FP32 form's int32 cell index and 32-bit node offsets
  if (cfg->precision == PDP3G_FP32_CELL &&
      (long long)cfg->n_grid_r * cfg->n_grid_z >= (1LL << 31))
    return PDP3G_INVALID_ARG;
  // an ordinal past the last device is the caller's error; checked first so
  // that no CUDA error is left pending on the calling thread
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
    cudaGetLastError();
    return PDP3G_CUDA_ERROR;
  }
  if (cfg->device < 0 || cfg->device >= ndev) return PDP3G_INVALID_ARG;
  pdp3g_ctx *ctx = new pdp3g_ctx();
  ctx->cfg = *cfg;
  ctx->device = cfg->device;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) {
    cudaGetLastError();  // this call's own error: not left for the caller's next check
    delete ctx;
    return PDP3G_CUDA_ERROR;
  }
  cudaDeviceGetAttribute(&ctx->n_sm, cudaDevAttrMultiProcessorCount, cfg->device);
  const int nr = cfg->n_grid_r, nz = cfg->n_grid_z;
  ctx->dr = cfg->r_size / (nr - 1);  // src/geometry.cpp:45-53
  ctx->dz = cfg->z_size / (nz - 1);
  ctx->t = cfg->current_time;
  size_t ng = (size_t)nr * nz;
  auto bail = [&](pdp3g_status s) {
    pdp3g_destroy(ctx);
    return s;
  };
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&ctx->stream_side, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming)) != cudaSuccess)
    return bail(PDP3G_CUDA_ERROR);
  if ((e = dalloc(ctx, &ctx->grid_mem, ng * PDP3G_NCOMP)) != cudaSuccess)
    return bail(e == cudaErrorMemoryAllocation ? PDP3G_NO_MEMORY : PDP3G_CUDA_ERROR);
  if ((e = cudaMemset(ctx->grid_mem, 0, sizeof(double) * ng * PDP3G_NCOMP)) != cudaSuccess)
    return bail(PDP3G_CUDA_ERROR);
  if ((e = dalloc(ctx, &ctx->d_err, 4)) != cudaSuccess) return bail(PDP3G_CUDA_ERROR);
  cudaMemset(ctx->d_err, 0, sizeof(unsigned) * 4);
  // pow(11, -o) for the injection sequence, from the host libm
  std::vector<double> inv11(48, 0.0);
  for (int o = 1; o < 48; o++) inv11[o] = std::pow((double)11, (-o));
  if ((e = dalloc(ctx, &ctx->d_inv_pow11, 48)) != cudaSuccess) return bail(PDP3G_CUDA_ERROR);
  cudaMemcpy(ctx->d_inv_pow11, inv11.data(), sizeof(double) * 48, cudaMemcpyHostToDevice);
  if (cfg->pml_l1 != 0 || cfg->pml_l2 != 0 || cfg->pml_l3 != 0) {
    std::vector<double> sig(ng, 0.0);
    host_set_pml(sig, nr, nz, ctx->dr, ctx->dz, cfg->r_size, cfg->z_size, cfg->pml_l1,
                 cfg->pml_l2, cfg->pml_l3, cfg->pml_sigma1, cfg->pml_sigma2);
    cudaMemcpy(ctx->grid_mem + (size_t)PDP3G_SIGMA * ng, sig.data(), sizeof(double) * ng,
               cudaMemcpyHostToDevice);
  }
  GridDev &g = ctx->g;
  g.nr = nr;
  g.nz = nz;
  g.r_size = cfg->r_size;
  g.z_size = cfg->z_size;
  g.dr = ctx->dr;
  g.dz = ctx->dz;
  g.dt = cfg->dt;
  g.er = comp_ptr(ctx, PDP3G_E_R);
  g.ephi = comp_ptr(ctx, PDP3G_E_PHI);
  g.ez = comp_ptr(ctx, PDP3G_E_Z);
  g.hr = comp_ptr(ctx, PDP3G_H_R);
  g.hphi = comp_ptr(ctx, PDP3G_H_PHI);
  g.hz = comp_ptr(ctx, PDP3G_H_Z);
  g.hrh = comp_ptr(ctx, PDP3G_H_R_HALF);
  g.hphih = comp_ptr(ctx, PDP3G_H_PHI_HALF);
  g.hzh = comp_ptr(ctx, PDP3G_H_Z_HALF);
  g.jr = comp_ptr(ctx, PDP3G_J_R);
  g.jphi = comp_ptr(ctx, PDP3G_J_PHI);
  g.jz = comp_ptr(ctx, PDP3G_J_Z);
  g.sigma = comp_ptr(ctx, PDP3G_SIGMA);
  g.err = ctx->d_err;
  if ((e = dalloc(ctx, &ctx->d_time, 1)) != cudaSuccess)
    return bail(e == cudaErrorMemoryAllocation ? PDP3G_NO_MEMORY : PDP3G_CUDA_ERROR);
  if (cfg->precision == PDP3G_FP32_CELL) {
    if ((e = dalloc(ctx, &ctx->mirror, 6 * ng)) != cudaSuccess)
      return bail(e == cudaErrorMemoryAllocation ? PDP3G_NO_MEMORY : PDP3G_CUDA_ERROR);
    if ((e = cudaMemset(ctx->mirror, 0, sizeof(float) * 6 * ng)) != cudaSuccess)
      return bail(PDP3G_CUDA_ERROR);
    g.e32 = ctx->mirror;
    g.hh32 = ctx->mirror + 3 * ng;
    const size_t ncells = (size_t)(cfg->n_grid_r - 1) * (cfg->n_grid_z - 1);
    if ((e = dalloc(ctx, &ctx->quads, 6 * ncells)) != cudaSuccess)
      return bail(e == cudaErrorMemoryAllocation ? PDP3G_NO_MEMORY : PDP3G_CUDA_ERROR);
    g.q32 = ctx->quads;
  }
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return bail(PDP3G_CUDA_ERROR);
  *out = ctx;
  return PDP3G_OK;
}

void pdp3g_destroy(pdp3g_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto &sp : ctx->species) {
    cudaFree(sp.dev.r);
    cudaFree(sp.dev.z);
    cudaFree(sp.dev.vr);
    cudaFree(sp.dev.vphi);
    cudaFree(sp.dev.vz);
    cudaFree((void *)sp.dev.w);
    cudaFree(sp.dev.alive);
    cudaFree(sp.f32.cell);
    cudaFree(sp.f32.fr);
    cudaFree(sp.f32.fz);
    cudaFree(sp.f32.ur);
    cudaFree(sp.f32.uphi);
    cudaFree(sp.f32.uz);
    cudaFree((void *)sp.f32.w);
    if (sp.f32.alive != sp.dev.alive) cudaFree(sp.f32.alive);
  }
  for (auto &se : ctx->step_events)
    for (auto &e : se.ev) cudaEventDestroy(e);
  cudaFree(ctx->grid_mem);
  if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
  cudaFree(ctx->d_time);
  cudaFree(ctx->mirror);
  cudaFree(ctx->quads);
  cudaFree(ctx->d_err);
  cudaFree(ctx->d_inv_pow11);
  cudaFree(ctx->d_rho0);
  cudaFree(ctx->d_scratch);
  cudaFree(ctx->d_scratch2);
  cudaFree(ctx->d_temp_acc);
  cudaFree(ctx->d_poisson);
  cudaFree(ctx->d_partials);
  cudaFree(ctx->d_red);
  cudaFree(ctx->d_sort);
  cudaFree(ctx->d_stage);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->stream_up) cudaStreamDestroy(ctx->stream_up);
  if (ctx->stream_side) cudaStreamDestroy(ctx->stream_side);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->ev_chunk) cudaEventDestroy(ctx->ev_chunk);
  if (ctx->ev_up) cudaEventDestroy(ctx->ev_up);
  for (cudaEvent_t e : ctx->xev) cudaEventDestroy(e);
  cudaFree(ctx->d_xstage);
  delete ctx;
}

static pdp3g_status alloc_species(pdp3g_ctx *ctx, Species &sp, int64_t n, bool with_alive) {
  CK(dalloc(ctx, &sp.dev.r, n));
  CK(dalloc(ctx, &sp.dev.z, n));
  CK(dalloc(ctx, &sp.dev.vr, n));
  CK(dalloc(ctx, &sp.dev.vphi, n));
  CK(dalloc(ctx, &sp.dev.vz, n));
  double *w = nullptr;
  CK(dalloc(ctx, &w, n));
  sp.dev.w = w;
  if (with_alive) CK(dalloc(ctx, &sp.dev.alive, n));
  sp.dev.n = n;
  return PDP3G_OK;
}

static void f32_constants(pdp3g_ctx *ctx, Species &sp) {
  const double dt = ctx->cfg.dt, dr = ctx->dr, dz = ctx->dz;
  const double q = sp.charge_si, m = sp.mass_si, c = LIGHT_SPEED;
  const double const1 = q * dt / (2 * m);
  SpeciesF32 &f = sp.f32;
  f.ke = (float)(const1 / c);
  f.kb = (float)(MAGN_CONST * const1);
  f.cr = (float)(c * dt / (2 * dr));
  f.cz = (float)(c * dt / (2 * dz));
  f.kphi = (float)(q * c / (2 * PI * dz * dr * dr));
  f.kz = (float)(q / (4 * PI * dr * dr * dt));
  f.kr = (float)(q / (2 * PI * dr * dz * dt));
  f.vay_e = (float)(2 * const1);
  f.vay_b = (float)(MAGN_CONST * const1 * 2 * const1 * const1);
  f.inv_c2 = (float)(1.0 / LIGHT_SPEED_POW_2);
}

static pdp3g_status stage_reserve(pdp3g_ctx *ctx, size_t n) {
  if (ctx->stage_n >= n) return PDP3G_OK;
  cudaFree(ctx->d_stage);
  ctx->d_stage = nullptr;
  ctx->stage_n = 0;
  CK(dalloc(ctx, &ctx->d_stage, 6 * n));
  ctx->stage_n = n;
  return PDP3G_OK;
}

// converts the FP64 arrays already in the staging buffer (r, z, vr, vphi, vz
// and, if with_w, w at slots 0..5) into the species' cell-local arrays
static pdp3g_status convert_staged_f32(pdp3g_ctx *ctx, Species &sp, bool with_w) {
  const size_t n = (size_t)sp.f32.n;
  double *S = ctx->d_stage;
  CK(cudaMemsetAsync(ctx->d_err + 1, 0, sizeof(unsigned), ctx->stream));
  launch_f64_to_cell(sp.f32, S, S + n, S + 2 * n, S + 3 * n, S + 4 * n, with_w ? S + 5 * n : nullptr,
                     ctx->dr, ctx->dz, ctx->cfg.n_grid_r, ctx->cfg.n_grid_z, ctx->d_err + 1,
                     ctx->stream);
  ctx->launches++;
  unsigned err = 0;
  CK(cudaMemcpyAsync(&err, ctx->d_err + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (err & ERR_NAN) return fail(ctx, PDP3G_NAN_DETECTED, "particle position is NaN or Inf");
  if (err & ERR_V_GE_C) return fail(ctx, PDP3G_V_GE_C, "velocity >= c");
  if (err & ERR_OUT_OF_GRID) return fail(ctx, PDP3G_OUT_OF_GRID, "particle outside the grid");
  return PDP3G_OK;
}

static pdp3g_status upload_f32(pdp3g_ctx *ctx, Species &sp, int64_t n, const double *r,
                               const double *z, const double *vr, const double *vphi,
                               const double *vz, const double *w) {
  pdp3g_status st = stage_reserve(ctx, (size_t)n);
  if (st != PDP3G_OK) return st;
  double *S = ctx->d_stage;
  const size_t b = sizeof(double) * (size_t)n;
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(S, r, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(S + n, z, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(S + 2 * n, vr, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(S + 3 * n, vphi, b, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(S + 4 * n, vz, b, cudaMemcpyHostToDevice, s));
  if (w) CK(cudaMemcpyAsync(S + 5 * n, w, b, cudaMemcpyHostToDevice, s));
  return convert_staged_f32(ctx, sp, w != nullptr);
}

pdp3g_status pdp3g_add_species(pdp3g_ctx *ctx, double charge_e, double mass_me, int64_t n,
                               const double *r, const double *z, const double *vr,
                               const double *vphi, const double *vz, const double *w,
                               const uint8_t *alive, int32_t *id) {
  if (!ctx || n < 0 || (n > 0 && (!r || !z || !vr || !vphi || !vz || !w)))
    return fail(ctx, PDP3G_INVALID_ARG, "add_species: null array");
  if (n > (int64_t)1 << 40) return fail(ctx, PDP3G_INVALID_ARG, "add_species: n too large");
  CK(cudaSetDevice(ctx->device));
  Species sp;
  sp.charge_si = charge_e * EL_CHARGE;  // src/particles.cpp:30-32
  sp.mass_si = mass_me * EL_MASS;
  if (ctx->cfg.precision == PDP3G_FP32_CELL) {
    sp.fp32 = true;
    SpeciesF32 &f = sp.f32;
    f.n = n;
    f.kind = KIND_PLASMA;
    f32_constants(ctx, sp);
    CK(dalloc(ctx, &f.cell, (size_t)n));
    CK(dalloc(ctx, &f.fr, (size_t)n));
    CK(dalloc(ctx, &f.fz, (size_t)n));
    CK(dalloc(ctx, &f.ur, (size_t)n));
    CK(dalloc(ctx, &f.uphi, (size_t)n));
    CK(dalloc(ctx, &f.uz, (size_t)n));
    float *wf = nullptr;
    CK(dalloc(ctx, &wf, (size_t)n));
    f.w = wf;
    pdp3g_status st = upload_f32(ctx, sp, n, r, z, vr, vphi, vz, w);
    if (st != PDP3G_OK) return st;
    if (alive) {
      CK(dalloc(ctx, &f.alive, (size_t)n));
      CK(cudaMemcpy(f.alive, alive, (size_t)n, cudaMemcpyHostToDevice));
    }
    ctx->species.push_back(sp);
    if (id) *id = (int32_t)ctx->species.size() - 1;
    return PDP3G_OK;
  }
  sp.dev.charge = sp.charge_si;
  sp.dev.mass = sp.mass_si;
  sp.dev.kind = KIND_PLASMA;
  pdp3g_status st = alloc_species(ctx, sp, n, alive != nullptr);
  if (st != PDP3G_OK) return st;
  size_t b = sizeof(double) * (size_t)n;
  CK(cudaMemcpy(sp.dev.r, r, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sp.dev.z, z, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sp.dev.vr, vr, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sp.dev.vphi, vphi, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sp.dev.vz, vz, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy((void *)sp.dev.w, w, b, cudaMemcpyHostToDevice));
  if (alive) CK(cudaMemcpy(sp.dev.alive, alive, (size_t)n, cudaMemcpyHostToDevice));
  ctx->species.push_back(sp);
  if (id) *id = (int32_t)ctx->species.size() - 1;
  return PDP3G_OK;
}

pdp3g_status pdp3g_add_species_device(pdp3g_ctx *ctx, double charge_e, double mass_me,
                                      int64_t n, const double *r, const double *z,
                                      const double *vr, const double *vphi, const double *vz,
                                      const double *w, int32_t *id) {
  if (!ctx || n <= 0 || !r || !z || !vr || !vphi || !vz || !w)
    return fail(ctx, PDP3G_INVALID_ARG, "add_species_device: null array");
  if (n > (int64_t)1 << 40) return fail(ctx, PDP3G_INVALID_ARG, "add_species_device: n too large");
  CK(cudaSetDevice(ctx->device));
  // the arrays may have been written on any stream of the device: wait for
  // all of it before reading them on the context's stream
  CK(cudaDeviceSynchronize());
  const double *src[6] = {r, z, vr, vphi, vz, w};
  for (const double *p : src) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
        at.device != ctx->device) {
      cudaGetLastError();
      return fail(ctx, PDP3G_INVALID_ARG,
                  "add_species_device: arrays must be device memory of the context's device");
    }
  }
  Species sp;
  sp.charge_si = charge_e * EL_CHARGE;  // src/particles.cpp:30-32
  sp.mass_si = mass_me * EL_MASS;
  cudaStream_t st = ctx->stream;
  const size_t b = sizeof(double) * (size_t)n;
  if (ctx->cfg.precision == PDP3G_FP32_CELL) {
    sp.fp32 = true;
    SpeciesF32 &f = sp.f32;
    f.n = n;
    f.kind = KIND_PLASMA;
    f32_constants(ctx, sp);
    CK(dalloc(ctx, &f.cell, (size_t)n));
    CK(dalloc(ctx, &f.fr, (size_t)n));
    CK(dalloc(ctx, &f.fz, (size_t)n));
    CK(dalloc(ctx, &f.ur, (size_t)n));
    CK(dalloc(ctx, &f.uphi, (size_t)n));
    CK(dalloc(ctx, &f.uz, (size_t)n));
    float *wf = nullptr;
    CK(dalloc(ctx, &wf, (size_t)n));
    f.w = wf;
    pdp3g_status rs = stage_reserve(ctx, (size_t)n);
    if (rs != PDP3G_OK) return rs;
    for (int j = 0; j < 6; j++)
      CK(cudaMemcpyAsync(ctx->d_stage + (size_t)j * n, src[j], b, cudaMemcpyDeviceToDevice, st));
    pdp3g_status cs = convert_staged_f32(ctx, sp, true);
    if (cs != PDP3G_OK) return cs;
  } else {
    sp.dev.charge = sp.charge_si;
    sp.dev.mass = sp.mass_si;
    sp.dev.kind = KIND_PLASMA;
    pdp3g_status as = alloc_species(ctx, sp, n, false);
    if (as != PDP3G_OK) return as;
    double *dst[6] = {sp.dev.r, sp.dev.z, sp.dev.vr, sp.dev.vphi, sp.dev.vz, (double *)sp.dev.w};
    for (int j = 0; j < 6; j++)
      CK(cudaMemcpyAsync(dst[j], src[j], b, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
  }
  ctx->species.push_back(sp);
  if (id) *id = (int32_t)ctx->species.size() - 1;
  return PDP3G_OK;
}

// LoadInitParam::init_particles for one species (src/loadInitParam.cpp:
// 157-164): the upstream's own initial state generated on the device
// (init.cu), then added as pdp3g_add_species_device adds device arrays.
pdp3g_status pdp3g_add_species_upstream(pdp3g_ctx *ctx, double charge_e, double mass_me,
                                        int64_t n, double left_density, double right_density,
                                        double left_plasma_boundary, double temperature,
                                        int32_t *id) {
  if (!ctx || n <= 0) return fail(ctx, PDP3G_INVALID_ARG, "add_species_upstream: n <= 0");
  // random_reverse takes (int) of npoints + i: the upstream's sequences are
  // defined for 2 n < 2^31
  if (n >= ((int64_t)1 << 30))
    return fail(ctx, PDP3G_INVALID_ARG, "add_species_upstream: n must be below 2^30");
  if (!(temperature >= 0))
    return fail(ctx, PDP3G_INVALID_ARG, "add_species_upstream: temperature must be >= 0");
  CK(cudaSetDevice(ctx->device));
  const size_t nn = (size_t)n;
  double *buf = nullptr, *inv_pow = nullptr;
  unsigned *err = nullptr;
  std::vector<double> tab((size_t)init_inv_pow_count());
  init_inv_pow_table(tab.data());
  cudaStream_t st = ctx->stream;
  pdp3g_status rs = PDP3G_OK;
  cudaError_t e = cudaMalloc((void **)&buf, sizeof(double) * (7 * nn + 1));
  if (e == cudaSuccess) e = cudaMalloc((void **)&inv_pow, sizeof(double) * tab.size());
  if (e == cudaSuccess) e = cudaMalloc((void **)&err, sizeof(unsigned));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(inv_pow, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(unsigned), st);
  unsigned herr = 0;
  if (e == cudaSuccess) {
    double *r = buf, *z = buf + nn, *vr = buf + 2 * nn, *vp = buf + 3 * nn, *vz = buf + 4 * nn;
    double *w = buf + 5 * nn, *vol = buf + 6 * nn, *sum = buf + 7 * nn;
    launch_init_species((unsigned)n, ctx->cfg.r_size, ctx->cfg.z_size, ctx->dr, ctx->dz,
                        left_density, right_density, left_plasma_boundary, temperature,
                        mass_me * EL_MASS, inv_pow, r, z, vr, vp, vz, w, vol, sum, err, st);
    ctx->launches += 4;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess && herr)
      rs = fail(ctx, PDP3G_TIMEOUT, "add_species_upstream: velocity sampler did not accept");
    if (e == cudaSuccess && rs == PDP3G_OK)
      rs = pdp3g_add_species_device(ctx, charge_e, mass_me, n, r, z, vr, vp, vz, w, id);
    cudaStreamSynchronize(st);  // the copies out of buf have finished
  }
  cudaFree(buf);
  cudaFree(inv_pow);
  cudaFree(err);
  if (e != cudaSuccess) return fail(ctx, PDP3G_CUDA_ERROR, cudaGetErrorString(e));
  return rs;
}

pdp3g_status pdp3g_add_bunch(pdp3g_ctx *ctx, double charge_e, double mass_me, int64_t n,
                             double duration, double radius, double density, double velocity,
                             int32_t bunch_number, double hole_duration, int32_t *id) {
  if (!ctx || n <= 0 || n > INT32_MAX || !(duration > 0) || !(velocity > 0))
    return fail(ctx, PDP3G_INVALID_ARG, "add_bunch: bad parameters");
  CK(cudaSetDevice(ctx->device));
  // Bunch::Bunch, src/bunch.cpp:6-80 (TESTMODE radial sequence)
  const double dr = ctx->dr, dz = ctx->dz;
  const double PI_ = pdp3g::PI;
  std::vector<double> r(n), z(n, 0.0), zero(n, 0.0), w(n);
  std::vector<uint8_t> alive(n, 0);
  double b_lenght = duration * velocity;
  double v_total = 0.;
  double N_total = PI_ * std::pow(radius, 2) * b_lenght * density;
  for (unsigned int i = 0; i < (unsigned int)n; i++) {
    double rand_r = random_reverse(i, 9);
    r[i] = (radius - dr) * rand_r + dr / 2;
    if (r[i] > dr)
      v_total += 2 * PI_ * r[i] * dr * dz;
    else
      v_total += PI_ * r[i] * r[i] * dz;
  }
  double v_avg = v_total / (unsigned int)n;
  double n_per_macro_avg = N_total / (unsigned int)n;
  for (int64_t i = 0; i < n; i++) {
    double norm;
    if (r[i] > dr / 2)
      norm = 2 * PI_ * r[i] * dr * dz / v_avg;
    else
      norm = PI_ * (r[i] * r[i] + r[i] * dr + dr * dr / 4) * dz / v_avg;
    w[i] = n_per_macro_avg * norm;
  }
  int32_t sid = -1;
  pdp3g_status st = pdp3g_add_species(ctx, charge_e, mass_me, n, r.data(), z.data(),
                                      zero.data(), zero.data(), zero.data(), w.data(),
                                      alive.data(), &sid);
  if (st != PDP3G_OK) return st;
  Species &sp = ctx->species[sid];
  sp.is_bunch = true;
  sp.dev.kind = KIND_BUNCH;
  sp.f32.kind = KIND_BUNCH;
  sp.duration = duration;
  sp.radius = radius;
  sp.density = density;
  sp.velocity = velocity;
  sp.hole_duration = hole_duration;
  sp.bunch_number = bunch_number;
  if (id) *id = sid;
  return PDP3G_OK;
}

int64_t pdp3g_species_size(pdp3g_ctx *ctx, int32_t id) {
  if (!ctx || id < 0 || id >= (int32_t)ctx->species.size()) return -1;
  const Species &sp = ctx->species[id];
  return sp.fp32 ? sp.f32.n : sp.dev.n;
}

// stable sort of every plasma species by cell (bunch species keep their
// slot order, which the injection schedule indexes)
static pdp3g_status sort_all(pdp3g_ctx *ctx) {
  long long nmax = 0;
  size_t need = 0;
  for (auto &sp : ctx->species) {
    if (sp.is_bunch) continue;
    const long long n = sp.fp32 ? sp.f32.n : sp.dev.n;
    nmax = std::max<long long>(nmax, n);
    need = std::max(need, sort_layout(n, sp.fp32 ? SORT_STATE_F32 : SORT_STATE_F64).total);
  }
  if (nmax <= 1) return PDP3G_OK;
  if (ctx->sort_bytes < need) {
    cudaFree(ctx->d_sort);
    ctx->d_sort = nullptr;
    ctx->sort_bytes = 0;
    CK(dalloc(ctx, &ctx->d_sort, need));
    ctx->sort_bytes = need;
  }
  for (auto &sp : ctx->species) {
    if (sp.is_bunch) continue;
    int nl = sp.fp32 ? sort_species_f32(ctx->g, sp.f32, ctx->d_sort, ctx->stream)
                     : sort_species_f64(ctx->g, sp.dev, ctx->d_sort, ctx->stream);
    ctx->launches += nl;
  }
  ctx->sorts++;
  CK(cudaGetLastError());
  return PDP3G_OK;
}

pdp3g_status pdp3g_sort(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  return sort_all(ctx);
}

// ---- the step's phases (LoadInitParam::run, src/loadInitParam.cpp:481-527, 586)

// the window of a bunch's injection (src/bunch.cpp:87-124): slots are
// injected while begin <= t < end, particles_in_step of them per step; one
// computation for the host schedule below and the device one of a captured
// step (phase_inject_dev)
static void inject_window_of(const pdp3g_ctx *ctx, const Species &sp, double &begin, double &end,
                             unsigned int &number, unsigned int &particles_in_step) {
  const double dt = ctx->cfg.dt;
  begin = sp.duration * sp.bunch_number + sp.hole_duration * sp.bunch_number;
  end = begin + sp.duration;
  const int steps_amount = (int)std::ceil(sp.duration / dt);
  number = (unsigned int)(sp.fp32 ? sp.f32.n : sp.dev.n);
  particles_in_step = steps_amount > 0 ? number / steps_amount : 0;
}

// Bunch::bunch_inject's schedule (src/bunch.cpp:87-124): the slots
// [start, start + count) that the bunch injects at time t (count 0: none)
static void inject_range(const pdp3g_ctx *ctx, const Species &sp, double t, long long &start,
                         long long &count) {
  start = 0;
  count = 0;
  const double dt = ctx->cfg.dt;
  double begin, end;
  unsigned int number, particles_in_step;
  inject_window_of(ctx, sp, begin, end, number, particles_in_step);
  int start_number = (t - begin) / dt * particles_in_step;
  if (t >= begin && t < end && particles_in_step > 0) {
    // indices start_number + i for i < particles_in_step, kept below number
    start = (long long)(unsigned int)start_number;
    count = particles_in_step;
    if (start >= (long long)number) count = 0;
    else if (start + count > (long long)number) count = (long long)number - start;
  }
}

// Bunch::bunch_inject of one FP32 bunch into the arrays of `view` (the
// species' own arrays, or a stored state of it)
static void inject_f32(pdp3g_ctx *ctx, const Species &sp, const SpeciesF32 &view) {
  long long start, count;
  inject_range(ctx, sp, ctx->t, start, count);
  if (count <= 0) return;
  const double dl = sp.velocity * ctx->cfg.dt;
  const double gv =
      sp.velocity / (LIGHT_SPEED * std::sqrt(1.0 - sp.velocity * sp.velocity / LIGHT_SPEED_POW_2));
  launch_bunch_inject_f32(view, start, count, dl, ctx->dz / 2.0, ctx->dz, ctx->cfg.n_grid_z - 1,
                          (float)gv, ctx->d_inv_pow11, ctx->stream);
  ctx->launches++;
}

// Bunch::bunch_inject for every bunch (src/bunch.cpp:87-124)
static void phase_inject(pdp3g_ctx *ctx) {
  cudaStream_t st = ctx->stream;
  for (auto &sp : ctx->species) {
    if (!sp.is_bunch) continue;
    if (sp.fp32) {
      inject_f32(ctx, sp, sp.f32);
      continue;
    }
    long long start, count;
    inject_range(ctx, sp, ctx->t, start, count);
    if (count > 0) {
      const double dl = sp.velocity * ctx->cfg.dt;
      launch_bunch_inject(sp.dev, start, count, dl, ctx->dz / 2.0, sp.velocity,
                          ctx->d_inv_pow11, st);
      ctx->launches++;
    }
  }
}

// HField::calc_field (src/hField.cpp:93-157)
static void phase_calc_h(pdp3g_ctx *ctx) {
  launch_yee_h(ctx->g, ctx->stream);
  ctx->launches++;
}

// Current::reset_j (src/current.cpp:125-135)
static cudaError_t phase_reset_j(pdp3g_ctx *ctx) {
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  return cudaMemsetAsync(ctx->g.jr, 0, sizeof(double) * ng * 3, ctx->stream);
}

// Species fork/join: with two or more species, every second species runs on
// the context's side stream between these two (the species only share
// atomic sums into the grids).
static cudaError_t species_fork(pdp3g_ctx *ctx) {
  if (ctx->species.size() < 2) return cudaSuccess;
  cudaError_t e = cudaEventRecord(ctx->ev_fork, ctx->stream);
  return e != cudaSuccess ? e : cudaStreamWaitEvent(ctx->stream_side, ctx->ev_fork, 0);
}
static cudaError_t species_join(pdp3g_ctx *ctx) {
  if (ctx->species.size() < 2) return cudaSuccess;
  cudaError_t e = cudaEventRecord(ctx->ev_join, ctx->stream_side);
  return e != cudaSuccess ? e : cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0);
}
static cudaStream_t species_stream(const pdp3g_ctx *ctx, size_t j) {
  return ctx->species.size() >= 2 && (j & 1) ? ctx->stream_side : ctx->stream;
}

// ParticlesList::step_v + full_current_distribution (src/particlesList.cpp:20-54).
// Species are independent apart from their sums into J (atomics), so with
// two or more species every second one runs on the side stream: the last,
// partial round of CTAs of one species' kernel overlaps the next kernel.
// The fork and join are checked: if the join's wait failed, the phases
// after this one would no longer be ordered after the side stream's J sums.
// the per-cell FP32 quads of E and the half-step H from their node copies,
// before every FP32 particle phase (the Yee updates, set_field and the
// checkpoint restores write the node copies)
static void pack_quads(pdp3g_ctx *ctx) {
  if (!ctx->quads) return;
  launch_pack_quads(ctx->g, ctx->quads, ctx->stream);
  ctx->launches++;
}

static cudaError_t phase_particles(pdp3g_ctx *ctx) {
  const bool fork = ctx->species.size() >= 2;
  cudaError_t e;
  pack_quads(ctx);
  if (fork) {
    if ((e = cudaEventRecord(ctx->ev_fork, ctx->stream)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ctx->stream_side, ctx->ev_fork, 0)) != cudaSuccess) return e;
  }
  for (size_t j = 0; j < ctx->species.size(); j++) {
    Species &sp = ctx->species[j];
    cudaStream_t st = fork && (j & 1) ? ctx->stream_side : ctx->stream;
    if (sp.fp32)
      launch_push_deposit_f32(ctx->g, sp.f32, ctx->cfg.pusher, ctx->n_sm, ctx->f32_blocks_per_sm,
                              st);
    else
      launch_push_deposit_f64(ctx->g, sp.dev, ctx->cfg.pusher, ctx->n_sm, st);
    ctx->launches++;
    ctx->particle_launches++;
  }
  if (fork) {
    if ((e = cudaEventRecord(ctx->ev_join, ctx->stream_side)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

// EField::calc_field (src/eField.cpp:85-170)
static void phase_calc_e(pdp3g_ctx *ctx) {
  launch_yee_e(ctx->g, ctx->stream);
  ctx->launches++;
}

// t += dt (src/loadInitParam.cpp:586)
static void phase_advance(pdp3g_ctx *ctx) {
  ctx->t = ctx->t + ctx->cfg.dt;
  ctx->steps++;
  ctx->sim_steps++;
}

// Bunch::bunch_inject of every bunch with the schedule evaluated on the
// device from the device copy of t (the form a captured step uses); the
// window constants are computed here as inject_range computes them.
static void phase_inject_dev(pdp3g_ctx *ctx) {
  const double dt = ctx->cfg.dt;
  for (auto &sp : ctx->species) {
    if (!sp.is_bunch) continue;
    double begin, end;
    unsigned number, pis;
    inject_window_of(ctx, sp, begin, end, number, pis);
    const double dl = sp.velocity * dt;
    if (sp.fp32) {
      const double b2 = sp.velocity * sp.velocity / LIGHT_SPEED_POW_2;
      const double gv = sp.velocity / (LIGHT_SPEED * std::sqrt(1.0 - b2));
      launch_bunch_inject_f32_dev(sp.f32, ctx->d_time, begin, end, dt, pis, dl, ctx->dz / 2.0,
                                  ctx->dz, ctx->cfg.n_grid_z - 1, (float)gv, ctx->d_inv_pow11,
                                  ctx->stream);
    } else {
      launch_bunch_inject_dev(sp.dev, ctx->d_time, begin, end, dt, pis, dl, ctx->dz / 2.0,
                              sp.velocity, ctx->d_inv_pow11, ctx->stream);
    }
    if (pis > 0) ctx->launches++;
  }
}

// One step of LoadInitParam::run's loop body, launched one kernel at a time
// (the timing path, re-sort steps, and the fallback of a failed capture).
static pdp3g_status step_eager(pdp3g_ctx *ctx) {
  cudaStream_t st = ctx->stream;
  StepEvents *ev = ctx->timing ? next_events(ctx) : nullptr;
  if (ev) cudaEventRecord(ev->ev[0], st);
  phase_inject(ctx);
  if (ev) cudaEventRecord(ev->ev[1], st);
  phase_calc_h(ctx);
  if (ev) cudaEventRecord(ev->ev[2], st);
  CK(phase_reset_j(ctx));
  if (ev) cudaEventRecord(ev->ev[3], st);
  if (ctx->cfg.sort_interval > 0 && ctx->sim_steps % ctx->cfg.sort_interval == 0) {
    pdp3g_status ss = sort_all(ctx);
    if (ss != PDP3G_OK) return ss;
  }
  if (ev) cudaEventRecord(ev->ev[4], st);
  CK(phase_particles(ctx));
  if (ev) cudaEventRecord(ev->ev[5], st);
  phase_calc_e(ctx);
  if (ev) cudaEventRecord(ev->ev[6], st);
  phase_advance(ctx);
  if (ctx->timing && ctx->events_used >= 4096) {
    pdp3g_status hs = harvest_timing(ctx);
    if (hs != PDP3G_OK) return hs;
  }
  return PDP3G_OK;
}

// Captures one step (injection from the device time, H, J clear, particles,
// E, t += dt on the device) as a graph.  False when the capture or the
// instantiation failed (nothing is left pending: the caller steps eagerly).
static bool capture_step(pdp3g_ctx *ctx) {
  if (ctx->step_exec) cudaGraphExecDestroy(ctx->step_exec);
  ctx->step_exec = nullptr;
  const int64_t l0 = ctx->launches, p0 = ctx->particle_launches;
  cudaStream_t st = ctx->stream;
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  phase_inject_dev(ctx);
  phase_calc_h(ctx);
  cudaError_t e = phase_reset_j(ctx);
  if (e == cudaSuccess) e = phase_particles(ctx);
  if (e == cudaSuccess) {
    phase_calc_e(ctx);
    launch_advance_time(ctx->d_time, ctx->cfg.dt, st);
    ctx->launches++;
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(st, &graph);
  ctx->graph_launches = ctx->launches - l0;
  ctx->graph_particle_launches = ctx->particle_launches - p0;
  ctx->launches = l0;
  ctx->particle_launches = p0;
  bool ok = e == cudaSuccess && ee == cudaSuccess && graph != nullptr &&
            cudaGraphInstantiate(&ctx->step_exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    ctx->step_exec = nullptr;
    cudaGetLastError();
    return false;
  }
  ctx->graph_nsp = ctx->species.size();
  ctx->graph_bpsm = ctx->f32_blocks_per_sm;
  return true;
}

pdp3g_status pdp3g_step(pdp3g_ctx *ctx, int32_t nsteps) {
  if (!ctx || nsteps < 0) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  // without timing: one graph launch per step (the launches of a step are
  // too short on small grids for the host to keep the GPU busy one by one)
  bool graph = !ctx->timing && !ctx->graph_off && nsteps > 0;
  if (graph && (!ctx->step_exec || ctx->graph_nsp != ctx->species.size() ||
                ctx->graph_bpsm != ctx->f32_blocks_per_sm)) {
    if (!capture_step(ctx)) {
      ctx->graph_off = true;
      graph = false;
    }
  }
  if (graph) {
    launch_set_time(ctx->d_time, ctx->t, st);
    ctx->launches++;
  }
  for (int s = 0; s < nsteps; s++) {
    const bool sort_step =
        ctx->cfg.sort_interval > 0 && ctx->sim_steps % ctx->cfg.sort_interval == 0;
    if (!graph || sort_step) {
      pdp3g_status es = step_eager(ctx);
      if (es != PDP3G_OK) return es;
      if (graph) {
        launch_set_time(ctx->d_time, ctx->t, st);  // the eager step advanced the host's t
        ctx->launches++;
      }
      continue;
    }
    CK(cudaGraphLaunch(ctx->step_exec, st));
    ctx->t = ctx->t + ctx->cfg.dt;  // the device did the same addition
    ctx->steps++;
    ctx->sim_steps++;
    ctx->launches += ctx->graph_launches;
    ctx->particle_launches += ctx->graph_particle_launches;
  }
  CK(cudaGetLastError());
  return PDP3G_OK;
}

pdp3g_status pdp3g_inject(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  phase_inject(ctx);
  CK(cudaGetLastError());
  return PDP3G_OK;
}

pdp3g_status pdp3g_calc_h(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  phase_calc_h(ctx);
  CK(cudaGetLastError());
  return PDP3G_OK;
}

pdp3g_status pdp3g_reset_j(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(phase_reset_j(ctx));
  return PDP3G_OK;
}

pdp3g_status pdp3g_push_deposit(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(phase_particles(ctx));
  return PDP3G_OK;
}

pdp3g_status pdp3g_calc_e(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  phase_calc_e(ctx);
  CK(cudaGetLastError());
  return PDP3G_OK;
}

pdp3g_status pdp3g_set_time(pdp3g_ctx *ctx, double current_time) {
  if (!ctx || !std::isfinite(current_time)) return PDP3G_INVALID_ARG;
  ctx->t = current_time;
  return PDP3G_OK;
}

pdp3g_status pdp3g_advance_time(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  phase_advance(ctx);
  return PDP3G_OK;
}

pdp3g_status pdp3g_sync(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  CK(cudaStreamSynchronize(ctx->stream));
  unsigned err = 0;
  CK(cudaMemcpy(&err, ctx->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (err & ERR_NAN) return fail(ctx, PDP3G_NAN_DETECTED, "particle position is NaN or Inf");
  if (err & ERR_V_GE_C) return fail(ctx, PDP3G_V_GE_C, "velocity >= c in get_gamma");
  if (err & ERR_OUT_OF_GRID) return fail(ctx, PDP3G_OUT_OF_GRID, "particle outside the grid");
  return PDP3G_OK;
}

pdp3g_status pdp3g_get_field(pdp3g_ctx *ctx, int32_t comp, double *host_out) {
  if (!ctx || !host_out || comp < 0 || comp >= PDP3G_NCOMP) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemcpyAsync(host_out, comp_ptr(ctx, comp), sizeof(double) * ng, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PDP3G_OK;
}

pdp3g_status pdp3g_set_field(pdp3g_ctx *ctx, int32_t comp, const double *host_in) {
  if (!ctx || !host_in || comp < 0 || comp >= PDP3G_NCOMP) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemcpyAsync(comp_ptr(ctx, comp), host_in, sizeof(double) * ng, cudaMemcpyHostToDevice,
                     ctx->stream));
  refresh_mirror(ctx, comp);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  return PDP3G_OK;
}

pdp3g_status pdp3g_get_species(pdp3g_ctx *ctx, int32_t id, double *r, double *z, double *vr,
                               double *vphi, double *vz, double *w, uint8_t *alive) {
  if (!ctx || id < 0 || id >= (int32_t)ctx->species.size()) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const Species &sp = ctx->species[id];
  if (sp.fp32) {
    const SpeciesF32 &f = sp.f32;
    const size_t n = (size_t)f.n;
    pdp3g_status rs = stage_reserve(ctx, n);
    if (rs != PDP3G_OK) return rs;
    double *S = ctx->d_stage;
    launch_cell_to_f64(f, ctx->dr, ctx->dz, ctx->cfg.n_grid_z - 1, S, S + n, S + 2 * n, S + 3 * n,
                       S + 4 * n, w ? S + 5 * n : nullptr, st);
    ctx->launches++;
    const size_t b = sizeof(double) * n;
    double *outs[6] = {r, z, vr, vphi, vz, w};
    for (int j = 0; j < 6; j++)
      if (outs[j]) CK(cudaMemcpyAsync(outs[j], S + j * n, b, cudaMemcpyDeviceToHost, st));
    if (alive) {
      if (f.alive)
        CK(cudaMemcpyAsync(alive, f.alive, n, cudaMemcpyDeviceToHost, st));
      else
        memset(alive, 1, n);
    }
    CK(cudaStreamSynchronize(st));
    return PDP3G_OK;
  }
  const SpeciesDev &d = sp.dev;
  size_t b = sizeof(double) * (size_t)d.n;
  if (r) CK(cudaMemcpyAsync(r, d.r, b, cudaMemcpyDeviceToHost, st));
  if (z) CK(cudaMemcpyAsync(z, d.z, b, cudaMemcpyDeviceToHost, st));
  if (vr) CK(cudaMemcpyAsync(vr, d.vr, b, cudaMemcpyDeviceToHost, st));
  if (vphi) CK(cudaMemcpyAsync(vphi, d.vphi, b, cudaMemcpyDeviceToHost, st));
  if (vz) CK(cudaMemcpyAsync(vz, d.vz, b, cudaMemcpyDeviceToHost, st));
  if (w) CK(cudaMemcpyAsync(w, d.w, b, cudaMemcpyDeviceToHost, st));
  if (alive) {
    if (d.alive)
      CK(cudaMemcpyAsync(alive, d.alive, (size_t)d.n, cudaMemcpyDeviceToHost, st));
    else
      memset(alive, 1, (size_t)d.n);
  }
  CK(cudaStreamSynchronize(st));
  return PDP3G_OK;
}

// pdp3g_exchange_species: the species' state out to host arrays and the
// next state in, pipelined by chunks of EXCHANGE_CHUNK particles: chunk c's
// device->host copies run on the context's stream, its host->device copies
// on a second stream once chunk c has left, so both PCIe directions work at
// once.  The host->device copy of a chunk overwrites the device staging (or,
// in the FP64 form, the state arrays) only after that chunk was copied out,
// which also makes in == out a correct round trip.
constexpr size_t EXCHANGE_CHUNK = (size_t)1 << 20;

pdp3g_status pdp3g_exchange_species(pdp3g_ctx *ctx, int32_t id, double *out_r, double *out_z,
                                    double *out_vr, double *out_vphi, double *out_vz,
                                    uint8_t *out_alive, const double *in_r, const double *in_z,
                                    const double *in_vr, const double *in_vphi,
                                    const double *in_vz, const uint8_t *in_alive) {
  if (!ctx || id < 0 || id >= (int32_t)ctx->species.size()) return PDP3G_INVALID_ARG;
  double *outs[5] = {out_r, out_z, out_vr, out_vphi, out_vz};
  const double *ins[5] = {in_r, in_z, in_vr, in_vphi, in_vz};
  for (int j = 0; j < 5; j++)
    if (!outs[j] || !ins[j]) return fail(ctx, PDP3G_INVALID_ARG, "exchange_species: null array");
  CK(cudaSetDevice(ctx->device));
  if (!ctx->stream_up) {
    CK(cudaStreamCreateWithFlags(&ctx->stream_up, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->ev_chunk, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->ev_up, cudaEventDisableTiming));
  }
  Species &sp = ctx->species[id];
  cudaStream_t down = ctx->stream, up = ctx->stream_up;
  const size_t n = (size_t)(sp.fp32 ? sp.f32.n : sp.dev.n);
  double *dev[5];
  uint8_t *dev_alive = sp.fp32 ? sp.f32.alive : sp.dev.alive;
  if (sp.fp32) {
    pdp3g_status rs = stage_reserve(ctx, n);
    if (rs != PDP3G_OK) return rs;
    double *S = ctx->d_stage;
    launch_cell_to_f64(sp.f32, ctx->dr, ctx->dz, ctx->cfg.n_grid_z - 1, S, S + n, S + 2 * n,
                       S + 3 * n, S + 4 * n, nullptr, down);
    ctx->launches++;
    for (int j = 0; j < 5; j++) dev[j] = S + j * n;
  } else {
    SpeciesDev &d = sp.dev;
    double *a[5] = {d.r, d.z, d.vr, d.vphi, d.vz};
    for (int j = 0; j < 5; j++) dev[j] = a[j];
  }
  // the upload stream starts after everything queued on the context's stream
  CK(cudaEventRecord(ctx->ev_up, down));
  CK(cudaStreamWaitEvent(up, ctx->ev_up, 0));
  for (size_t c0 = 0; c0 < n; c0 += EXCHANGE_CHUNK) {
    const size_t cn = std::min(EXCHANGE_CHUNK, n - c0), b = sizeof(double) * cn;
    for (int j = 0; j < 5; j++)
      CK(cudaMemcpyAsync(outs[j] + c0, dev[j] + c0, b, cudaMemcpyDeviceToHost, down));
    if (dev_alive && out_alive)
      CK(cudaMemcpyAsync(out_alive + c0, dev_alive + c0, cn, cudaMemcpyDeviceToHost, down));
    CK(cudaEventRecord(ctx->ev_chunk, down));
    CK(cudaStreamWaitEvent(up, ctx->ev_chunk, 0));
    for (int j = 0; j < 5; j++)
      CK(cudaMemcpyAsync(dev[j] + c0, ins[j] + c0, b, cudaMemcpyHostToDevice, up));
    if (dev_alive && in_alive)
      CK(cudaMemcpyAsync(dev_alive + c0, in_alive + c0, cn, cudaMemcpyHostToDevice, up));
  }
  CK(cudaEventRecord(ctx->ev_up, up));
  CK(cudaStreamWaitEvent(down, ctx->ev_up, 0));
  if (sp.fp32) {
    pdp3g_status rs = convert_staged_f32(ctx, sp, false);  // synchronises the stream
    if (rs != PDP3G_OK) return rs;
  } else {
    CK(cudaStreamSynchronize(down));
  }
  if (!dev_alive && out_alive) memset(out_alive, 1, n);
  return PDP3G_OK;
}

// pdp3g_exchange_all: one pipeline over the items.  Streams: the context's
// stream (down) carries every device->host copy, item after item; stream_up
// every host->device copy, chunk c of an item after that chunk went out;
// stream_side the FP32 items' conversions, to the FP64 layout before their
// copies out (side by side with the previous items' copies) and back after
// their copies in.  Each FP32 item has its own FP64 staging, so no item
// waits for another's conversion.
pdp3g_status pdp3g_exchange_all(pdp3g_ctx *ctx, const pdp3g_exchange_item *items,
                                int32_t n_items) {
  if (!ctx || n_items < 0 || (n_items > 0 && !items)) return PDP3G_INVALID_ARG;
  const int nsp = (int)ctx->species.size();
  std::vector<char> seen(nsp, 0);
  size_t stage_total = 0;
  for (int j = 0; j < n_items; j++) {
    const pdp3g_exchange_item &it = items[j];
    if (it.id < 0 || it.id >= nsp || seen[it.id])
      return fail(ctx, PDP3G_INVALID_ARG, "exchange_all: unknown or repeated species id");
    seen[it.id] = 1;
    const void *arr[10] = {it.out_r, it.out_z, it.out_vr, it.out_vphi, it.out_vz,
                           it.in_r,  it.in_z,  it.in_vr,  it.in_vphi,  it.in_vz};
    for (const void *a : arr)
      if (!a) return fail(ctx, PDP3G_INVALID_ARG, "exchange_all: null array");
    const Species &sp = ctx->species[it.id];
    if (sp.fp32) stage_total += 5 * (size_t)sp.f32.n;
  }
  if (n_items == 0) return PDP3G_OK;
  CK(cudaSetDevice(ctx->device));
  if (!ctx->stream_up) {
    CK(cudaStreamCreateWithFlags(&ctx->stream_up, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->ev_chunk, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->ev_up, cudaEventDisableTiming));
  }
  while (ctx->xev.size() < 2 * (size_t)n_items + 2) {
    cudaEvent_t e;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->xev.push_back(e);
  }
  if (ctx->xstage_n < stage_total) {
    cudaFree(ctx->d_xstage);
    ctx->d_xstage = nullptr;
    ctx->xstage_n = 0;
    CK(dalloc(ctx, &ctx->d_xstage, stage_total));
    ctx->xstage_n = stage_total;
  }
  cudaStream_t down = ctx->stream, up = ctx->stream_up, side = ctx->stream_side;
  cudaEvent_t *ev_conv = ctx->xev.data(), *ev_in = ctx->xev.data() + n_items;
  cudaEvent_t ev_begin = ctx->xev[2 * n_items], ev_side_end = ctx->xev[2 * n_items + 1];
  // everything already queued on the context's stream first
  CK(cudaEventRecord(ev_begin, down));
  CK(cudaStreamWaitEvent(up, ev_begin, 0));
  CK(cudaStreamWaitEvent(side, ev_begin, 0));
  CK(cudaMemsetAsync(ctx->d_err + 1, 0, sizeof(unsigned), side));
  const int ncz = ctx->cfg.n_grid_z - 1;
  std::vector<double *> stage(n_items, nullptr);
  size_t off = 0;
  for (int j = 0; j < n_items; j++) {
    Species &sp = ctx->species[items[j].id];
    if (!sp.fp32) continue;
    const size_t n = (size_t)sp.f32.n;
    double *S = ctx->d_xstage + off;
    off += 5 * n;
    stage[j] = S;
    launch_cell_to_f64(sp.f32, ctx->dr, ctx->dz, ncz, S, S + n, S + 2 * n, S + 3 * n, S + 4 * n,
                       nullptr, side);
    ctx->launches++;
    CK(cudaEventRecord(ev_conv[j], side));
  }
  for (int j = 0; j < n_items; j++) {
    const pdp3g_exchange_item &it = items[j];
    Species &sp = ctx->species[it.id];
    const size_t n = (size_t)(sp.fp32 ? sp.f32.n : sp.dev.n);
    double *outs[5] = {it.out_r, it.out_z, it.out_vr, it.out_vphi, it.out_vz};
    const double *ins[5] = {it.in_r, it.in_z, it.in_vr, it.in_vphi, it.in_vz};
    double *dev[5];
    uint8_t *dev_alive = sp.fp32 ? sp.f32.alive : sp.dev.alive;
    if (sp.fp32) {
      for (int k = 0; k < 5; k++) dev[k] = stage[j] + k * n;
      CK(cudaStreamWaitEvent(down, ev_conv[j], 0));
    } else {
      double *a[5] = {sp.dev.r, sp.dev.z, sp.dev.vr, sp.dev.vphi, sp.dev.vz};
      for (int k = 0; k < 5; k++) dev[k] = a[k];
    }
    // five arrays at one stride on both sides (the device side only in the
    // FP32 form, whose staging is one allocation; the host arrays when they
    // are one block): one 2-D copy of 5 rows per chunk and direction
    // instead of five copies.  A 2-D copy the runtime refuses (host arrays
    // equally spaced but not one allocation) falls back to five copies.
    const auto strided = [](const void *const p[5], ptrdiff_t &pitch) {
      pitch = (const char *)p[1] - (const char *)p[0];
      if (pitch <= 0 || pitch >= ((ptrdiff_t)1 << 30)) return false;  // 2-D copy pitch limit
      for (int k = 2; k < 5; k++)
        if ((const char *)p[k] - (const char *)p[k - 1] != pitch) return false;
      return true;
    };
    ptrdiff_t p_dev = 0, p_out = 0, p_in = 0;
    const void *pd[5] = {dev[0], dev[1], dev[2], dev[3], dev[4]};
    const void *po[5] = {outs[0], outs[1], outs[2], outs[3], outs[4]};
    const void *pi[5] = {ins[0], ins[1], ins[2], ins[3], ins[4]};
    bool rows_out = sp.fp32 && strided(pd, p_dev) && strided(po, p_out);
    bool rows_in = sp.fp32 && strided(pd, p_dev) && strided(pi, p_in);
    for (size_t c0 = 0; c0 < n; c0 += EXCHANGE_CHUNK) {
      const size_t cn = std::min(EXCHANGE_CHUNK, n - c0), b = sizeof(double) * cn;
      if (rows_out && cudaMemcpy2DAsync(outs[0] + c0, (size_t)p_out, dev[0] + c0,
                                        (size_t)p_dev, b, 5, cudaMemcpyDeviceToHost,
                                        down) != cudaSuccess) {
        cudaGetLastError();  // refused before anything was queued
        rows_out = false;
      }
      if (!rows_out) {
        for (int k = 0; k < 5; k++)
          CK(cudaMemcpyAsync(outs[k] + c0, dev[k] + c0, b, cudaMemcpyDeviceToHost, down));
      }
      if (dev_alive && it.out_alive)
        CK(cudaMemcpyAsync(it.out_alive + c0, dev_alive + c0, cn, cudaMemcpyDeviceToHost, down));
      CK(cudaEventRecord(ctx->ev_chunk, down));
      CK(cudaStreamWaitEvent(up, ctx->ev_chunk, 0));
      if (rows_in && cudaMemcpy2DAsync(dev[0] + c0, (size_t)p_dev, ins[0] + c0, (size_t)p_in,
                                       b, 5, cudaMemcpyHostToDevice, up) != cudaSuccess) {
        cudaGetLastError();
        rows_in = false;
      }
      if (!rows_in) {
        for (int k = 0; k < 5; k++)
          CK(cudaMemcpyAsync(dev[k] + c0, ins[k] + c0, b, cudaMemcpyHostToDevice, up));
      }
      if (dev_alive && it.in_alive)
        CK(cudaMemcpyAsync(dev_alive + c0, it.in_alive + c0, cn, cudaMemcpyHostToDevice, up));
    }
    CK(cudaEventRecord(ev_in[j], up));
    if (sp.fp32) {
      CK(cudaStreamWaitEvent(side, ev_in[j], 0));
      launch_f64_to_cell(sp.f32, stage[j], stage[j] + n, stage[j] + 2 * n, stage[j] + 3 * n,
                         stage[j] + 4 * n, nullptr, ctx->dr, ctx->dz, ctx->cfg.n_grid_r,
                         ctx->cfg.n_grid_z, ctx->d_err + 1, side);
      ctx->launches++;
    }
  }
  // the context's stream continues after the last copy in and conversion
  CK(cudaEventRecord(ev_side_end, side));
  CK(cudaEventRecord(ctx->ev_up, up));
  CK(cudaStreamWaitEvent(down, ev_side_end, 0));
  CK(cudaStreamWaitEvent(down, ctx->ev_up, 0));
  unsigned err = 0;
  CK(cudaMemcpyAsync(&err, ctx->d_err + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, down));
  CK(cudaStreamSynchronize(down));
  for (int j = 0; j < n_items; j++) {
    const Species &sp = ctx->species[items[j].id];
    const uint8_t *dev_alive = sp.fp32 ? sp.f32.alive : sp.dev.alive;
    if (!dev_alive && items[j].out_alive)
      memset(items[j].out_alive, 1, (size_t)(sp.fp32 ? sp.f32.n : sp.dev.n));
  }
  if (err & ERR_NAN) return fail(ctx, PDP3G_NAN_DETECTED, "particle position is NaN or Inf");
  if (err & ERR_V_GE_C) return fail(ctx, PDP3G_V_GE_C, "velocity >= c");
  if (err & ERR_OUT_OF_GRID) return fail(ctx, PDP3G_OUT_OF_GRID, "particle outside the grid");
  return PDP3G_OK;
}

pdp3g_status pdp3g_set_species(pdp3g_ctx *ctx, int32_t id, const double *r, const double *z,
                               const double *vr, const double *vphi, const double *vz,
                               const uint8_t *alive) {
  if (!ctx || id < 0 || id >= (int32_t)ctx->species.size()) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  Species &sp = ctx->species[id];
  if (sp.fp32) {
    // the cell index packs r and z: rebuild the full FP64 state on the
    // device, replace the given arrays and convert back
    const size_t n = (size_t)sp.f32.n;
    pdp3g_status rs = stage_reserve(ctx, n);
    if (rs != PDP3G_OK) return rs;
    double *S = ctx->d_stage;
    cudaStream_t st = ctx->stream;
    const double *ins[5] = {r, z, vr, vphi, vz};
    if (!(r && z && vr && vphi && vz)) {
      launch_cell_to_f64(sp.f32, ctx->dr, ctx->dz, ctx->cfg.n_grid_z - 1, S, S + n, S + 2 * n,
                         S + 3 * n, S + 4 * n, nullptr, st);
      ctx->launches++;
    }
    for (int j = 0; j < 5; j++)
      if (ins[j]) CK(cudaMemcpyAsync(S + j * n, ins[j], sizeof(double) * n, cudaMemcpyHostToDevice, st));
    if (r || z || vr || vphi || vz) {
      rs = convert_staged_f32(ctx, sp, false);
      if (rs != PDP3G_OK) return rs;
    }
    if (alive) {
      if (!sp.f32.alive) CK(dalloc(ctx, &sp.f32.alive, n));
      CK(cudaMemcpyAsync(sp.f32.alive, alive, n, cudaMemcpyHostToDevice, st));
      CK(cudaStreamSynchronize(st));
    }
    return PDP3G_OK;
  }
  SpeciesDev &d = sp.dev;
  size_t b = sizeof(double) * (size_t)d.n;
  cudaStream_t st = ctx->stream;
  if (alive && !d.alive) {
    CK(dalloc(ctx, &d.alive, (size_t)d.n));
  }
  if (r) CK(cudaMemcpyAsync(d.r, r, b, cudaMemcpyHostToDevice, st));
  if (z) CK(cudaMemcpyAsync(d.z, z, b, cudaMemcpyHostToDevice, st));
  if (vr) CK(cudaMemcpyAsync(d.vr, vr, b, cudaMemcpyHostToDevice, st));
  if (vphi) CK(cudaMemcpyAsync(d.vphi, vphi, b, cudaMemcpyHostToDevice, st));
  if (vz) CK(cudaMemcpyAsync(d.vz, vz, b, cudaMemcpyHostToDevice, st));
  if (alive) CK(cudaMemcpyAsync(d.alive, alive, (size_t)d.n, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return PDP3G_OK;
}

static pdp3g_status ensure_scratch(pdp3g_ctx *ctx) {
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  if (ctx->d_scratch) return PDP3G_OK;
  CK(dalloc(ctx, &ctx->d_scratch, ng));
  CK(dalloc(ctx, &ctx->d_scratch2, ng));
  CK(dalloc(ctx, &ctx->d_partials, (size_t)diag_blocks() * 4));
  CK(dalloc(ctx, &ctx->d_red, 16));
  ctx->scratch_bytes = ng * sizeof(double);
  return PDP3G_OK;
}

// charge weighting of the species in mask into dst (device grid)
static pdp3g_status rho_into(pdp3g_ctx *ctx, uint32_t mask, double *dst) {
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemsetAsync(dst, 0, ng * sizeof(double), ctx->stream));
  for (size_t s = 0; s < ctx->species.size() && s < 32; s++)
    if (mask & (1u << s)) {
      const Species &sp = ctx->species[s];
      if (sp.fp32)
        launch_charge_density_f32(ctx->g, sp.f32, sp.charge_si, dst, ctx->stream);
      else
        launch_charge_density_f64(ctx->g, sp.dev, dst, ctx->stream);
      ctx->launches++;
    }
  return PDP3G_OK;
}

pdp3g_status pdp3g_charge_density(pdp3g_ctx *ctx, uint32_t mask, double *host_out) {
  if (!ctx || !host_out) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  pdp3g_status st = ensure_scratch(ctx);
  if (st != PDP3G_OK) return st;
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  if ((st = rho_into(ctx, mask, ctx->d_scratch)) != PDP3G_OK) return st;
  CK(cudaMemcpyAsync(host_out, ctx->d_scratch, ng * sizeof(double), cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PDP3G_OK;
}

// number of values of a probe region (0: outside the grid)
static long long probe_count(const pdp3g_ctx *ctx, int type, int r0, int z0, int r1, int z1) {
  const int nr = ctx->cfg.n_grid_r, nz = ctx->cfg.n_grid_z;
  switch (type) {
    case 0:
      return (0 <= r0 && r0 < r1 && r1 <= nr && 0 <= z0 && z0 < z1 && z1 <= nz)
                 ? (long long)(r1 - r0) * (z1 - z0) : 0;
    case 1:
      return (0 <= r0 && r0 < r1 && r1 <= nr && 0 <= z0 && z0 < nz) ? r1 - r0 : 0;
    case 2:
      return (0 <= r0 && r0 < nr && 0 <= z0 && z0 < z1 && z1 <= nz) ? z1 - z0 : 0;
    case 3:
      return (0 <= r0 && r0 < nr && 0 <= z0 && z0 < nz) ? 1 : 0;
  }
  return 0;
}

// gathers a probe region of the device grid src into host_out
static pdp3g_status probe_to_host(pdp3g_ctx *ctx, const double *src, int type, int r0, int z0,
                                  int r1, int z1, long long n, double *host_out, int64_t *count) {
  launch_probe_gather(src, ctx->cfg.n_grid_z, type, r0, z0, r1, z1, n, ctx->d_scratch,
                      ctx->stream);
  ctx->launches++;
  CK(cudaMemcpyAsync(host_out, ctx->d_scratch, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (count) *count = n;
  return PDP3G_OK;
}

// TemperatureClassic::calc_t + normalize of species id into dst (device grid)
static pdp3g_status temperature_into(pdp3g_ctx *ctx, int id, double *dst) {
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  if (!ctx->d_temp_acc) CK(dalloc(ctx, &ctx->d_temp_acc, 5 * ng));
  CK(cudaMemsetAsync(ctx->d_temp_acc, 0, sizeof(double) * 5 * ng, ctx->stream));
  CK(cudaMemsetAsync(dst, 0, sizeof(double) * ng, ctx->stream));
  const Species &sp = ctx->species[id];
  if (sp.fp32)
    launch_temperature_f32(ctx->g, sp.f32, ctx->d_temp_acc, ctx->stream);
  else
    launch_temperature_f64(ctx->g, sp.dev, ctx->d_temp_acc, ctx->stream);
  launch_temperature_normalize(ctx->g, ctx->d_temp_acc, sp.mass_si, sp.charge_si, dst,
                               ctx->stream);
  ctx->launches += 2;
  return PDP3G_OK;
}

// ParticlesDensity::reset + calc_density of species id into dst (device grid)
static pdp3g_status density_into(pdp3g_ctx *ctx, int id, double *dst) {
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemsetAsync(dst, 0, sizeof(double) * ng, ctx->stream));
  const Species &sp = ctx->species[id];
  if (sp.fp32)
    launch_density_f32(ctx->g, sp.f32, sp.mass_si, dst, ctx->stream);
  else
    launch_density_f64(ctx->g, sp.dev, dst, ctx->stream);
  ctx->launches++;
  return PDP3G_OK;
}

// the per-species component comp of species id into ctx->d_scratch2
static pdp3g_status species_diag_into(pdp3g_ctx *ctx, int32_t comp, int32_t id) {
  if (comp == PDP3G_PROBE_T) return temperature_into(ctx, id, ctx->d_scratch2);
  if (comp == PDP3G_PROBE_DENSITY) return density_into(ctx, id, ctx->d_scratch2);
  return fail(ctx, PDP3G_INVALID_ARG, "unknown per-species component");
}

// ProbePlain::write's region (src/probePlain.cpp:80-170) of one component
pdp3g_status pdp3g_probe_read(pdp3g_ctx *ctx, int32_t comp, int32_t type, int32_t r0, int32_t z0,
                              int32_t r1, int32_t z1, double *host_out, int64_t capacity,
                              int64_t *count) {
  if (!ctx || !host_out) return PDP3G_INVALID_ARG;
  const long long n = probe_count(ctx, type, r0, z0, r1, z1);
  if (n == 0) return fail(ctx, PDP3G_INVALID_ARG, "probe_read: region outside the grid");
  if (capacity < n) return fail(ctx, PDP3G_INVALID_ARG, "probe_read: output too small");
  const bool rho_beam = comp == PDP3G_PROBE_RHO_BEAM;
  if (!rho_beam && (comp < 0 || comp >= PDP3G_NCOMP))
    return fail(ctx, PDP3G_INVALID_ARG, "probe_read: unknown component");
  CK(cudaSetDevice(ctx->device));
  pdp3g_status es = ensure_scratch(ctx);
  if (es != PDP3G_OK) return es;
  const double *src = comp_ptr(ctx, rho_beam ? 0 : comp);
  if (rho_beam) {
    // LoadInitParam::dump_data: every bunch's charge_weighting into c_rho_bunch
    uint32_t mask = 0;
    for (size_t s = 0; s < ctx->species.size() && s < 32; s++)
      if (ctx->species[s].is_bunch) mask |= 1u << s;
    pdp3g_status rs = rho_into(ctx, mask, ctx->d_scratch2);
    if (rs != PDP3G_OK) return rs;
    src = ctx->d_scratch2;
  }
  return probe_to_host(ctx, src, type, r0, z0, r1, z1, n, host_out, count);
}

// dump_data's per-species probes: T (TemperatureClassic) or density
// (ParticlesDensity) of species id
pdp3g_status pdp3g_probe_read_species(pdp3g_ctx *ctx, int32_t comp, int32_t id, int32_t type,
                                      int32_t r0, int32_t z0, int32_t r1, int32_t z1,
                                      double *host_out, int64_t capacity, int64_t *count) {
  if (!ctx || !host_out || id < 0 || id >= (int32_t)ctx->species.size())
    return fail(ctx, PDP3G_INVALID_ARG, "probe_read_species: bad arguments");
  if (comp != PDP3G_PROBE_T && comp != PDP3G_PROBE_DENSITY)
    return fail(ctx, PDP3G_INVALID_ARG, "probe_read_species: unknown component");
  const long long n = probe_count(ctx, type, r0, z0, r1, z1);
  if (n == 0) return fail(ctx, PDP3G_INVALID_ARG, "probe_read_species: region outside the grid");
  if (capacity < n) return fail(ctx, PDP3G_INVALID_ARG, "probe_read_species: output too small");
  CK(cudaSetDevice(ctx->device));
  pdp3g_status es = ensure_scratch(ctx);
  if (es != PDP3G_OK) return es;
  pdp3g_status ts = species_diag_into(ctx, comp, id);
  if (ts != PDP3G_OK) return ts;
  return probe_to_host(ctx, ctx->d_scratch2, type, r0, z0, r1, z1, n, host_out, count);
}

static pdp3g_status species_diag_to_host(pdp3g_ctx *ctx, int32_t comp, int32_t id,
                                         double *host_out) {
  if (!ctx || !host_out || id < 0 || id >= (int32_t)ctx->species.size()) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  pdp3g_status es = ensure_scratch(ctx);
  if (es != PDP3G_OK) return es;
  pdp3g_status ts = species_diag_into(ctx, comp, id);
  if (ts != PDP3G_OK) return ts;
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemcpyAsync(host_out, ctx->d_scratch2, sizeof(double) * ng, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return PDP3G_OK;
}

pdp3g_status pdp3g_temperature(pdp3g_ctx *ctx, int32_t id, double *host_out) {
  return species_diag_to_host(ctx, PDP3G_PROBE_T, id, host_out);
}

pdp3g_status pdp3g_density(pdp3g_ctx *ctx, int32_t id, double *host_out) {
  return species_diag_to_host(ctx, PDP3G_PROBE_DENSITY, id, host_out);
}

// PoissonDirichlet::poisson_solve (src/poissonDirichlet.cpp:23-98): phi from
// rho (the given host grid, or the charge density of every species), then
// E_r and E_z from phi (poisson.cu).  phi persists in the context with its
// last row 0 (EField::set_fi_on_z).
pdp3g_status pdp3g_poisson_solve(pdp3g_ctx *ctx, const double *host_rho, double *host_fi) {
  if (!ctx) return PDP3G_INVALID_ARG;
  const int nr = ctx->cfg.n_grid_r, nz = ctx->cfg.n_grid_z;
  if (poisson_check(nz) != 0)
    return fail(ctx, PDP3G_INVALID_ARG,
                "poisson_solve: 2 n_grid_z + 2 must be a power of two <= 8192 (the radix-2 sine "
                "transform)");
  CK(cudaSetDevice(ctx->device));
  pdp3g_status es = ensure_scratch(ctx);
  if (es != PDP3G_OK) return es;
  const size_t ng = (size_t)nr * nz;
  cudaStream_t st = ctx->stream;
  if (!ctx->d_poisson) {
    // t, fi, alpha, beta grids and the nz mode constants
    CK(dalloc(ctx, &ctx->d_poisson, 4 * ng + (size_t)nz));
    CK(cudaMemsetAsync(ctx->d_poisson, 0, sizeof(double) * (4 * ng + (size_t)nz), st));
    // b = 2 (1 - dr^2/dz^2 (cos(PI (k+1) / (n_grid_z+1)) - 1)) with the host libm
    std::vector<double> b(nz);
    const double dr = ctx->dr, dz = ctx->dz;
    for (int k = 0; k < nz; k++)
      b[k] = 2. * (1. - dr * dr / (dz * dz) * (std::cos(PI * (k + 1) / (nz + 1)) - 1));
    CK(cudaMemcpyAsync(ctx->d_poisson + 4 * ng, b.data(), sizeof(double) * nz,
                       cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
  }
  double *t = ctx->d_poisson, *fi = t + ng, *alpha = t + 2 * ng, *beta = t + 3 * ng;
  const double *b_mode = t + 4 * ng;
  if (host_rho) {
    CK(cudaMemcpyAsync(ctx->d_scratch2, host_rho, sizeof(double) * ng, cudaMemcpyHostToDevice, st));
  } else {
    pdp3g_status rs = rho_into(ctx, 0xFFFFFFFFu, ctx->d_scratch2);
    if (rs != PDP3G_OK) return rs;
  }
  CK(launch_poisson(ctx->g, ctx->d_scratch2, t, fi, alpha, beta, b_mode,
                    comp_ptr(ctx, PDP3G_E_R), comp_ptr(ctx, PDP3G_E_Z), st));
  ctx->launches += 4;
  refresh_mirror(ctx, PDP3G_E_R);
  refresh_mirror(ctx, PDP3G_E_Z);
  if (host_fi) CK(cudaMemcpyAsync(host_fi, fi, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(st));
  return PDP3G_OK;
}

// ProbePlain::mpwrite's selection (src/probePlain.cpp:172-224)
pdp3g_status pdp3g_probe_particles(pdp3g_ctx *ctx, int32_t id, int32_t r0, int32_t z0, int32_t r1,
                                   int32_t z1, double *r, double *z, double *vr, double *vphi,
                                   double *vz, int64_t capacity, int64_t *count) {
  if (!ctx || !count || id < 0 || id >= (int32_t)ctx->species.size()) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const Species &sp = ctx->species[id];
  const long long n = sp.fp32 ? sp.f32.n : sp.dev.n;
  *count = 0;
  if (n <= 0) return PDP3G_OK;
  // the species in the upstream units: FP64 arrays in place, or the FP32
  // cell-local state converted into the staging buffer
  const double *src[5];
  pdp3g_status rs = stage_reserve(ctx, (size_t)n * 2);  // 6n for the state, the rest for output
  if (rs != PDP3G_OK) return rs;
  double *S = ctx->d_stage;
  if (sp.fp32) {
    launch_cell_to_f64(sp.f32, ctx->dr, ctx->dz, ctx->cfg.n_grid_z - 1, S, S + n, S + 2 * n,
                       S + 3 * n, S + 4 * n, nullptr, st);
    ctx->launches++;
    for (int a = 0; a < 5; a++) src[a] = S + (size_t)a * n;
  } else {
    src[0] = sp.dev.r;
    src[1] = sp.dev.z;
    src[2] = sp.dev.vr;
    src[3] = sp.dev.vphi;
    src[4] = sp.dev.vz;
  }
  const long long nb = mp_blocks(n);
  unsigned *d_counts = nullptr;
  unsigned long long *d_off = nullptr;
  CK(cudaMalloc(&d_counts, sizeof(unsigned) * (size_t)nb));
  cudaError_t e = cudaMalloc(&d_off, sizeof(unsigned long long) * (size_t)nb);
  if (e != cudaSuccess) {
    cudaFree(d_counts);
    return cuda_fail(ctx, e, "probe_particles");
  }
  launch_mp_count(src[0], src[1], n, ctx->dr, ctx->dz, r0, z0, r1, z1, d_counts, st);
  std::vector<unsigned> counts((size_t)nb);
  std::vector<unsigned long long> off((size_t)nb);
  e = cudaMemcpyAsync(counts.data(), d_counts, sizeof(unsigned) * (size_t)nb,
                      cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  unsigned long long total = 0;
  for (long long b = 0; b < nb; b++) {
    off[(size_t)b] = total;
    total += counts[(size_t)b];
  }
  if (e == cudaSuccess && (long long)total <= capacity && total > 0) {
    // the selected particles land after the converted state (6n staging holds 12n doubles
    // after the reserve above)
    double *D = S + (size_t)6 * n;
    MpArrays arr;
    for (int a = 0; a < 5; a++) {
      arr.src[a] = src[a];
      arr.dst[a] = D + (size_t)a * total;
    }
    e = cudaMemcpyAsync(d_off, off.data(), sizeof(unsigned long long) * (size_t)nb,
                        cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
      launch_mp_write(arr, n, ctx->dr, ctx->dz, r0, z0, r1, z1, d_off, st);
      ctx->launches++;
      double *outs[5] = {r, z, vr, vphi, vz};
      for (int a = 0; a < 5 && e == cudaSuccess; a++)
        if (outs[a])
          e = cudaMemcpyAsync(outs[a], arr.dst[a], sizeof(double) * (size_t)total,
                              cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
  }
  cudaFree(d_counts);
  cudaFree(d_off);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "probe_particles");
  *count = (int64_t)total;
  if ((long long)total > capacity)
    return fail(ctx, PDP3G_INVALID_ARG, "probe_particles: output too small (count holds the need)");
  return PDP3G_OK;
}

pdp3g_status pdp3g_mark_initial_charge(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  if (!ctx->d_rho0) CK(dalloc(ctx, &ctx->d_rho0, ng));
  pdp3g_status st = rho_into(ctx, 0xFFFFFFFFu, ctx->d_rho0);
  if (st != PDP3G_OK) return st;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->has_rho0 = true;
  return PDP3G_OK;
}

pdp3g_status pdp3g_diagnostics(pdp3g_ctx *ctx, pdp3g_diag *out) {
  if (!ctx || !out) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  pdp3g_status st = ensure_scratch(ctx);
  if (st != PDP3G_OK) return st;
  cudaStream_t s = ctx->stream;
  double *red = ctx->d_red;
  // red[0..2]: field energy, sum res^2, sum rho dV; red[3]: sum over species of |rho_s|^2;
  // red[4..5]: kinetic energy, alive (accumulated below on the host)
  if ((st = rho_into(ctx, 0xFFFFFFFFu, ctx->d_scratch)) != PDP3G_OK) return st;
  launch_grid_diag(ctx->g, ctx->d_scratch, ctx->has_rho0 ? ctx->d_rho0 : nullptr,
                   ctx->d_partials, red, s);
  double host[16] = {0};
  CK(cudaMemcpyAsync(host, red, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double rho_sq = 0, kin = 0, alive = 0;
  for (size_t sp = 0; sp < ctx->species.size() && sp < 32; sp++) {
    if ((st = rho_into(ctx, 1u << sp, ctx->d_scratch2)) != PDP3G_OK) return st;
    launch_rho_norm(ctx->g, ctx->d_scratch2, ctx->d_partials, red + 8, s);
    if (ctx->species[sp].fp32)
      launch_kinetic_f32(ctx->species[sp].f32, ctx->species[sp].mass_si, ctx->d_partials, red + 9,
                         s);
    else
      launch_kinetic_f64(ctx->species[sp].dev, ctx->d_partials, red + 9, s);
    double h3[3];
    CK(cudaMemcpyAsync(h3, red + 8, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    rho_sq += h3[0];
    kin += h3[1];
    alive += h3[2];
  }
  CK(cudaGetLastError());
  out->field_energy = host[0];
  out->gauss_residual = std::sqrt(host[1]);
  out->charge_total = host[2];
  out->gauss_norm = std::sqrt(rho_sq);
  out->kinetic_energy = kin;
  out->alive = (int64_t)alive;
  return PDP3G_OK;
}

pdp3g_status pdp3g_set_timing(pdp3g_ctx *ctx, int32_t enabled) {
  if (!ctx) return PDP3G_INVALID_ARG;
  ctx->timing = enabled != 0;
  return PDP3G_OK;
}

pdp3g_status pdp3g_reset_timing(pdp3g_ctx *ctx) {
  if (!ctx) return PDP3G_INVALID_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->events_used = 0;
  ctx->acc = pdp3g_timing{};
  ctx->launches = ctx->particle_launches = ctx->steps = 0;
  return PDP3G_OK;
}

pdp3g_status pdp3g_get_timing(pdp3g_ctx *ctx, pdp3g_timing *out) {
  if (!ctx || !out) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  pdp3g_status st = harvest_timing(ctx);
  if (st != PDP3G_OK) return st;
  *out = ctx->acc;
  out->launches = ctx->launches;
  out->particle_launches = ctx->particle_launches;
  out->steps = ctx->steps;
  return PDP3G_OK;
}

double pdp3g_current_time(pdp3g_ctx *ctx) { return ctx ? ctx->t : 0.0; }
void *pdp3g_stream(pdp3g_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
int64_t pdp3g_device_bytes(pdp3g_ctx *ctx) { return ctx ? ctx->bytes : 0; }


// ------------------------------------------------------------ batched ensemble

struct pdp3g_ensemble {
  std::vector<pdp3g_ctx *> runs;
  int device = 0;
  int n_sm = 148;
  cudaStream_t stream = nullptr;
  EnsRun *d_runs = nullptr;
  EnsSpecies *d_species = nullptr;
  int *d_status = nullptr;
  long long *d_budget = nullptr;
  int *h_cancel = nullptr;  // host-mapped
  int *d_cancel = nullptr;
  EnsembleDev dev{};
  std::vector<EnsRun> h_runs;
  int blocks_per_sm = 0;
  int max_blocks_per_sm = 0;
  int pusher = -1;  // the pusher every run uses (compiled into the kernel), or -1
  double budget_ms = 0;
  long long budget_host = 0;  // cycles, source of the copy to d_budget
  long long clock_khz = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_blocks = -1;
  int sort_interval = 0;        // re-sort every run by cell every this many steps
  int64_t steps_total = 0;      // steps advanced by this ensemble (sort schedule)
  bool graph_ok = true;
  bool last_used_graph = false;
  double last_ms = 0;
  int64_t last_steps_done = 0;
  int64_t total_particles = 0;
  std::string last_error;
  // step-graph mode: one captured graph of one step of every run
  int mode = PDP3G_ENS_PERSISTENT;
  int graph_bpsm = 0;  // CTAs per SM of the runs' particle kernels in the step graph (0: theirs)
  cudaGraph_t step_graph = nullptr;
  cudaGraphExec_t step_exec = nullptr;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
};

static pdp3g_status ens_fail(pdp3g_ensemble *e, pdp3g_status st, const std::string &m) {
  if (e) e->last_error = m;
  return st;
}

#define EK(call)                                                                  \
  do {                                                                            \
    cudaError_t _e = (call);                                                      \
    if (_e != cudaSuccess)                                                        \
      return ens_fail(e, _e == cudaErrorMemoryAllocation ? PDP3G_NO_MEMORY : PDP3G_CUDA_ERROR, \
                      std::string(#call) + ": " + cudaGetErrorString(_e));      \
  } while (0)

void pdp3g_ensemble_destroy(pdp3g_ensemble *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  if (e->step_exec) cudaGraphExecDestroy(e->step_exec);
  if (e->step_graph) cudaGraphDestroy(e->step_graph);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  for (auto ev : e->ev_join) cudaEventDestroy(ev);
  cudaFree(e->d_runs);
  cudaFree(e->d_species);
  cudaFree(e->d_status);
  cudaFree(e->d_budget);
  if (e->h_cancel) cudaFreeHost(e->h_cancel);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

pdp3g_status pdp3g_ensemble_create(pdp3g_ctx *const *runs, int32_t n_runs, pdp3g_ensemble **out) {
  if (!runs || n_runs <= 0 || !out) return PDP3G_INVALID_ARG;
  *out = nullptr;
  pdp3g_ensemble *e = new pdp3g_ensemble();
  e->device = runs[0]->device;
  auto bail = [&](pdp3g_status st, const std::string &m) {
    if (runs[0]) runs[0]->last_error = m;
    pdp3g_ensemble_destroy(e);
    return st;
  };
  std::vector<EnsSpecies> hs;
  long long h = 0, ee = 0, j = 0, ch = 0;
  for (int r = 0; r < n_runs; r++) {
    pdp3g_ctx *c = runs[r];
    if (!c || c->device != e->device)
      return bail(PDP3G_INVALID_ARG, "ensemble runs must share one device");
    if (c->cfg.precision != PDP3G_FP32_CELL)
      return bail(PDP3G_NOT_SUPPORTED, "ensemble runs use the FP32 cell-local form");
    e->runs.push_back(c);
    EnsRun er{};
    er.g = c->g;
    er.t = c->t;
    er.pusher = c->cfg.pusher;
    er.h_begin = h;
    er.e_begin = ee;
    er.j_begin = j;
    er.chunk_begin = ch;
    h += (long long)c->g.nr * (c->g.nz - 1);
    ee += (long long)(c->g.nr - 1) * (c->g.nz - 1);
    j += (long long)c->g.nr * c->g.nz;
    for (auto &sp : c->species) {
      EnsSpecies es{};
      es.s = sp.f32;
      es.run = r;
      es.chunk_begin = ch;
      es.is_bunch = sp.is_bunch ? 1 : 0;
      es.duration = sp.duration;
      es.bunch_number = sp.bunch_number;
      es.hole_duration = sp.hole_duration;
      es.velocity = sp.velocity;
      if (sp.is_bunch)
        es.uz_beam = (float)(sp.velocity / (LIGHT_SPEED * std::sqrt(1.0 - sp.velocity * sp.velocity /
                                                                           LIGHT_SPEED_POW_2)));
      ch += (sp.f32.n + F32_CHUNK - 1) / F32_CHUNK;
      e->total_particles += sp.f32.n;
      hs.push_back(es);
    }
    e->h_runs.push_back(er);
  }
  cudaError_t ce = cudaSetDevice(e->device);
  if (ce != cudaSuccess) return bail(PDP3G_CUDA_ERROR, "cudaSetDevice");
  cudaDeviceGetAttribute(&e->n_sm, cudaDevAttrMultiProcessorCount, e->device);
  int khz = 0;
  cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, e->device);
  e->clock_khz = khz;
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&e->d_runs, sizeof(EnsRun) * n_runs) != cudaSuccess ||
      cudaMalloc(&e->d_species, sizeof(EnsSpecies) * std::max<size_t>(hs.size(), 1)) !=
          cudaSuccess ||
      cudaMalloc(&e->d_status, sizeof(int) * 4) != cudaSuccess ||
      cudaMalloc(&e->d_budget, sizeof(long long)) != cudaSuccess ||
      cudaHostAlloc(&e->h_cancel, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&e->d_cancel, e->h_cancel, 0) != cudaSuccess)
    return bail(PDP3G_CUDA_ERROR, "ensemble allocation");
  *e->h_cancel = 0;
  cudaMemcpy(e->d_runs, e->h_runs.data(), sizeof(EnsRun) * n_runs, cudaMemcpyHostToDevice);
  if (!hs.empty())
    cudaMemcpy(e->d_species, hs.data(), sizeof(EnsSpecies) * hs.size(), cudaMemcpyHostToDevice);
  EnsembleDev &d = e->dev;
  d.runs = e->d_runs;
  d.nruns = n_runs;
  d.species = e->d_species;
  d.nspecies = (int)hs.size();
  d.total_h = h;
  d.total_e = ee;
  d.total_j = j;
  d.total_chunks = ch;
  d.inv_pow11 = runs[0]->d_inv_pow11;
  d.cancel = e->d_cancel;
  d.status = e->d_status;
  d.budget_cycles = e->d_budget;
  cudaMemset(e->d_budget, 0, sizeof(long long));
  for (auto *c : e->runs)
    if (c->cfg.sort_interval > 0 &&
        (e->sort_interval == 0 || c->cfg.sort_interval < e->sort_interval))
      e->sort_interval = c->cfg.sort_interval;
  e->pusher = e->runs[0]->cfg.pusher;
  for (auto *c : e->runs)
    if (c->cfg.pusher != e->pusher) e->pusher = -1;
  e->max_blocks_per_sm = ensemble_max_blocks_per_sm(e->pusher);
  if (e->max_blocks_per_sm <= 0) return bail(PDP3G_CUDA_ERROR, "ensemble kernel does not fit");
  e->blocks_per_sm = e->max_blocks_per_sm;
  *out = e;
  return PDP3G_OK;
}

static pdp3g_status ens_launch(pdp3g_ensemble *e, bool allow_graph) {
  const int blocks = e->n_sm * e->blocks_per_sm;
  // 0 means no budget; any positive budget is at least one cycle.  Written
  // to device memory on the launch stream, so a replayed graph reads it.
  e->budget_host =
      e->budget_ms > 0 ? std::max<long long>(1, (long long)std::ceil(e->budget_ms * e->clock_khz)) : 0;
  EK(cudaMemcpyAsync(e->d_budget, &e->budget_host, sizeof(long long), cudaMemcpyHostToDevice,
                     e->stream));
  e->last_used_graph = false;
  if (allow_graph && e->graph_ok) {
    if (e->exec && e->graph_blocks != blocks) {
      cudaGraphExecDestroy(e->exec);
      cudaGraphDestroy(e->graph);
      e->exec = nullptr;
      e->graph = nullptr;
    }
    if (!e->exec) {
      cudaError_t c1 = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
      cudaError_t c2 = c1 == cudaSuccess ? ensemble_launch(e->dev, blocks, e->pusher, e->stream) : c1;
      cudaGraph_t g = nullptr;
      cudaError_t c3 = c1 == cudaSuccess ? cudaStreamEndCapture(e->stream, &g) : c1;
      // the captured node must keep the cooperative attribute: the kernel's
      // grid-wide barriers need co-resident CTAs
      bool coop = false;
      if (c2 == cudaSuccess && c3 == cudaSuccess && g) {
        size_t nn = 0;
        if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn == 1) {
          cudaGraphNode_t node;
          cudaGraphNodeType ty;
          cudaLaunchAttributeValue v = {};
          if (cudaGraphGetNodes(g, &node, &nn) == cudaSuccess &&
              cudaGraphNodeGetType(node, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel &&
              cudaGraphKernelNodeGetAttribute(node, cudaLaunchAttributeCooperative, &v) ==
                  cudaSuccess)
            coop = v.cooperative != 0;
        }
      }
      cudaError_t c4 = (c2 == cudaSuccess && c3 == cudaSuccess && coop)
                           ? cudaGraphInstantiate(&e->exec, g, 0)
                           : cudaErrorUnknown;
      if (c4 == cudaSuccess) {
        e->graph = g;
        e->graph_blocks = blocks;
      } else {
        if (g) cudaGraphDestroy(g);
        e->exec = nullptr;
        e->graph_ok = false;  // capture of a cooperative launch refused: launch directly
        cudaGetLastError();
      }
    }
    if (e->exec) {
      EK(cudaGraphLaunch(e->exec, e->stream));
      e->last_used_graph = true;
      return PDP3G_OK;
    }
  }
  EK(ensemble_launch(e->dev, blocks, e->pusher, e->stream));
  return PDP3G_OK;
}

// Step-graph mode: captures one step of every run as one graph.  The
// injection of every bunch runs first (device time of each run), then each
// run's own phases on its own streams (HField::calc_field, reset_j, the
// particle phase with its two-stream fork, EField::calc_field; the same
// launches as pdp3g_step), and after the runs' branches join, t += dt of
// every run on the device.  Nothing in the graph depends on the step, so one
// graph serves every step.
static pdp3g_status ens_capture_step(pdp3g_ensemble *e) {
  if (e->step_exec) return PDP3G_OK;
  if (!e->ev_fork) EK(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
  while (e->ev_join.size() < e->runs.size()) {
    cudaEvent_t ev;
    EK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    e->ev_join.push_back(ev);
  }
  // the runs' particle kernels take the step graph's CTAs-per-SM count while
  // it is captured; each context keeps its own for its own steps
  std::vector<int> own_bpsm;
  for (auto *c : e->runs) {
    own_bpsm.push_back(c->f32_blocks_per_sm);
    if (e->graph_bpsm > 0) c->f32_blocks_per_sm = e->graph_bpsm;
  }
  cudaError_t ce = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
  if (ce != cudaSuccess) {
    for (size_t r = 0; r < e->runs.size(); r++) e->runs[r]->f32_blocks_per_sm = own_bpsm[r];
    return ens_fail(e, PDP3G_CUDA_ERROR, cudaGetErrorString(ce));
  }
  ce = ensemble_inject_all(e->dev, e->stream);
  if (ce == cudaSuccess) ce = cudaEventRecord(e->ev_fork, e->stream);
  for (size_t r = 0; r < e->runs.size() && ce == cudaSuccess; r++) {
    pdp3g_ctx *ctx = e->runs[r];
    ce = cudaStreamWaitEvent(ctx->stream, e->ev_fork, 0);
    if (ce != cudaSuccess) break;
    phase_calc_h(ctx);
    ce = phase_reset_j(ctx);
    if (ce == cudaSuccess) ce = phase_particles(ctx);
    if (ce != cudaSuccess) break;
    phase_calc_e(ctx);
    ce = cudaEventRecord(e->ev_join[r], ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->stream, e->ev_join[r], 0);
  }
  if (ce == cudaSuccess) ce = ensemble_advance(e->dev, e->stream);
  cudaGraph_t g = nullptr;
  cudaError_t ce2 = cudaStreamEndCapture(e->stream, &g);
  for (size_t r = 0; r < e->runs.size(); r++) e->runs[r]->f32_blocks_per_sm = own_bpsm[r];
  if (ce == cudaSuccess) ce = ce2;
  if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->step_exec, g, 0);
  if (ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    e->step_exec = nullptr;
    cudaGetLastError();
    return ens_fail(e, PDP3G_CUDA_ERROR,
                    std::string("step graph capture: ") + cudaGetErrorString(ce));
  }
  e->step_graph = g;
  return PDP3G_OK;
}

// nsteps replays of the step graph; the cancel flag and the budget are
// checked between steps, with at most kInFlight steps queued ahead
static pdp3g_status ens_segment_graph(pdp3g_ensemble *e, int nsteps, float *ms_out, int *done,
                                      int *stop) {
  pdp3g_status cs = ens_capture_step(e);
  if (cs != PDP3G_OK) return cs;
  for (size_t r = 0; r < e->runs.size(); r++) e->h_runs[r].t = e->runs[r]->t;
  EK(cudaMemcpyAsync(e->d_runs, e->h_runs.data(), sizeof(EnsRun) * e->h_runs.size(),
                     cudaMemcpyHostToDevice, e->stream));
  const int init[4] = {0, 0, nsteps, 0};
  EK(cudaMemcpyAsync(e->d_status, init, sizeof(init), cudaMemcpyHostToDevice, e->stream));
  constexpr int kInFlight = 8;
  cudaEvent_t start = nullptr, end = nullptr, mark[kInFlight] = {};
  auto free_events = [&]() {
    if (start) cudaEventDestroy(start);
    if (end) cudaEventDestroy(end);
    for (int i = 0; i < kInFlight; i++)
      if (mark[i]) cudaEventDestroy(mark[i]);
  };
  bool made = cudaEventCreate(&start) == cudaSuccess && cudaEventCreate(&end) == cudaSuccess;
  for (int i = 0; i < kInFlight && made; i++) made = cudaEventCreate(&mark[i]) == cudaSuccess;
  if (!made || cudaEventRecord(start, e->stream) != cudaSuccess) {
    free_events();
    cudaGetLastError();
    return ens_fail(e, PDP3G_CUDA_ERROR, "step graph: timing events");
  }
  int launched = 0, st_code = 0;
  cudaError_t err = cudaSuccess;
  e->last_used_graph = true;
  for (; launched < nsteps; launched++) {
    if (*(volatile int *)e->h_cancel) { st_code = 1; break; }
    if (launched >= kInFlight) {
      // the step launched kInFlight steps ago has ended: its time against the budget
      cudaEvent_t old = mark[launched % kInFlight];
      if ((err = cudaEventSynchronize(old)) != cudaSuccess) break;
      float el = 0;
      cudaEventElapsedTime(&el, start, old);
      if (e->budget_ms > 0 && el > e->budget_ms) { st_code = 2; break; }
    }
    if ((err = cudaGraphLaunch(e->step_exec, e->stream)) != cudaSuccess) break;
    cudaEventRecord(mark[launched % kInFlight], e->stream);
  }
  cudaEventRecord(end, e->stream);
  cudaError_t sync = cudaStreamSynchronize(e->stream);
  float ms = 0;
  cudaEventElapsedTime(&ms, start, end);
  free_events();
  if (err != cudaSuccess) return ens_fail(e, PDP3G_CUDA_ERROR, cudaGetErrorString(err));
  if (sync != cudaSuccess) return ens_fail(e, PDP3G_CUDA_ERROR, cudaGetErrorString(sync));
  for (auto *c : e->runs) {
    for (int i = 0; i < launched; i++) c->t = c->t + c->cfg.dt;
    c->steps += launched;
    c->sim_steps += launched;
  }
  e->steps_total += launched;
  *ms_out = ms;
  *done = launched;
  *stop = st_code;
  return PDP3G_OK;
}

// one persistent launch of nsteps steps; *done receives the steps done
static pdp3g_status ens_segment(pdp3g_ensemble *e, int nsteps, bool allow_graph, float *ms_out,
                                int *done, int *stop) {
  for (size_t r = 0; r < e->runs.size(); r++) e->h_runs[r].t = e->runs[r]->t;
  EK(cudaMemcpyAsync(e->d_runs, e->h_runs.data(), sizeof(EnsRun) * e->h_runs.size(),
                     cudaMemcpyHostToDevice, e->stream));
  const int init[4] = {0, 0, nsteps, 0};
  EK(cudaMemcpyAsync(e->d_status, init, sizeof(init), cudaMemcpyHostToDevice, e->stream));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, e->stream);
  pdp3g_status st = ens_launch(e, allow_graph);
  cudaEventRecord(b, e->stream);
  cudaError_t sync = cudaStreamSynchronize(e->stream);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (st != PDP3G_OK) return st;
  if (sync != cudaSuccess) return ens_fail(e, PDP3G_CUDA_ERROR, cudaGetErrorString(sync));
  int status[4] = {0, 0, 0, 0};
  EK(cudaMemcpy(status, e->d_status, sizeof(status), cudaMemcpyDeviceToHost));
  for (auto *c : e->runs) {
    for (int i = 0; i < status[0]; i++) c->t = c->t + c->cfg.dt;
    c->steps += status[0];
    c->sim_steps += status[0];
  }
  e->steps_total += status[0];
  *ms_out = ms;
  *done = status[0];
  *stop = status[1];
  return PDP3G_OK;
}

// re-sort every run's plasma species by cell (pdp3g_sort), device-timed
static pdp3g_status ens_sort(pdp3g_ensemble *e, float *ms_out) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, e->stream);
  for (auto *c : e->runs) {
    EK(cudaStreamWaitEvent(c->stream, a, 0));
    pdp3g_status st = sort_all(c);
    if (st != PDP3G_OK) return ens_fail(e, st, "ensemble re-sort: " + c->last_error);
    cudaEvent_t done;
    cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
    cudaEventRecord(done, c->stream);
    EK(cudaStreamWaitEvent(e->stream, done, 0));
    cudaEventDestroy(done);
  }
  cudaEventRecord(b, e->stream);
  EK(cudaStreamSynchronize(e->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms_out = ms;
  return PDP3G_OK;
}

static pdp3g_status ens_run(pdp3g_ensemble *e, int nsteps, bool allow_graph, float *ms_out) {
  EK(cudaSetDevice(e->device));
  for (auto *c : e->runs) EK(cudaStreamSynchronize(c->stream));
  float total = 0;
  int done_total = 0, stop = 0;
  while (done_total < nsteps && stop == 0) {
    int seg = nsteps - done_total;
    if (e->sort_interval > 0) {
      if (e->steps_total % e->sort_interval == 0) {
        float ms = 0;
        pdp3g_status st = ens_sort(e, &ms);
        if (st != PDP3G_OK) return st;
        total += ms;
      }
      seg = std::min<int>(seg, e->sort_interval - (int)(e->steps_total % e->sort_interval));
    }
    // the budget covers the whole call: each segment gets what is left
    const double saved_budget = e->budget_ms;
    if (saved_budget > 0) {
      if (total >= saved_budget) {
        stop = 2;
        break;
      }
      e->budget_ms = saved_budget - total;
    }
    float ms = 0;
    int done = 0;
    pdp3g_status st = e->mode == PDP3G_ENS_STEP_GRAPH
                          ? ens_segment_graph(e, seg, &ms, &done, &stop)
                          : ens_segment(e, seg, allow_graph, &ms, &done, &stop);
    e->budget_ms = saved_budget;
    if (st != PDP3G_OK) return st;
    total += ms;
    done_total += done;
  }
  e->last_ms = total;
  e->last_steps_done = done_total;
  if (ms_out) *ms_out = total;
  if (stop == 1) return ens_fail(e, PDP3G_TIMEOUT, "ensemble cancelled");
  if (stop == 2) return ens_fail(e, PDP3G_TIMEOUT, "ensemble time budget exhausted");
  return PDP3G_OK;
}

pdp3g_status pdp3g_ensemble_run(pdp3g_ensemble *e, int32_t nsteps) {
  if (!e || nsteps < 0) return PDP3G_INVALID_ARG;
  if (nsteps == 0) return PDP3G_OK;
  return ens_run(e, nsteps, true, nullptr);
}

pdp3g_status pdp3g_ensemble_autotune(pdp3g_ensemble *e, int32_t steps_per_trial,
                                     int32_t *blocks_per_sm) {
  if (!e || steps_per_trial <= 0) return PDP3G_INVALID_ARG;
  float best = 0;
  int best_b = e->blocks_per_sm;
  e->mode = PDP3G_ENS_PERSISTENT;
  for (int b = 1; b <= e->max_blocks_per_sm; b++) {
    e->blocks_per_sm = b;
    float ms = 0;
    pdp3g_status st = ens_run(e, steps_per_trial, false, &ms);
    if (st != PDP3G_OK) return st;
    if (b == 1 || ms < best) {
      best = ms;
      best_b = b;
    }
  }
  e->blocks_per_sm = best_b;
  // the step graph at 2, 4 and 8 CTAs per SM for the runs' particle kernels
  // (each capture and its first replay untimed: one warm-up step)
  e->mode = PDP3G_ENS_STEP_GRAPH;
  float ms_graph = 0;
  int best_g = 0;
  for (int gb : {2, 4, 8}) {
    if (e->step_exec) cudaGraphExecDestroy(e->step_exec);
    if (e->step_graph) cudaGraphDestroy(e->step_graph);
    e->step_exec = nullptr;
    e->step_graph = nullptr;
    e->graph_bpsm = gb;
    float ms = 0;
    pdp3g_status st = ens_run(e, 1, false, nullptr);
    if (st == PDP3G_OK) st = ens_run(e, steps_per_trial, false, &ms);
    if (st != PDP3G_OK) return st;
    if (best_g == 0 || ms < ms_graph) {
      ms_graph = ms;
      best_g = gb;
    }
  }
  if (best_g != e->graph_bpsm) {
    cudaGraphExecDestroy(e->step_exec);
    cudaGraphDestroy(e->step_graph);
    e->step_exec = nullptr;
    e->step_graph = nullptr;
    e->graph_bpsm = best_g;
  }
  e->mode = ms_graph < best ? PDP3G_ENS_STEP_GRAPH : PDP3G_ENS_PERSISTENT;
  if (blocks_per_sm) *blocks_per_sm = e->mode == PDP3G_ENS_STEP_GRAPH ? 0 : best_b;
  return PDP3G_OK;
}

pdp3g_status pdp3g_ensemble_set_mode(pdp3g_ensemble *e, int32_t mode) {
  if (!e || (mode != PDP3G_ENS_PERSISTENT && mode != PDP3G_ENS_STEP_GRAPH))
    return PDP3G_INVALID_ARG;
  e->mode = mode;
  return PDP3G_OK;
}

pdp3g_status pdp3g_ensemble_set_sort_interval(pdp3g_ensemble *e, int32_t steps) {
  if (!e || steps < 0) return PDP3G_INVALID_ARG;
  e->sort_interval = steps;
  return PDP3G_OK;
}

pdp3g_status pdp3g_ensemble_set_budget(pdp3g_ensemble *e, double max_ms) {
  if (!e || max_ms < 0) return PDP3G_INVALID_ARG;
  e->budget_ms = max_ms;
  return PDP3G_OK;
}

pdp3g_status pdp3g_ensemble_cancel(pdp3g_ensemble *e, int32_t cancel) {
  if (!e) return PDP3G_INVALID_ARG;
  *(volatile int *)e->h_cancel = cancel ? 1 : 0;
  return PDP3G_OK;
}

pdp3g_status pdp3g_ensemble_info(pdp3g_ensemble *e, pdp3g_ensemble_stats *out) {
  if (!e || !out) return PDP3G_INVALID_ARG;
  out->runs = (int32_t)e->runs.size();
  out->blocks_per_sm = e->blocks_per_sm;
  out->blocks = e->n_sm * e->blocks_per_sm;
  out->used_graph = e->last_used_graph ? 1 : 0;
  out->last_ms = e->last_ms;
  out->last_steps_done = e->last_steps_done;
  out->particles = e->total_particles;
  out->mode = e->mode;
  out->graph_blocks_per_sm = e->graph_bpsm;
  return PDP3G_OK;
}

const char *pdp3g_ensemble_last_error(pdp3g_ensemble *e) { return e ? e->last_error.c_str() : ""; }

}  // extern "C"

// ------------------------------------------------------------------ adjoint
// Forward/backward (vector-Jacobian) pair over a window of FP32 steps.  The
// forward stores the fields (E, H) and the particle state at the start of
// every checkpoint interval and at the end; the backward walks the
// intervals last to first, recomputes each interval's steps from its
// checkpoint while storing every step's particle-phase input (particle
// state after injection, E and the half-step H), then runs the reverse of
// each step (adjoint.cu) from the last step of the interval to the first.

namespace {

struct AdjSnap {  // one species' FP32 particle state
  int *cell = nullptr;
  float *fr = nullptr, *fz = nullptr, *ur = nullptr, *uphi = nullptr, *uz = nullptr;
  uint8_t *alive = nullptr;
};

}  // namespace

struct pdp3g_adjoint {
  pdp3g_ctx *ctx = nullptr;
  int window = 0, interval = 0, r0 = 0, r1 = 0, z0 = 0, z1 = 0;
  int nwin = 0;
  std::vector<void *> allocs;
  int64_t bytes = 0;
  AdjGrids A{};
  double *lgrids = nullptr;  // 9 grids: lE, lH, lHh
  float *lj = nullptr;       // 3 grids: lJ
  std::vector<AdjSpeciesDev> ls;
  double *d_lv = nullptr;    // per species: adjoint of the bunch velocity
  double *d_loss = nullptr;
  double *ck_fields = nullptr;                 // (nwin + 1) x 6 grids (E, H)
  std::vector<std::vector<AdjSnap>> ck_parts;  // [nwin + 1][species]
  std::vector<double> ck_t;
  std::vector<int64_t> ck_steps;
  uint8_t *active = nullptr;                   // per cell, the reverse step's k_adj_active
  float4 *cap_quads = nullptr;                 // interval x 6 x cells: E and the half-step
                                               // H per cell (GridDev::q32), FP32
  std::vector<std::vector<AdjSnap>> cap_parts; // [interval + 1][species]: states of the
                                               // recomputed interval, slot j = step j's input
  std::vector<double> cap_t;
  bool have_forward = false;
  bool tail_captured = false;  // the capture slots hold the last interval as the forward ran it
  int face_terms = PDP3G_ADJ_DEFAULT_JUMPS;
  float face_h = PDP3G_ADJ_DEFAULT_FACE_WIDTH;  // adj::Consts::face_h
  double loss = 0;
  float fwd_ms = 0, bwd_ms = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

template <typename T>
cudaError_t aalloc(pdp3g_adjoint *a, T **p, size_t count) {
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * (count ? count : 1));
  if (e == cudaSuccess) {
    a->allocs.push_back((void *)*p);
    a->bytes += (int64_t)(sizeof(T) * count);
  }
  return e;
}

cudaError_t snap_alloc(pdp3g_adjoint *a, const SpeciesF32 &f, AdjSnap &s) {
  const size_t n = (size_t)f.n;
  cudaError_t e;
  if ((e = aalloc(a, &s.cell, n)) != cudaSuccess) return e;
  if ((e = aalloc(a, &s.fr, n)) != cudaSuccess) return e;
  if ((e = aalloc(a, &s.fz, n)) != cudaSuccess) return e;
  if ((e = aalloc(a, &s.ur, n)) != cudaSuccess) return e;
  if ((e = aalloc(a, &s.uphi, n)) != cudaSuccess) return e;
  if ((e = aalloc(a, &s.uz, n)) != cudaSuccess) return e;
  if (f.alive && (e = aalloc(a, &s.alive, n)) != cudaSuccess) return e;
  return cudaSuccess;
}

// dir 0: species -> snapshot, 1: snapshot -> species
cudaError_t snap_copy(const SpeciesF32 &f, const AdjSnap &s, int dir, cudaStream_t st) {
  const size_t n = (size_t)f.n;
  void *dev[7] = {f.cell, f.fr, f.fz, f.ur, f.uphi, f.uz, f.alive};
  void *snp[7] = {s.cell, s.fr, s.fz, s.ur, s.uphi, s.uz, s.alive};
  const size_t sz[7] = {4, 4, 4, 4, 4, 4, 1};
  for (int j = 0; j < 7; j++) {
    if (!dev[j] || !snp[j] || n == 0) continue;
    cudaError_t e = dir == 0 ? cudaMemcpyAsync(snp[j], dev[j], n * sz[j], cudaMemcpyDeviceToDevice, st)
                             : cudaMemcpyAsync(dev[j], snp[j], n * sz[j], cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

pdp3g_status adj_save_checkpoint(pdp3g_adjoint *a, int idx) {
  pdp3g_ctx *ctx = a->ctx;
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemcpyAsync(a->ck_fields + (size_t)idx * 6 * ng, comp_ptr(ctx, PDP3G_E_R),
                     sizeof(double) * 6 * ng, cudaMemcpyDeviceToDevice, ctx->stream));
  for (size_t j = 0; j < ctx->species.size(); j++)
    CK(snap_copy(ctx->species[j].f32, a->ck_parts[idx][j], 0, ctx->stream));
  a->ck_t[idx] = ctx->t;
  a->ck_steps[idx] = ctx->sim_steps;
  return PDP3G_OK;
}

// particles: also copy the checkpoint's particles into the context's species
// (the backward's recompute reads them from capture slot 0 instead)
pdp3g_status adj_restore_checkpoint(pdp3g_adjoint *a, int idx, bool particles = true) {
  pdp3g_ctx *ctx = a->ctx;
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemcpyAsync(comp_ptr(ctx, PDP3G_E_R), a->ck_fields + (size_t)idx * 6 * ng,
                     sizeof(double) * 6 * ng, cudaMemcpyDeviceToDevice, ctx->stream));
  for (int c = PDP3G_E_R; c <= PDP3G_E_Z; c++) refresh_mirror(ctx, c);
  for (size_t j = 0; particles && j < ctx->species.size(); j++)
    CK(snap_copy(ctx->species[j].f32, a->ck_parts[idx][j], 1, ctx->stream));
  ctx->t = a->ck_t[idx];
  ctx->sim_steps = a->ck_steps[idx];
  return PDP3G_OK;
}

// one step of the window (LoadInitParam::run's sequence without re-sorting:
// the adjoint keeps every particle in its slot); cap >= 0 stores the
// particle-phase input of the step into capture slot cap
// species j's arrays replaced by state slot `slot` of the window
SpeciesF32 slot_view(const pdp3g_adjoint *a, size_t j, int slot) {
  SpeciesF32 v = a->ctx->species[j].f32;
  const AdjSnap &sn = a->cap_parts[slot][j];
  v.cell = sn.cell;
  v.fr = sn.fr;
  v.fz = sn.fz;
  v.ur = sn.ur;
  v.uphi = sn.uphi;
  v.uz = sn.uz;
  v.alive = sn.alive;
  return v;
}

// one step of the window (LoadInitParam::run's sequence without re-sorting:
// the adjoint keeps every particle in its slot).  cap < 0: the context's own
// state, in place.  cap >= 0 (the backward's recompute): the particles of
// state slot cap are injected into, pushed and written to slot cap + 1, so
// slot cap keeps the particle phase's input for the reverse, with no copy.
pdp3g_status adj_forward_step(pdp3g_adjoint *a, int cap) {
  pdp3g_ctx *ctx = a->ctx;
  const size_t ncells = (size_t)(ctx->cfg.n_grid_r - 1) * (ctx->cfg.n_grid_z - 1);
  if (cap < 0) {
    phase_inject(ctx);
    phase_calc_h(ctx);
    CK(phase_reset_j(ctx));
    CK(phase_particles(ctx));
    phase_calc_e(ctx);
    phase_advance(ctx);
    return PDP3G_OK;
  }
  a->cap_t[cap] = ctx->t;
  for (size_t j = 0; j < ctx->species.size(); j++)
    if (ctx->species[j].is_bunch) inject_f32(ctx, ctx->species[j], slot_view(a, j, cap));
  phase_calc_h(ctx);
  CK(phase_reset_j(ctx));
  // the per-cell FP32 quads of E and the half-step H that this step's
  // particles gather, kept for the reverse
  pack_quads(ctx);
  CK(cudaMemcpyAsync(a->cap_quads + (size_t)cap * 6 * ncells, ctx->quads,
                     sizeof(float4) * 6 * ncells, cudaMemcpyDeviceToDevice, ctx->stream));
  CK(species_fork(ctx));
  for (size_t j = 0; j < ctx->species.size(); j++) {
    const SpeciesF32 in = slot_view(a, j, cap), nx = slot_view(a, j, cap + 1);
    launch_push_deposit_f32_to(ctx->g, in, in_place(nx), ctx->cfg.pusher, ctx->n_sm,
                               ctx->f32_blocks_per_sm, species_stream(ctx, j));
    ctx->launches++;
    ctx->particle_launches++;
  }
  CK(species_join(ctx));
  phase_calc_e(ctx);
  phase_advance(ctx);
  return PDP3G_OK;
}

// reverse of the step stored in capture slot cap; the species' reverses on
// two streams as in the forward step
cudaError_t adj_reverse_step(pdp3g_adjoint *a, int cap) {
  pdp3g_ctx *ctx = a->ctx;
  const size_t ncells = (size_t)(ctx->cfg.n_grid_r - 1) * (ctx->cfg.n_grid_z - 1);
  adj_launch_e(ctx->g, a->A, ctx->stream);
  adj_launch_active(ctx->g, a->A, a->active, ctx->stream);
  const float4 *Q = a->cap_quads + (size_t)cap * 6 * ncells;
  cudaError_t e = species_fork(ctx);
  if (e != cudaSuccess) return e;
  for (size_t j = 0; j < ctx->species.size(); j++) {
    const Species &sp = ctx->species[j];
    const cudaStream_t st = species_stream(ctx, j);
    AdjSpeciesDev S = a->ls[j];
    S.st = slot_view(a, j, cap);
    adj_launch_particles(ctx->g, Q, S, a->A, a->active, a->face_terms, a->face_h, st);
    if (sp.is_bunch) {
      long long start, count;
      inject_range(ctx, sp, a->cap_t[cap], start, count);
      adj_launch_inject(S, start, count, ctx->cfg.dt, ctx->dz, sp.velocity, ctx->d_inv_pow11,
                        a->d_lv + j, st);
    }
  }
  if ((e = species_join(ctx)) != cudaSuccess) return e;
  adj_launch_h(ctx->g, a->A, ctx->stream);
  return cudaGetLastError();
}

pdp3g_status adj_fail(pdp3g_adjoint *a, pdp3g_status st, const std::string &m) {
  if (a && a->ctx) a->ctx->last_error = m;
  return st;
}

}  // namespace

void pdp3g_adjoint_destroy(pdp3g_adjoint *a) {
  if (!a) return;
  if (a->ctx) cudaSetDevice(a->ctx->device);
  for (void *p : a->allocs) cudaFree(p);
  if (a->ev0) cudaEventDestroy(a->ev0);
  if (a->ev1) cudaEventDestroy(a->ev1);
  delete a;
}

pdp3g_status pdp3g_adjoint_create(pdp3g_ctx *ctx, int32_t window_steps,
                                  int32_t checkpoint_interval, int32_t probe_r0,
                                  int32_t probe_r1, int32_t probe_z0, int32_t probe_z1,
                                  pdp3g_adjoint **out) {
  if (!ctx || !out || window_steps <= 0 || checkpoint_interval <= 0)
    return fail(ctx, PDP3G_INVALID_ARG, "adjoint_create: bad arguments");
  *out = nullptr;
  const int nr = ctx->cfg.n_grid_r, nz = ctx->cfg.n_grid_z;
  if (probe_r0 < 0 || probe_r1 > nr || probe_r0 >= probe_r1 || probe_z0 < 0 || probe_z1 > nz ||
      probe_z0 >= probe_z1)
    return fail(ctx, PDP3G_INVALID_ARG, "adjoint_create: probe outside the grid");
  if (ctx->cfg.precision != PDP3G_FP32_CELL || ctx->cfg.pusher != PDP3G_PUSHER_BORIS)
    return fail(ctx, PDP3G_NOT_SUPPORTED,
                "adjoint: the FP32 cell-local form with the relativistic Boris pusher only");
  CK(cudaSetDevice(ctx->device));
  pdp3g_adjoint *a = new pdp3g_adjoint();
  a->ctx = ctx;
  a->window = window_steps;
  a->interval = std::min(checkpoint_interval, window_steps);
  a->nwin = (window_steps + a->interval - 1) / a->interval;
  a->r0 = probe_r0;
  a->r1 = probe_r1;
  a->z0 = probe_z0;
  a->z1 = probe_z1;
  const size_t ng = (size_t)nr * nz;
  const size_t nsp = ctx->species.size();
  cudaError_t e = cudaSuccess;
#define ACK(call)                                   \
  do {                                              \
    e = (call);                                     \
    if (e != cudaSuccess) {                         \
      pdp3g_adjoint_destroy(a);                     \
      return cuda_fail(ctx, e, #call);              \
    }                                               \
  } while (0)
  ACK(aalloc(a, &a->lgrids, 9 * ng));
  ACK(aalloc(a, &a->lj, 3 * ng));
  double *L = a->lgrids;
  float *J = a->lj;
  a->A = AdjGrids{L, L + ng, L + 2 * ng, L + 3 * ng, L + 4 * ng, L + 5 * ng,
                  L + 6 * ng, L + 7 * ng, L + 8 * ng, J, J + ng, J + 2 * ng};
  a->ls.resize(nsp);
  for (size_t j = 0; j < nsp; j++) {
    const size_t n = (size_t)ctx->species[j].f32.n;
    AdjSpeciesDev &S = a->ls[j];
    ACK(aalloc(a, &S.la, n));
    ACK(aalloc(a, &S.lb, n));
    ACK(aalloc(a, &S.lur, n));
    ACK(aalloc(a, &S.luphi, n));
    ACK(aalloc(a, &S.luz, n));
    ACK(aalloc(a, &S.lw, n));
  }
  ACK(aalloc(a, &a->d_lv, nsp + 1));
  ACK(aalloc(a, &a->d_loss, 1));
  ACK(aalloc(a, &a->ck_fields, (size_t)(a->nwin + 1) * 6 * ng));
  a->ck_parts.assign(a->nwin + 1, std::vector<AdjSnap>(nsp));
  a->ck_t.assign(a->nwin + 1, 0.0);
  a->ck_steps.assign(a->nwin + 1, 0);
  for (int c = 0; c <= a->nwin; c++)
    for (size_t j = 0; j < nsp; j++) ACK(snap_alloc(a, ctx->species[j].f32, a->ck_parts[c][j]));
  const size_t ncells = (size_t)(nr - 1) * (nz - 1);
  ACK(aalloc(a, &a->cap_quads, (size_t)a->interval * 6 * ncells));
  ACK(aalloc(a, &a->active, ncells));
  a->cap_parts.assign(a->interval + 1, std::vector<AdjSnap>(nsp));
  a->cap_t.assign(a->interval, 0.0);
  for (int c = 0; c <= a->interval; c++)
    for (size_t j = 0; j < nsp; j++) ACK(snap_alloc(a, ctx->species[j].f32, a->cap_parts[c][j]));
  ACK(cudaEventCreate(&a->ev0));
  ACK(cudaEventCreate(&a->ev1));
#undef ACK
  *out = a;
  return PDP3G_OK;
}

pdp3g_status pdp3g_forward_window(pdp3g_adjoint *a, double *loss) {
  if (!a) return PDP3G_INVALID_ARG;
  pdp3g_ctx *ctx = a->ctx;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  // The last interval runs through the capture slots, as the backward's
  // recompute would run it, so the first backward reverses it directly.
  const int tail0 = (a->nwin - 1) * a->interval;
  a->tail_captured = false;
  CK(cudaEventRecord(a->ev0, st));
  for (int s = 0; s < a->window; s++) {
    if (s % a->interval == 0) {
      pdp3g_status cs = adj_save_checkpoint(a, s / a->interval);
      if (cs != PDP3G_OK) return cs;
    }
    if (s == tail0)
      for (size_t j = 0; j < ctx->species.size(); j++)
        CK(snap_copy(ctx->species[j].f32, a->cap_parts[0][j], 0, st));
    pdp3g_status fs = adj_forward_step(a, s >= tail0 ? s - tail0 : -1);
    if (fs != PDP3G_OK) return fs;
  }
  for (size_t j = 0; j < ctx->species.size(); j++)
    CK(snap_copy(ctx->species[j].f32, a->cap_parts[a->window - tail0][j], 1, st));
  pdp3g_status cs = adj_save_checkpoint(a, a->nwin);
  if (cs != PDP3G_OK) return cs;
  CK(cudaMemsetAsync(a->d_loss, 0, sizeof(double), st));
  CK(cudaMemsetAsync(a->A.lEz, 0, sizeof(double) * ng, st));
  adj_launch_seed(ctx->g, a->A, a->r0, a->r1, a->z0, a->z1, a->d_loss, st);
  CK(cudaEventRecord(a->ev1, st));
  CK(cudaMemcpyAsync(&a->loss, a->d_loss, sizeof(double), cudaMemcpyDeviceToHost, st));
  pdp3g_status ss = pdp3g_sync(ctx);
  if (ss != PDP3G_OK) return ss;
  CK(cudaEventElapsedTime(&a->fwd_ms, a->ev0, a->ev1));
  a->have_forward = true;
  a->tail_captured = true;
  if (loss) *loss = a->loss;
  return PDP3G_OK;
}

pdp3g_status pdp3g_backward_window(pdp3g_adjoint *a) {
  if (!a) return PDP3G_INVALID_ARG;
  pdp3g_ctx *ctx = a->ctx;
  if (!a->have_forward)
    return adj_fail(a, PDP3G_INVALID_ARG, "backward_window: no forward_window to reverse");
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaEventRecord(a->ev0, st));
  CK(cudaMemsetAsync(a->lgrids, 0, sizeof(double) * 9 * ng, st));
  CK(cudaMemsetAsync(a->lj, 0, sizeof(float) * 3 * ng, st));
  for (size_t j = 0; j < a->ls.size(); j++) {
    const size_t n = (size_t)ctx->species[j].f32.n;
    AdjSpeciesDev &S = a->ls[j];
    float *fl[5] = {S.la, S.lb, S.lur, S.luphi, S.luz};
    for (float *p : fl) CK(cudaMemsetAsync(p, 0, sizeof(float) * n, st));
    CK(cudaMemsetAsync(S.lw, 0, sizeof(double) * n, st));
  }
  CK(cudaMemsetAsync(a->d_lv, 0, sizeof(double) * (a->ls.size() + 1), st));
  pdp3g_status rs = adj_restore_checkpoint(a, a->nwin);
  if (rs != PDP3G_OK) return rs;
  CK(cudaMemsetAsync(a->d_loss, 0, sizeof(double), st));
  adj_launch_seed(ctx->g, a->A, a->r0, a->r1, a->z0, a->z1, a->d_loss, st);
  for (int w = a->nwin - 1; w >= 0; w--) {
    const int s0 = w * a->interval, s1 = std::min(a->window, s0 + a->interval);
    if (!(w == a->nwin - 1 && a->tail_captured)) {
      rs = adj_restore_checkpoint(a, w, false);
      if (rs != PDP3G_OK) return rs;
      for (size_t j = 0; j < ctx->species.size(); j++)
        CK(snap_copy(slot_view(a, j, 0), a->ck_parts[w][j], 1, st));
      for (int s = s0; s < s1; s++) {
        pdp3g_status fs = adj_forward_step(a, s - s0);
        if (fs != PDP3G_OK) return fs;
      }
    }
    a->tail_captured = false;  // the slots now hold interval w
    for (int s = s1 - 1; s >= s0; s--) CK(adj_reverse_step(a, s - s0));
  }
  rs = adj_restore_checkpoint(a, a->nwin);
  if (rs != PDP3G_OK) return rs;
  CK(cudaEventRecord(a->ev1, st));
  CK(cudaGetLastError());
  pdp3g_status ss = pdp3g_sync(ctx);
  if (ss != PDP3G_OK) return ss;
  CK(cudaEventElapsedTime(&a->bwd_ms, a->ev0, a->ev1));
  return PDP3G_OK;
}

pdp3g_status pdp3g_adjoint_species(pdp3g_adjoint *a, int32_t id, double *l_r, double *l_z,
                                   double *l_ur, double *l_uphi, double *l_uz, double *l_w) {
  if (!a || id < 0 || id >= (int32_t)a->ls.size()) return PDP3G_INVALID_ARG;
  pdp3g_ctx *ctx = a->ctx;
  CK(cudaSetDevice(ctx->device));
  const size_t n = (size_t)ctx->species[id].f32.n;
  const AdjSpeciesDev &S = a->ls[id];
  std::vector<float> buf(n);
  const float *src[5] = {S.la, S.lb, S.lur, S.luphi, S.luz};
  double *dst[5] = {l_r, l_z, l_ur, l_uphi, l_uz};
  const double scale[5] = {1.0 / ctx->dr, 1.0 / ctx->dz, 1.0, 1.0, 1.0};
  for (int j = 0; j < 5; j++) {
    if (!dst[j] || n == 0) continue;
    CK(cudaMemcpy(buf.data(), src[j], sizeof(float) * n, cudaMemcpyDeviceToHost));
    for (size_t p = 0; p < n; p++) dst[j][p] = (double)buf[p] * scale[j];
  }
  if (l_w && n) CK(cudaMemcpy(l_w, S.lw, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return PDP3G_OK;
}

pdp3g_status pdp3g_adjoint_field(pdp3g_adjoint *a, int32_t comp, double *host_out) {
  if (!a || !host_out || comp < PDP3G_E_R || comp > PDP3G_H_Z) return PDP3G_INVALID_ARG;
  pdp3g_ctx *ctx = a->ctx;
  CK(cudaSetDevice(ctx->device));
  const size_t ng = (size_t)ctx->cfg.n_grid_r * ctx->cfg.n_grid_z;
  CK(cudaMemcpy(host_out, a->lgrids + (size_t)comp * ng, sizeof(double) * ng,
                cudaMemcpyDeviceToHost));
  return PDP3G_OK;
}

pdp3g_status pdp3g_adjoint_bunch_velocity(pdp3g_adjoint *a, int32_t id, double *l_v) {
  if (!a || !l_v || id < 0 || id >= (int32_t)a->ls.size()) return PDP3G_INVALID_ARG;

  pdp3g_ctx *ctx = a->ctx;
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpy(l_v, a->d_lv + id, sizeof(double), cudaMemcpyDeviceToHost));
  return PDP3G_OK;
}

pdp3g_status pdp3g_adjoint_timing(pdp3g_adjoint *a, double *forward_ms, double *backward_ms) {
  if (!a) return PDP3G_INVALID_ARG;
  if (forward_ms) *forward_ms = a->fwd_ms;
  if (backward_ms) *backward_ms = a->bwd_ms;
  return PDP3G_OK;
}

int64_t pdp3g_adjoint_bytes(pdp3g_adjoint *a) { return a ? a->bytes : 0; }

pdp3g_status pdp3g_adjoint_set_mode(pdp3g_adjoint *a, int32_t mode) {
  if (!a || (mode != PDP3G_ADJ_MEAN_FIELD && mode != PDP3G_ADJ_PATHWISE)) return PDP3G_INVALID_ARG;
  a->face_terms = mode == PDP3G_ADJ_MEAN_FIELD ? PDP3G_ADJ_DEFAULT_JUMPS : 0;
  return PDP3G_OK;
}

pdp3g_status pdp3g_adjoint_set_jump_terms(pdp3g_adjoint *a, uint32_t terms) {
  const uint32_t all = PDP3G_ADJ_GATHER_JUMPS | PDP3G_ADJ_WALL_JUMPS | PDP3G_ADJ_WALL_CELLS;
  if (!a || (terms & ~all)) return PDP3G_INVALID_ARG;
  a->face_terms = (int)terms;  // the bits of adj::Consts::face
  return PDP3G_OK;
}

pdp3g_status pdp3g_adjoint_set_face_width(pdp3g_adjoint *a, double half_width) {
  if (!a || !(half_width >= 0.0 && half_width <= 0.5)) return PDP3G_INVALID_ARG;
  a->face_h = (float)half_width;
  return PDP3G_OK;
}
