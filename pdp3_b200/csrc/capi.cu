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
  cudaEvent_t ev[6];
};

}  // namespace

struct pdp3g_ctx {
  pdp3g_config cfg{};
  int device = 0;
  int n_sm = 148;
  cudaStream_t stream = nullptr;
  double dr = 0, dz = 0, t = 0;
  double *grid_mem = nullptr;
  GridDev g{};
  unsigned *d_err = nullptr;
  double *d_inv_pow11 = nullptr;
  double *d_rho0 = nullptr;
  double *d_scratch = nullptr;   // one grid (charge density)
  double *d_scratch2 = nullptr;  // one grid (per-species charge density)
  double *d_partials = nullptr;  // per-block reduction partials
  double *d_red = nullptr;       // reduction results
  char *d_sort = nullptr;        // radix-sort scratch
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
  int64_t launches = 0, particle_launches = 0, steps = 0;
  std::string last_error;
  int64_t bytes = 0;
  int f32_blocks_per_sm = 4;  // CTAs per SM for the FP32 particle kernel
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
    float ms[5];
    for (int j = 0; j < 5; j++)
      CK(cudaEventElapsedTime(&ms[j], ctx->step_events[s].ev[j], ctx->step_events[s].ev[j + 1]));
    // ev0..1 injection, 1..2 H update, 2..3 J clear, 3..4 particles, 4..5 E update
    ctx->acc.ms_other += ms[0] + ms[2];
    ctx->acc.ms_fields += ms[1] + ms[4];
    ctx->acc.ms_particles += ms[3];
    ctx->acc.ms_step_total += ms[0] + ms[1] + ms[2] + ms[3] + ms[4];
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
  pdp3g_ctx *ctx = new pdp3g_ctx();
  ctx->cfg = *cfg;
  ctx->device = cfg->device;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) {
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
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
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
  cudaFree(ctx->d_err);
  cudaFree(ctx->d_inv_pow11);
  cudaFree(ctx->d_rho0);
  cudaFree(ctx->d_scratch);
  cudaFree(ctx->d_scratch2);
  cudaFree(ctx->d_partials);
  cudaFree(ctx->d_red);
  cudaFree(ctx->d_sort);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
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

// FP64 (r, z, v) -> cell-local FP32 (cell, offsets, u = gamma v / c)
static pdp3g_status to_cell_local(pdp3g_ctx *ctx, int64_t n, const double *r, const double *z,
                                  const double *vr, const double *vphi, const double *vz,
                                  std::vector<int> &cell, std::vector<float> &fr,
                                  std::vector<float> &fz, std::vector<float> &ur,
                                  std::vector<float> &uphi, std::vector<float> &uz) {
  const int nr = ctx->cfg.n_grid_r, nz = ctx->cfg.n_grid_z, ncz = nz - 1;
  const double dr = ctx->dr, dz = ctx->dz;
  cell.resize(n); fr.resize(n); fz.resize(n); ur.resize(n); uphi.resize(n); uz.resize(n);
  for (int64_t p = 0; p < n; p++) {
    if (!std::isfinite(r[p]) || !std::isfinite(z[p]))
      return fail(ctx, PDP3G_NAN_DETECTED, "particle position is NaN or Inf");
    int i = (int)std::ceil(r[p] / dr) - 1, k = (int)std::ceil(z[p] / dz) - 1;
    if (i < 0) i = 0;
    if (k < 0) k = 0;
    if (i > nr - 2 || k > nz - 2) return fail(ctx, PDP3G_OUT_OF_GRID, "particle outside the grid");
    cell[p] = i * ncz + k;
    fr[p] = (float)(r[p] / dr - i);
    fz[p] = (float)(z[p] / dz - k);
    const double v2 = vr[p] * vr[p] + vphi[p] * vphi[p] + vz[p] * vz[p];
    if (!(v2 < LIGHT_SPEED_POW_2)) return fail(ctx, PDP3G_V_GE_C, "velocity >= c");
    const double gc = 1.0 / (LIGHT_SPEED * std::sqrt(1.0 - v2 / LIGHT_SPEED_POW_2));
    ur[p] = (float)(vr[p] * gc);
    uphi[p] = (float)(vphi[p] * gc);
    uz[p] = (float)(vz[p] * gc);
  }
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

static pdp3g_status upload_f32(pdp3g_ctx *ctx, Species &sp, int64_t n, const double *r,
                               const double *z, const double *vr, const double *vphi,
                               const double *vz) {
  std::vector<int> cell;
  std::vector<float> fr, fz, ur, uphi, uz;
  pdp3g_status st = to_cell_local(ctx, n, r, z, vr, vphi, vz, cell, fr, fz, ur, uphi, uz);
  if (st != PDP3G_OK) return st;
  SpeciesF32 &f = sp.f32;
  size_t b = sizeof(float) * (size_t)n;
  CK(cudaMemcpy(f.cell, cell.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f.fr, fr.data(), b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f.fz, fz.data(), b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f.ur, ur.data(), b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f.uphi, uphi.data(), b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(f.uz, uz.data(), b, cudaMemcpyHostToDevice));
  return PDP3G_OK;
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
    pdp3g_status st = upload_f32(ctx, sp, n, r, z, vr, vphi, vz);
    if (st != PDP3G_OK) return st;
    std::vector<float> wv(w, w + n);
    CK(cudaMemcpy(wf, wv.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice));
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
  for (auto &sp : ctx->species)
    if (!sp.is_bunch) nmax = std::max<long long>(nmax, sp.fp32 ? sp.f32.n : sp.dev.n);
  if (nmax <= 1) return PDP3G_OK;
  const size_t need = sort_layout(nmax).total;
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

// Bunch::bunch_inject for every bunch (src/bunch.cpp:87-124)
static void phase_inject(pdp3g_ctx *ctx) {
  cudaStream_t st = ctx->stream;
  for (auto &sp : ctx->species) {
    if (!sp.is_bunch) continue;
    const double dt = ctx->cfg.dt;
    double begin = sp.duration * sp.bunch_number + sp.hole_duration * sp.bunch_number;
    double end = begin + sp.duration;
    double dl = sp.velocity * dt;
    int steps_amount = (int)std::ceil(sp.duration / dt);
    unsigned int number = (unsigned int)(sp.fp32 ? sp.f32.n : sp.dev.n);
    unsigned int particles_in_step = number / steps_amount;
    int start_number = (ctx->t - begin) / dt * particles_in_step;
    if (ctx->t >= begin && ctx->t < end && particles_in_step > 0) {
      // indices start_number + i for i < particles_in_step, kept below number
      long long start = (long long)(unsigned int)start_number;
      long long count = particles_in_step;
      if (start >= (long long)number) count = 0;
      else if (start + count > (long long)number) count = (long long)number - start;
      if (count > 0) {
        if (sp.fp32) {
          const double gv = sp.velocity / (LIGHT_SPEED * std::sqrt(1.0 - sp.velocity * sp.velocity /
                                                                              LIGHT_SPEED_POW_2));
          launch_bunch_inject_f32(sp.f32, start, count, dl, ctx->dz / 2.0, ctx->dz,
                                  ctx->cfg.n_grid_z - 1, (float)gv, ctx->d_inv_pow11, st);
        } else {
          launch_bunch_inject(sp.dev, start, count, dl, ctx->dz / 2.0, sp.velocity,
                              ctx->d_inv_pow11, st);
        }
        ctx->launches++;
      }
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

// ParticlesList::step_v + full_current_distribution (src/particlesList.cpp:20-54)
static void phase_particles(pdp3g_ctx *ctx) {
  for (auto &sp : ctx->species) {
    if (sp.fp32)
      launch_push_deposit_f32(ctx->g, sp.f32, ctx->cfg.pusher, ctx->n_sm, ctx->f32_blocks_per_sm,
                              ctx->stream);
    else
      launch_push_deposit_f64(ctx->g, sp.dev, ctx->cfg.pusher, ctx->n_sm, ctx->stream);
    ctx->launches++;
    ctx->particle_launches++;
  }
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
}

pdp3g_status pdp3g_step(pdp3g_ctx *ctx, int32_t nsteps) {
  if (!ctx || nsteps < 0) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  for (int s = 0; s < nsteps; s++) {
    StepEvents *ev = ctx->timing ? next_events(ctx) : nullptr;
    if (ev) cudaEventRecord(ev->ev[0], st);
    phase_inject(ctx);
    if (ev) cudaEventRecord(ev->ev[1], st);
    phase_calc_h(ctx);
    if (ev) cudaEventRecord(ev->ev[2], st);
    CK(phase_reset_j(ctx));
    if (ctx->cfg.sort_interval > 0 && ctx->steps % ctx->cfg.sort_interval == 0) {
      pdp3g_status ss = sort_all(ctx);
      if (ss != PDP3G_OK) return ss;
    }
    if (ev) cudaEventRecord(ev->ev[3], st);
    phase_particles(ctx);
    if (ev) cudaEventRecord(ev->ev[4], st);
    phase_calc_e(ctx);
    if (ev) cudaEventRecord(ev->ev[5], st);
    phase_advance(ctx);
    if (ctx->timing && ctx->events_used >= 4096) {
      pdp3g_status hs = harvest_timing(ctx);
      if (hs != PDP3G_OK) return hs;
    }
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
  phase_particles(ctx);
  CK(cudaGetLastError());
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
    std::vector<int> cell(n);
    std::vector<float> fr(n), fz(n), ur(n), uphi(n), uz(n), wf(n);
    CK(cudaMemcpyAsync(cell.data(), f.cell, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(fr.data(), f.fr, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(fz.data(), f.fz, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ur.data(), f.ur, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(uphi.data(), f.uphi, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(uz.data(), f.uz, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(wf.data(), f.w, sizeof(float) * n, cudaMemcpyDeviceToHost, st));
    if (alive) {
      if (f.alive)
        CK(cudaMemcpyAsync(alive, f.alive, n, cudaMemcpyDeviceToHost, st));
      else
        memset(alive, 1, n);
    }
    CK(cudaStreamSynchronize(st));
    const int ncz = ctx->cfg.n_grid_z - 1;
    for (size_t p = 0; p < n; p++) {
      const int i = cell[p] / ncz, k = cell[p] - (cell[p] / ncz) * ncz;
      if (r) r[p] = (i + (double)fr[p]) * ctx->dr;
      if (z) z[p] = (k + (double)fz[p]) * ctx->dz;
      const double u2 = (double)ur[p] * ur[p] + (double)uphi[p] * uphi[p] + (double)uz[p] * uz[p];
      const double c_over_g = LIGHT_SPEED / std::sqrt(1.0 + u2);
      if (vr) vr[p] = ur[p] * c_over_g;
      if (vphi) vphi[p] = uphi[p] * c_over_g;
      if (vz) vz[p] = uz[p] * c_over_g;
      if (w) w[p] = wf[p];
    }
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

pdp3g_status pdp3g_set_species(pdp3g_ctx *ctx, int32_t id, const double *r, const double *z,
                               const double *vr, const double *vphi, const double *vz,
                               const uint8_t *alive) {
  if (!ctx || id < 0 || id >= (int32_t)ctx->species.size()) return PDP3G_INVALID_ARG;
  CK(cudaSetDevice(ctx->device));
  Species &sp = ctx->species[id];
  if (sp.fp32) {
    // the cell index packs r and z: rebuild the full FP64 state, replace the
    // given arrays and convert back
    const size_t n = (size_t)sp.f32.n;
    std::vector<double> R(n), Z(n), VR(n), VP(n), VZ(n);
    pdp3g_status gs = pdp3g_get_species(ctx, id, R.data(), Z.data(), VR.data(), VP.data(),
                                        VZ.data(), nullptr, nullptr);
    if (gs != PDP3G_OK) return gs;
    if (r) memcpy(R.data(), r, n * sizeof(double));
    if (z) memcpy(Z.data(), z, n * sizeof(double));
    if (vr) memcpy(VR.data(), vr, n * sizeof(double));
    if (vphi) memcpy(VP.data(), vphi, n * sizeof(double));
    if (vz) memcpy(VZ.data(), vz, n * sizeof(double));
    gs = upload_f32(ctx, sp, (int64_t)n, R.data(), Z.data(), VR.data(), VP.data(), VZ.data());
    if (gs != PDP3G_OK) return gs;
    if (alive) {
      if (!sp.f32.alive) CK(dalloc(ctx, &sp.f32.alive, n));
      CK(cudaMemcpy(sp.f32.alive, alive, n, cudaMemcpyHostToDevice));
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

}  // extern "C"
