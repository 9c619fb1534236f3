// Initial state of a plasma species on the device: LoadInitParam::
// init_particles (src/loadInitParam.cpp:134-166) = the Particles constructor,
// Particles::load_cylindrical_spatial_distribution (src/particles.cpp:
// 278-331) and Particles::velocity_distribution (src/particles.cpp:228-276)
// with its Maxwell-Juttner sampler (src/math/maxwellJuttner.cpp:314-399) and
// the TESTMODE random_reverse sequences (src/math/rand.cpp:37-53).
//
// Positions and weights are the upstream's bit for bit: random_reverse with
// host-computed pow(p, -k) terms, IEEE arithmetic in the upstream order
// (--fmad=false), and the volume sum v_sum added sequentially in slot order.
// Velocities pass through log, exp and pow: CUDA's double functions differ
// from the host libm by an ulp or two, and the sampler's inverse-CDF tables
// (mj_tables.h) are computed from their definition, so velocities agree with
// the upstream's to about 1e-13 relative rather than bit for bit.
#include "pdp3g_internal.cuh"
#include "mj_tables.h"

namespace pdp3g {

// inv_pow[p * RR_ORDERS + k] = pow((double)p, -k) from the host libm, p < RR_BASES
constexpr int RR_BASES = 16, RR_ORDERS = 40;
constexpr long long MJ_MAX_TRIES = 100000;  // rejection-loop bound per particle

// random_reverse(x, POWER) for a tabulated base (a compile-time divisor)
template <int POWER>
__device__ __forceinline__ double rr_tab(unsigned x, const double *inv_pow) {
  static_assert(POWER >= 2 && POWER < RR_BASES, "tabulated bases only");
  int v = (int)x;
  double r = 0;
  int order = 1;
  while (v >= 1 && order < RR_ORDERS) {
    const int ost = v % POWER;
    r = r + (double)ost * inv_pow[POWER * RR_ORDERS + order];
    v = (v - ost) / POWER;
    order = order + 1;
  }
  return r;
}

// random_reverse(x, power) for any base: pow(power, -k) as the correctly
// rounded reciprocal of the exact power^k (exact while power^k < 2^53)
__device__ __forceinline__ double rr_any(unsigned x, unsigned power) {
  long long v = (int)x;
  double r = 0, pk = 1;
  while (v >= 1) {
    const long long ost = v % power;
    pk = pk * (double)power;
    r = r + (double)ost * (1.0 / pk);
    v = (v - ost) / power;
  }
  return r;
}

struct InitSpatial {
  unsigned n;             // number of macroparticles
  double r_size, z_size, dr, dz;
  double n1, dn, n1_sq, dn_sq;  // densities; pow(n1, 2) and pow(dn, 2) from the host
  double left;            // left_plasma_boundary
};

// load_cylindrical_spatial_distribution, first loop (positions, volumes)
__global__ void k_init_positions(InitSpatial p, const double *inv_pow, double *r_out,
                                 double *z_out, double *vol_out) {
  for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < p.n; n += gridDim.x * blockDim.x) {
    const double rand_r = rr_tab<13>(n, inv_pow);
    const double rand_z = rr_tab<11>(p.n - 1 - n, inv_pow);
    const double r = (p.r_size - p.dr) * rand_r + p.dr / 2;
    double z;
    if (p.dn == 0)
      z = rand_z * (p.z_size - p.dz) + p.left + p.dz / 2;
    else
      z = (p.z_size - p.left - p.dz) / p.dn *
              (sqrt(p.n1_sq + rand_z * (2 * p.n1 * p.dn + p.dn_sq)) - p.n1) +
          p.left + p.dz / 2;
    r_out[n] = r;
    z_out[n] = z;
    vol_out[n] = 2 * PI * r * p.dr * p.dz;
  }
}

// v_sum += ... in slot order, by one thread so the rounding is the
// upstream's.  The block streams the terms through a double-buffered
// shared-memory tile (coalesced loads by all threads) while thread 0 adds the
// previous tile from shared memory, so the sum runs at the FP64 add latency.
constexpr int SUM_THREADS = 256, SUM_TILE = 2048;  // 2 x 16 KB of shared memory

__global__ void __launch_bounds__(SUM_THREADS) k_sequential_sum(const double *vol, unsigned n,
                                                                double *out) {
  __shared__ double tile[2][SUM_TILE];
  const unsigned ntiles = (n + SUM_TILE - 1) / SUM_TILE;
  double s = 0;
  auto load = [&](unsigned t, int buf) {
    const unsigned base = t * SUM_TILE;
    for (int j = threadIdx.x; j < SUM_TILE; j += SUM_THREADS)
      if (base + j < n) tile[buf][j] = __ldg(vol + base + j);
  };
  if (ntiles > 0) load(0, 0);
  __syncthreads();
  for (unsigned t = 0; t < ntiles; t++) {
    const int buf = t & 1;
    if (t + 1 < ntiles) load(t + 1, buf ^ 1);
    if (threadIdx.x == 0) {
      const unsigned base = t * SUM_TILE;
      const int cnt = (n - base < (unsigned)SUM_TILE) ? (int)(n - base) : SUM_TILE;
      int j = 0;
      for (; j + 8 <= cnt; j += 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) v[q] = tile[buf][j + q];
#pragma unroll
        for (int q = 0; q < 8; q++) s += v[q];
      }
      for (; j < cnt; j++) s += tile[buf][j];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s;
}

// second loop: n_per_macro = n_per_macro_avg * norm (the weight w; the
// upstream's charge_array = charge * w, mass_array = mass * w)
__global__ void k_init_weights(InitSpatial p, const double *r_in, const double *v_sum,
                               double n_per_macro_avg, double *w_out) {
  const double v_avg = *v_sum / p.n;
  for (unsigned n = blockIdx.x * blockDim.x + threadIdx.x; n < p.n; n += gridDim.x * blockDim.x) {
    const double r = r_in[n];
    double norm;
    if (r > p.dr / 2)
      norm = 2 * PI * r * p.dr * p.dz / v_avg;
    else
      norm = PI * (r * r + r * p.dr + p.dr * p.dr / 4) * p.dz / v_avg;
    w_out[n] = n_per_macro_avg * norm;
  }
}

struct InitVelocity {
  unsigned n;
  double temperature;  // eV, as the upstream passes it to the sampler
  double mass;         // SI, one physical particle
  double h0;           // -1/T + log(1 + 1/T + 1/(2 T^2)) from the host libm
  double mb_small;     // 3 sqrt(pi) / 4 from the host libm
};

// math::maxwell_juttner::maxwellJuttner for particle i (energy, eV units of
// the upstream), NaN where the upstream's own branches give NaN
__device__ double mj_energy(const InitVelocity &p, unsigned i, const double *inv_pow,
                            unsigned *err) {
  const double T = p.temperature;
  if (T < 0.1) {
    // classical: one draw, random_reverse(npoints - i, 9 + i)
    const double U = rr_any(p.n - i, 9u + i);
    const double lnlnU = log(-log(U));
    double invF;
    if (lnlnU > 2.) {
      invF = p.mb_small * pow(U, 2. / 3.);
    } else if (lnlnU < -19.) {
      invF = 1.;
    } else {
      const double I = (lnlnU + 19.) * (999. / (2. + 19.));
      unsigned index = (unsigned)I;
      if (index > 998) index = 998;  // I == 999 exactly: the upstream reads past its table
      const double rem = I - (double)index;
      invF = exp(LN_INV_F[index] + rem * (LN_INV_F[index + 1] - LN_INV_F[index]));
    }
    return T * invF;
  }
  // relativistic: rejection on beta
  double gamma, U;
  long long k = 0;
  do {
    U = rr_tab<13>(p.n + i - (unsigned)k, inv_pow);
    const double lnU = log(-log(1. - U) - p.h0);
    double invH;
    if (lnU < -26.) {
      invH = pow(-6. * U, 1. / 3.);
    } else if (lnU > 12.) {
      invH = -U + 11.35 * pow(-U, 0.06);
    } else {
      const double I = (lnU + 30.) * (999. / (12. + 30.));
      unsigned index = (unsigned)I;
      if (index > 998) index = 998;
      const double rem = I - (double)index;
      invH = exp(LN_INV_H[index] + rem * (LN_INV_H[index + 1] - LN_INV_H[index]));
    }
    gamma = T * invH;
    U = rr_tab<15>(p.n - i + (unsigned)k, inv_pow);
    k++;
    if (k >= MJ_MAX_TRIES) {
      atomicOr(err, 1u);
      break;
    }
  } while (U >= sqrt(1. - 1. / (gamma * gamma)));
  return gamma - 1.;
}

// velocity_distribution: therm_vel_el = 0.74 sqrt(2 e E / m), signs and
// magnitudes from random_reverse(p, 3..8), then v *= get_gamma_inv(v^2)
__global__ void k_init_velocities(InitVelocity p, const double *inv_pow, double *vr,
                                  double *vphi, double *vz, unsigned *err) {
  for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += gridDim.x * blockDim.x) {
    const double energy = mj_energy(p, i, inv_pow, err);
    double therm = sqrt(2 * EL_CHARGE * energy / p.mass);
    therm *= 0.74;
    double rnd0 = rr_tab<3>(i, inv_pow), rnd1 = rr_tab<5>(i, inv_pow), rnd2 = rr_tab<7>(i, inv_pow);
    const double k0 = rr_tab<4>(i, inv_pow), k1 = rr_tab<6>(i, inv_pow), k2 = rr_tab<8>(i, inv_pow);
    if (k0 > 0.5) rnd0 = -rnd0;
    if (k1 > 0.5) rnd1 = -rnd1;
    if (k2 > 0.5) rnd2 = -rnd2;
    double v0 = rnd0 * therm, v1 = rnd1 * therm, v2 = rnd2 * therm;
    // lib::get_gamma_inv, src/lib.cpp:72-80: (1 + v^2/c^2)^(-1/2)
    v0 *= 1.0 / sqrt(1.0 + v0 * v0 / LIGHT_SPEED_POW_2);
    v1 *= 1.0 / sqrt(1.0 + v1 * v1 / LIGHT_SPEED_POW_2);
    v2 *= 1.0 / sqrt(1.0 + v2 * v2 / LIGHT_SPEED_POW_2);
    vr[i] = v0;
    vphi[i] = v1;
    vz[i] = v2;
  }
}

static int init_blocks(unsigned n) {
  long long b = ((long long)n + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

void launch_init_species(unsigned n, double r_size, double z_size, double dr, double dz,
                         double n1, double n2, double left, double temperature, double mass,
                         const double *inv_pow, double *r, double *z, double *vr, double *vphi,
                         double *vz, double *w, double *scratch_vol, double *d_sum, unsigned *err,
                         cudaStream_t st) {
  InitSpatial sp;
  sp.n = n;
  sp.r_size = r_size;
  sp.z_size = z_size;
  sp.dr = dr;
  sp.dz = dz;
  sp.n1 = n1;
  sp.dn = n2 - n1;
  sp.n1_sq = std::pow(n1, 2);
  sp.dn_sq = std::pow(sp.dn, 2);
  sp.left = left;
  const int blocks = init_blocks(n);
  k_init_positions<<<blocks, 256, 0, st>>>(sp, inv_pow, r, z, scratch_vol);
  k_sequential_sum<<<1, SUM_THREADS, 0, st>>>(scratch_vol, n, d_sum);
  // N_total = (n1 + n2) / 2 * PI * r_size^2 * z_size; n_per_macro_avg = N_total / number
  const double n_total = (n1 + n2) / 2 * PI * r_size * r_size * z_size;
  const double n_per_macro_avg = n_total / n;
  k_init_weights<<<blocks, 256, 0, st>>>(sp, r, d_sum, n_per_macro_avg, w);
  InitVelocity vp;
  vp.n = n;
  vp.temperature = temperature;
  vp.mass = mass;
  const double inv_t = 1. / temperature;
  vp.h0 = -inv_t + std::log(1. + inv_t + 0.5 * inv_t * inv_t);
  vp.mb_small = 3. * std::sqrt(M_PI) / 4.;
  k_init_velocities<<<blocks, 256, 0, st>>>(vp, inv_pow, vr, vphi, vz, err);
}

// pow((double)p, -k) for p < RR_BASES, k < RR_ORDERS on the host libm
void init_inv_pow_table(double *host) {
  for (int p = 0; p < RR_BASES; p++)
    for (int k = 0; k < RR_ORDERS; k++)
      host[p * RR_ORDERS + k] = (p >= 2) ? std::pow((double)p, -k) : 0.0;
}

int init_inv_pow_count() { return RR_BASES * RR_ORDERS; }

}  // namespace pdp3g
