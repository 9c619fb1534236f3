// The per-species diagnostics of LoadInitParam::dump_data on the device.
//
// TemperatureClassic (src/temperatureClassic.cpp:57-159): per cell
// (CELL_NUMBER of r and z) the sums of |v|, v_r, v_phi, v_z and the particle
// count, then T = m v_sc^2 / 2 with v_sc^2 = ((sum |v|)^2 - |sum v|^2) /
// count^2 (relativistic m c^2 (gamma - 1) at v_sc > 5e7 m/s), in
// electronvolts; empty cells give NaN (0/0), as upstream.
//
// ParticlesDensity (src/particlesDensity.cpp:45-257): each particle's
// mass_array / EL_MASS spread over the four nodes around it by ring-piece
// volumes, with the upstream's three radial branches.
//
// Compiled with --fmad=false: the per-particle and per-cell arithmetic keeps
// the upstream order; only the order of the sums (warp run sums, then FP64
// atomics) differs.
#include "pdp3g_internal.cuh"

namespace pdp3g {

constexpr double REL_LIMIT = 5e7;  // src/temperatureClassic.cpp:4-6

// acc: 5 grids [nr][nz]: sum |v|, sum v_r, sum v_phi, sum v_z, count.
// Every lane of the warp calls it (live: this lane holds a particle); runs
// of lanes in the same cell are summed in the warp (warp_run_sum_f64) and
// added with one set of FP64 atomics.  A cell outside the grid adds nothing.
__device__ __forceinline__ void temp_run_add(const GridDev &g, double *acc, bool live, int ri,
                                             int zk, double vr, double vphi, double vz) {
  const bool inside = live && (unsigned)ri < (unsigned)g.nr && (unsigned)zk < (unsigned)g.nz;
  double v[5] = {0, 0, 0, 0, 0};
  if (inside) {
    v[0] = sqrt(vr * vr + vphi * vphi + vz * vz);
    v[1] = vr;
    v[2] = vphi;
    v[3] = vz;
    v[4] = 1.0;
  }
  const int key = inside ? ri * g.nz + zk : -1;
  if (!warp_run_sum_f64<5>(key, v) || !inside) return;
  const size_t ng = (size_t)g.nr * g.nz, t = (size_t)ri * g.nz + zk;
#pragma unroll
  for (int j = 0; j < 5; j++) atomicAdd(acc + j * ng + t, v[j]);
}

// The loops below run whole warps: every lane takes part in the warp sums.
__global__ void k_temp_accum_f64(GridDev g, SpeciesDev s, double *acc) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); p0 < s.n;
       p0 += stride) {
    const long long p = p0 + (threadIdx.x & 31);
    const bool live = p < s.n;
    int ri = -1, zk = -1;
    double vr = 0, vphi = 0, vz = 0;
    if (live) {
      ri = (int)ceil(s.r[p] / g.dr) - 1;
      zk = (int)ceil(s.z[p] / g.dz) - 1;
      vr = s.vr[p];
      vphi = s.vphi[p];
      vz = s.vz[p];
    }
    temp_run_add(g, acc, live, ri, zk, vr, vphi, vz);
  }
}

// the cell-local form, read as FP64 r, z, v exactly as the species getter
// does (r = (i + f_r) dr, v = u c / sqrt(1 + u^2)), then CELL_NUMBER as above
__global__ void k_temp_accum_f32(GridDev g, SpeciesF32 s, double *acc) {
  const int ncz = g.nz - 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); p0 < s.n;
       p0 += stride) {
    const long long p = p0 + (threadIdx.x & 31);
    const bool live = p < s.n;
    int ri = -1, zk = -1;
    double vr = 0, vphi = 0, vz = 0;
    if (live) {
      const int c = s.cell[p];
      const int i = c / ncz, k = c - i * ncz;
      const double r = (i + (double)s.fr[p]) * g.dr, z = (k + (double)s.fz[p]) * g.dz;
      ri = (int)ceil(r / g.dr) - 1;
      zk = (int)ceil(z / g.dz) - 1;
      const double ur = s.ur[p], up = s.uphi[p], uz = s.uz[p];
      const double gc = LIGHT_SPEED / sqrt(1.0 + (ur * ur + up * up + uz * uz));
      vr = ur * gc;
      vphi = up * gc;
      vz = uz * gc;
    }
    temp_run_add(g, acc, live, ri, zk, vr, vphi, vz);
  }
}

// TemperatureClassic::normalize over r < nr-1, z < nz-1 (others left 0)
__global__ void k_temp_normalize(GridDev g, const double *acc, double mass, double charge,
                                 double *t_out) {
  const int nr = g.nr, nz = g.nz;
  const size_t ng = (size_t)nr * nz;
  const long long total = (long long)(nr - 1) * (nz - 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(q / (nz - 1)), z = (int)(q - (long long)r * (nz - 1));
    const size_t t = (size_t)r * nz + z;
    const double sum = acc[t], vr = acc[ng + t], vp = acc[2 * ng + t], vz = acc[3 * ng + t];
    const double cnt = acc[4 * ng + t];
    const double v_vec_sum_2 = vr * vr + vp * vp + vz * vz;
    const double v_sc_sum_2 = (sum * sum - v_vec_sum_2) / (cnt * cnt);
    double tv;
    if (v_sc_sum_2 < REL_LIMIT * REL_LIMIT) {
      tv = mass * v_sc_sum_2 / 2;
    } else {
      // lib::get_gamma (src/lib.cpp:45-70): beta == 1 gives 1e100; beta > 1
      // is an upstream exit, gamma 1 here
      const double beta = v_sc_sum_2 / LIGHT_SPEED_POW_2;
      double gamma = beta > 1 ? 1.0 : 1 / sqrt(1.0 - beta);
      if (isinf(gamma)) gamma = 1e100;
      tv = mass * LIGHT_SPEED_POW_2 * (gamma - 1);
    }
    t_out[t] = tv / fabs(charge);
  }
}

// ParticlesDensity::calc_density for one particle (r, z, mass_array m):
// the node block (ri, zk) and the 4 values (nodes ri..ri+1 x zk..zk+1)
__device__ __forceinline__ void density_values(const GridDev &g, double r, double z, double m,
                                               int &ri, int &zk, double (&out)[4]) {
  const double dr = g.dr, dz = g.dz;
  ri = (int)ceil(r / dr) - 1;
  zk = (int)ceil(z / dz) - 1;
  const bool outer = r > dr, inner = !outer && r <= dr / 2.;
  if (inner) ri = 0;
  const double rif = (double)ri;
  const double dz1 = (zk + 0.5) * dz - (z - 0.5 * dz);
  const double dz2 = (z + 0.5 * dz) - (zk + 0.5) * dz;
  const double r1 = inner ? 0. : r - 0.5 * dr;
  const double r2 = (rif + 0.5) * dr;
  const double r3 = r + 0.5 * dr;
  const double v0 = inner ? PI * dz * (2. * r * r + dr * dr / 2.) : 2. * PI * dz * dr * r;
  const double ro_p = m / EL_MASS / v0;
  const double v1 = outer ? PI * dz * dr * dr * 2.0 * rif : PI * dz * dr * dr / 4.;
  const double v2 = PI * dz * dr * dr * 2.0 * (rif + 1);
  double val[4];
  if (inner) {
    val[0] = PI * dz1 * (dr * dr / 2. - r * dr + r * r) / v1;
    val[2] = PI * dz2 * (dr * dr / 2. - r * dr + r * r) / v1;
  } else {
    val[0] = PI * dz1 * (r2 * r2 - r1 * r1) / v1;
    val[2] = PI * dz2 * (r2 * r2 - r1 * r1) / v1;
  }
  val[1] = PI * dz1 * (r3 * r3 - r2 * r2) / v2;
  val[3] = PI * dz2 * (r3 * r3 - r2 * r2) / v2;
#pragma unroll
  for (int j = 0; j < 4; j++) out[j] = ro_p * val[j];
}

// out += the density values of a warp's particles, one run sum per node
// block; nodes outside the grid are skipped (no flag, as upstream's bounds
// test); a block that reaches outside the grid is not merged with others.
__device__ __forceinline__ void density_run_add(const GridDev &g, double *out, bool live, int ri,
                                                int zk, double (&v)[4]) {
  const bool inside = ri >= 0 && zk >= 0 && ri <= g.nr - 2 && zk <= g.nz - 2;
  const int key = !live ? -1 : (inside ? ri * g.nz + zk : -2 - (int)(threadIdx.x & 31));
  if (!warp_run_sum_f64<4>(key, v) || !live) return;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int i = ri + (j & 1), k = zk + (j >> 1);
    if ((unsigned)i < (unsigned)g.nr && (unsigned)k < (unsigned)g.nz)
      atomicAdd(out + (size_t)i * g.nz + k, v[j]);
  }
}

__global__ void k_density_f64(GridDev g, SpeciesDev s, double *out) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); p0 < s.n;
       p0 += stride) {
    const long long p = p0 + (threadIdx.x & 31);
    const bool live = p < s.n;
    int ri = 0, zk = 0;
    double v[4] = {0, 0, 0, 0};
    if (live) density_values(g, s.r[p], s.z[p], s.mass * s.w[p], ri, zk, v);
    density_run_add(g, out, live, ri, zk, v);
  }
}

__global__ void k_density_f32(GridDev g, SpeciesF32 s, double mass, double *out) {
  const int ncz = g.nz - 1;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); p0 < s.n;
       p0 += stride) {
    const long long p = p0 + (threadIdx.x & 31);
    const bool live = p < s.n;
    int ri = 0, zk = 0;
    double v[4] = {0, 0, 0, 0};
    if (live) {
      const int c = s.cell[p];
      const int i = c / ncz, k = c - i * ncz;
      density_values(g, (i + (double)s.fr[p]) * g.dr, (k + (double)s.fz[p]) * g.dz,
                     mass * (double)s.w[p], ri, zk, v);
    }
    density_run_add(g, out, live, ri, zk, v);
  }
}

static int blocks_of(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

void launch_temperature_f64(const GridDev &g, const SpeciesDev &s, double *acc, cudaStream_t st) {
  if (s.n > 0) k_temp_accum_f64<<<blocks_of(s.n), 256, 0, st>>>(g, s, acc);
}

void launch_temperature_f32(const GridDev &g, const SpeciesF32 &s, double *acc, cudaStream_t st) {
  if (s.n > 0) k_temp_accum_f32<<<blocks_of(s.n), 256, 0, st>>>(g, s, acc);
}

void launch_temperature_normalize(const GridDev &g, const double *acc, double mass, double charge,
                                  double *t_out, cudaStream_t st) {
  k_temp_normalize<<<blocks_of((long long)(g.nr - 1) * (g.nz - 1)), 256, 0, st>>>(g, acc, mass,
                                                                                 charge, t_out);
}

void launch_density_f64(const GridDev &g, const SpeciesDev &s, double *out, cudaStream_t st) {
  if (s.n > 0) k_density_f64<<<blocks_of(s.n), 256, 0, st>>>(g, s, out);
}

void launch_density_f32(const GridDev &g, const SpeciesF32 &s, double mass, double *out,
                        cudaStream_t st) {
  if (s.n > 0) k_density_f32<<<blocks_of(s.n), 256, 0, st>>>(g, s, mass, out);
}

}  // namespace pdp3g
