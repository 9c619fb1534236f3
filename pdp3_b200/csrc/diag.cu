// FP64 diagnostics: field energy, particle kinetic energy, Gauss-law
// residual.  (No upstream counterpart: the upstream loop prints none.)
//
// Every reduction is two-pass and deterministic for a given launch shape:
// each block writes its partial sums to partials[block * nv + v], then one
// block adds the partials in block order.
//
// Gauss residual at a node (i, k), on the Yee layout the upstream update
// uses (E_r at (i+1/2, k), E_z at (i, k+1/2), rho at (i, k)):
//   div E = (E_r[i][k] (i+1/2) - E_r[i-1][k] (i-1/2)) / (i dr)
//         + (E_z[i][k] - E_z[i][k-1]) / dz
//   res   = eps0 div E - (rho - rho_0)
// summed over 2 <= i <= nr-3, 2 <= k <= nz-3 where sigma == 0 (the
// absorbing layer damps E and does not conserve div E).  With the upstream
// deposition (which is charge-conserving for this div and for the upstream
// charge weighting) the FP64 step keeps it at rounding level.
#include "pdp3g_internal.cuh"

namespace pdp3g {

constexpr int RED_THREADS = 256;

template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double *partials) {
  __shared__ double sh[NV][RED_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; j++) {
    double x = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[j][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0;
    for (int w = 0; w < RED_THREADS / 32; w++) s += sh[threadIdx.x][w];
    partials[(size_t)blockIdx.x * NV + threadIdx.x] = s;
  }
}

// partials -> out[v] for v < nv, summed in block order by one block.
__global__ void k_finalize(const double *partials, int nblocks, int nv, double *out) {
  __shared__ double sh[RED_THREADS];
  for (int v = 0; v < nv; v++) {
    double s = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(size_t)b * nv + v];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[v] = sh[0];
    __syncthreads();
  }
}

// Nodes where the discrete Gauss law is conserved by the update: the node's
// divergence reads E_r at (i +- 1/2, k) and E_z at (i, k +- 1/2), stored at
// nodes (i, k), (i-1, k) and (i, k), (i, k-1); when all of them are updated
// without the absorbing layer's damping the curl-H terms cancel in the
// divergence and the charge-conserving deposition keeps the residual.
__device__ __forceinline__ bool gauss_node(const double *sigma, long long t, int nz) {
  return sigma[t] == 0.0 && sigma[t - nz] == 0.0 && sigma[t - 1] == 0.0;
}

// v0: field energy, v1: sum res^2, v2: sum rho dV
__global__ void __launch_bounds__(RED_THREADS) k_grid_diag(GridDev g, const double *rho,
                                                           const double *rho0,
                                                           double *partials) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz;
  double v[3] = {0, 0, 0};
  const long long total = (long long)nr * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nz), k = (int)(t - (long long)i * nz);
    const double vol = i == 0 ? PI * dz * dr * dr / 4. : 2.0 * PI * dz * dr * dr * i;
    const double e2 = g.er[t] * g.er[t] + g.ephi[t] * g.ephi[t] + g.ez[t] * g.ez[t];
    const double h2 = g.hr[t] * g.hr[t] + g.hphi[t] * g.hphi[t] + g.hz[t] * g.hz[t];
    v[0] += 0.5 * (EPSILON0 * e2 + MAGN_CONST * h2) * vol;
    v[2] += rho[t] * vol;
    if (i >= 2 && i <= nr - 3 && k >= 2 && k <= nz - 3 && gauss_node(g.sigma, t, nz)) {
      const double div = (g.er[t] * (i + 0.5) - g.er[t - nz] * (i - 0.5)) / (i * dr) +
                         (g.ez[t] - g.ez[t - 1]) / dz;
      const double res = EPSILON0 * div - (rho[t] - (rho0 ? rho0[t] : 0.0));
      v[1] += res * res;
    }
  }
  block_reduce_store<3>(v, partials);
}

// v0: sum rho^2 over the Gauss nodes
__global__ void __launch_bounds__(RED_THREADS) k_rho_norm(GridDev g, const double *rho,
                                                          double *partials) {
  const int nr = g.nr, nz = g.nz;
  double v[1] = {0};
  const long long total = (long long)nr * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nz), k = (int)(t - (long long)i * nz);
    if (i >= 2 && i <= nr - 3 && k >= 2 && k <= nz - 3 && gauss_node(g.sigma, t, nz))
      v[0] += rho[t] * rho[t];
  }
  block_reduce_store<1>(v, partials);
}

// v0: sum m c^2 (gamma - 1), v1: alive count (FP64 plain form)
__global__ void __launch_bounds__(RED_THREADS) k_kinetic_f64(SpeciesDev s, double *partials) {
  double v[2] = {0, 0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x) {
    if (s.alive != nullptr && !s.alive[p]) continue;
    const double v2 = s.vr[p] * s.vr[p] + s.vphi[p] * s.vphi[p] + s.vz[p] * s.vz[p];
    const double beta2 = v2 / LIGHT_SPEED_POW_2;
    const double m = s.mass * s.w[p];
    if (beta2 < 1.0) {
      // gamma - 1 = beta^2 / (sqrt(1 - beta^2) (1 + sqrt(1 - beta^2))), no cancellation
      const double sq = sqrt(1.0 - beta2);
      v[0] += m * LIGHT_SPEED_POW_2 * beta2 / (sq * (1.0 + sq));
    }
    v[1] += 1.0;
  }
  block_reduce_store<2>(v, partials);
}

int diag_blocks() { return 148 * 4; }

void launch_finalize(const double *partials, int nblocks, int nv, double *out, cudaStream_t st) {
  k_finalize<<<1, RED_THREADS, 0, st>>>(partials, nblocks, nv, out);
}

void launch_grid_diag(const GridDev &g, const double *rho, const double *rho0, double *partials,
                      double *out, cudaStream_t st) {
  const int nb = diag_blocks();
  k_grid_diag<<<nb, RED_THREADS, 0, st>>>(g, rho, rho0, partials);
  k_finalize<<<1, RED_THREADS, 0, st>>>(partials, nb, 3, out);
}

void launch_rho_norm(const GridDev &g, const double *rho, double *partials, double *out,
                     cudaStream_t st) {
  const int nb = diag_blocks();
  k_rho_norm<<<nb, RED_THREADS, 0, st>>>(g, rho, partials);
  k_finalize<<<1, RED_THREADS, 0, st>>>(partials, nb, 1, out);
}

void launch_kinetic_f64(const SpeciesDev &s, double *partials, double *out, cudaStream_t st) {
  const int nb = diag_blocks();
  k_kinetic_f64<<<nb, RED_THREADS, 0, st>>>(s, partials);
  k_finalize<<<1, RED_THREADS, 0, st>>>(partials, nb, 2, out);
}

}  // namespace pdp3g
