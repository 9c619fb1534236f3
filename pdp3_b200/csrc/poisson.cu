// Initial electrostatic field: PoissonDirichlet::poisson_solve
// (src/poissonDirichlet.cpp:23-98) on the device.
//
//   1. every radial row of rho gets a sine transform along z
//      (Fourier::fast_sine_transform, src/math/fourier.cpp:17-51: the odd
//      extension of length 2 n_grid_z + 2 through the radix-2 FFT of
//      Fourier::fast_fourier_alg, :93-142), one CTA per row in shared memory;
//   2. per axial mode k, the radial three-point equation is swept (the
//      upstream's alpha/beta recurrence and back substitution, one thread
//      per k; the mode constant b is evaluated on the host with its libm);
//   3. the inverse sine transform of every row of phi;
//   4. E_r = (phi_i - phi_i+1) / dr, E_z = (phi_k - phi_k+1) / dz.
//
// Compiled with --fmad=false: every step keeps the upstream's operation
// order; the FFT's twiddle factors come from CUDA's sin/cos instead of the
// host libm, so phi and E agree with the upstream's to rounding (about
// 1e-13 relative), not bit for bit.
#include "pdp3g_internal.cuh"

namespace pdp3g {

constexpr int DST_THREADS = 512;
constexpr int DST_MAX_LEN = 8192;  // 2 n_grid_z + 2: 128 KB of shared memory

// the transform of row `row` of grid a ([nr][nz]) in place
__global__ void __launch_bounds__(DST_THREADS) k_sine_transform(double *a, int nz, int len,
                                                                int log2_len, bool inverse) {
  extern __shared__ double2 sh[];
  double *row = a + (size_t)blockIdx.x * nz;
  // a_sinc: 0 at 0 and nz + 1, a[k] at k + 1, -a[k] at 2 nz - k + 1
  for (int j = threadIdx.x; j < len; j += blockDim.x) sh[j] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {
    const double v = row[k];
    sh[2 * nz - k + 1] = make_double2(-v, 0.0);
    sh[k + 1] = make_double2(v, 0.0);
  }
  __syncthreads();
  // bit-reversal permutation
  for (int k = threadIdx.x; k < len; k += blockDim.x) {
    const int j = (int)(__brev((unsigned)k) >> (32 - log2_len));
    if (k < j) {
      const double2 t = sh[k];
      sh[k] = sh[j];
      sh[j] = t;
    }
  }
  __syncthreads();
  // butterflies, n_step = 1, 2, 4, ...: W = exp(i (-PI 2 k) / (2 n_step))
  for (int n_step = 1; n_step < len; n_step *= 2) {
    for (int b = threadIdx.x; b < len / 2; b += blockDim.x) {
      const int k = b % n_step;
      const int m = (b / n_step) * 2 * n_step + k;
      const double theta = -PI * (double)2.0 * k / (n_step * 2);
      double ws, wc;
      sincos(theta, &ws, &wc);
      const double2 x = sh[m + n_step], am = sh[m];
      // W * x as the complex product (a + bi)(c + di) = (ac - bd) + (ad + bc)i
      const double tr = wc * x.x - ws * x.y, ti = wc * x.y + ws * x.x;
      sh[m] = make_double2(am.x + tr, am.y + ti);
      sh[m + n_step] = make_double2(am.x - tr, am.y - ti);
    }
    __syncthreads();
  }
  // a[k] = real(-1 / (2i) * a_sinc[k + 1]) = real((0 + 0.5i) * a_sinc[k + 1])
  for (int k = threadIdx.x; k < nz; k += blockDim.x) {
    const double2 x = sh[k + 1];
    double v = 0.0 * x.x - 0.5 * x.y;
    if (inverse) v = v * 2.0 / (nz + 1);
    row[k] = v;
  }
}

// the radial sweep of mode k (one thread per k); alpha, beta: [nr][nz]
// scratch; fi[nr-1][k] is the boundary value (set_fi_on_z: 0)
__global__ void k_poisson_sweep(const double *t, const double *b_mode, double *fi, double *alpha,
                                double *beta, int nr, int nz, double dr) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nz) return;
  const double b = b_mode[k];
  double d = dr * dr * t[k] / EPSILON0;
  alpha[(size_t)1 * nz + k] = 4. / (2. + b);
  beta[(size_t)1 * nz + k] = d / (2. + b);
  double al = alpha[(size_t)1 * nz + k], be = beta[(size_t)1 * nz + k];
  for (int i = 1; i < nr - 1; i++) {
    const double a = 1. - 1. / (2. * (i));
    const double c = 1. + 1. / (2. * (i));
    d = dr * dr * t[(size_t)i * nz + k] / EPSILON0;
    const double na = c / (b - al * a);
    const double nb = (d + be * a) / (b - al * a);
    alpha[(size_t)(i + 1) * nz + k] = na;
    beta[(size_t)(i + 1) * nz + k] = nb;
    al = na;
    be = nb;
  }
  for (int i = nr - 2; i >= 0; i--)
    fi[(size_t)i * nz + k] =
        beta[(size_t)(i + 1) * nz + k] + alpha[(size_t)(i + 1) * nz + k] * fi[(size_t)(i + 1) * nz + k];
}

// e1[i][k] = (fi[i][k] - fi[i+1][k]) / dr (i < nr-1); e3[i][k] = (fi[i][k] -
// fi[i][k+1]) / dz (k < nz-1); the last row of E_r and column of E_z keep
// their values
__global__ void k_poisson_field(const double *fi, double *er, double *ez, int nr, int nz,
                                double dr, double dz) {
  const long long total = (long long)nr * nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / nz), k = (int)(q - (long long)i * nz);
    if (i < nr - 1) er[q] = (fi[q] - fi[q + nz]) / dr;
    if (k < nz - 1) ez[q] = (fi[q] - fi[q + 1]) / dz;
  }
}

// 0 if 2 nz + 2 is a power of two the shared-memory FFT holds, else -1
int poisson_check(int nz) {
  const int len = 2 * nz + 2;
  if (len > DST_MAX_LEN || (len & (len - 1)) != 0) return -1;
  return 0;
}

cudaError_t launch_poisson(const GridDev &g, const double *rho, double *t, double *fi,
                           double *alpha, double *beta, const double *b_mode, double *er,
                           double *ez, cudaStream_t st) {
  const int nr = g.nr, nz = g.nz, len = 2 * nz + 2;
  int log2_len = 0;
  while ((1 << log2_len) < len) log2_len++;
  const size_t smem = sizeof(double2) * (size_t)len;
  cudaError_t e = cudaFuncSetAttribute(k_sine_transform,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyAsync(t, rho, sizeof(double) * (size_t)nr * nz, cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  k_sine_transform<<<nr, DST_THREADS, smem, st>>>(t, nz, len, log2_len, false);
  k_poisson_sweep<<<(nz + 127) / 128, 128, 0, st>>>(t, b_mode, fi, alpha, beta, nr, nz, g.dr);
  k_sine_transform<<<nr, DST_THREADS, smem, st>>>(fi, nz, len, log2_len, true);
  long long blocks = ((long long)nr * nz + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_poisson_field<<<(int)blocks, 256, 0, st>>>(fi, er, ez, nr, nz, g.dr, g.dz);
  return cudaGetLastError();
}

}  // namespace pdp3g
