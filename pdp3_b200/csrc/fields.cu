// Yee FDTD updates of the axisymmetric (r, phi, z) grid.
//
// Compiled with --fmad=false: the arithmetic keeps the upstream operation
// order so the FP64 result matches the CPU step bit for bit.
//
// Both kernels are HBM-bound streaming stencils (one thread per node, the
// z index fastest so warps read contiguous rows; the r-neighbour rows come
// from L2).  Algorithmic bytes per node: H update reads E (3) and H (3),
// writes H (3) and H_half (3): 96 B; E update reads E (3), H (3), J (3),
// sigma, writes E (3): 104 B.
#include "pdp3g_internal.cuh"

namespace pdp3g {

#define IDX(i, k) ((size_t)(i) * (size_t)nz + (size_t)(k))

// HField::calc_field, src/hField.cpp:93-157.  H_r is updated for
// i in [0, nr-1], H_phi and H_z for i in [0, nr-2]; k in [0, nz-2].
// H_half = H_old + dH/2 (H_z: H_old - dH/2, the upstream sign convention).
__global__ void __launch_bounds__(256) k_yee_h(GridDev g) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const long long total = (long long)nr * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1));
    const int k = (int)(t - (long long)i * (nz - 1));
    const double ephi_ik = g.ephi[IDX(i, k)];
    const double ephi_ik1 = g.ephi[IDX(i, k + 1)];
    const double a = dt * (ephi_ik1 - ephi_ik) / (dz * MAGN_CONST);
    const double hr = g.hr[IDX(i, k)];
    g.hrh[IDX(i, k)] = hr + a / 2;
    g.hr[IDX(i, k)] = hr + a;
    if (i < nr - 1) {
      const double b = dt * ((g.ez[IDX(i + 1, k)] - g.ez[IDX(i, k)]) / dr -
                             (g.er[IDX(i, k + 1)] - g.er[IDX(i, k)]) / dz) / MAGN_CONST;
      const double hphi = g.hphi[IDX(i, k)];
      g.hphih[IDX(i, k)] = hphi + b / 2;
      g.hphi[IDX(i, k)] = hphi + b;
      const double ephi_i1k = g.ephi[IDX(i + 1, k)];
      const double c = dt * ((ephi_i1k + ephi_ik) / (2.0 * dr * (i + 0.5)) +
                             (ephi_i1k - ephi_ik) / dr) / MAGN_CONST;
      const double hz = g.hz[IDX(i, k)];
      g.hzh[IDX(i, k)] = hz - c / 2;
      g.hz[IDX(i, k)] = hz - c;
    }
  }
}

// EField::calc_field, src/eField.cpp:85-170 (epsilon == 1):
//   E_r   i in [0, nr-2], k in [1, nz-2]
//   E_phi i in [1, nr-2], k in [1, nz-2]
//   E_z   i = 0 (on-axis form, 4/dr * H_phi), k in [0, nz-2];
//         i in [1, nr-2], k in [0, nz-2] (interior form, also the k = 0 row)
__global__ void __launch_bounds__(256) k_yee_e(GridDev g) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const long long total = (long long)(nr - 1) * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1));
    const int k = (int)(t - (long long)i * (nz - 1));
    const double epsx2 = 2 * 1.0 * EPSILON0;
    const double sigma_t = g.sigma[IDX(i, k)] * dt;
    const double koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);
    const double koef_h = 2 * dt / (epsx2 + sigma_t);
    const double hphi_ik = g.hphi[IDX(i, k)];
    if (k >= 1) {
      g.er[IDX(i, k)] = g.er[IDX(i, k)] * koef_e -
                        (g.jr[IDX(i, k)] + (hphi_ik - g.hphi[IDX(i, k - 1)]) / dz) * koef_h;
    }
    if (i == 0) {
      g.ez[IDX(i, k)] = g.ez[IDX(i, k)] * koef_e - (g.jz[IDX(i, k)] - 4.0 / dr * hphi_ik) * koef_h;
    } else {
      const double hphi_m = g.hphi[IDX(i - 1, k)];
      g.ez[IDX(i, k)] = g.ez[IDX(i, k)] * koef_e -
                        (g.jz[IDX(i, k)] - (hphi_ik - hphi_m) / dr -
                         (hphi_ik + hphi_m) / (2.0 * dr * i)) * koef_h;
      if (k >= 1) {
        g.ephi[IDX(i, k)] = g.ephi[IDX(i, k)] * koef_e -
                            (g.jphi[IDX(i, k)] - (g.hr[IDX(i, k)] - g.hr[IDX(i, k - 1)]) / dz +
                             (g.hz[IDX(i, k)] - g.hz[IDX(i - 1, k)]) / dr) * koef_h;
      }
    }
  }
}

static int grid_blocks(long long total) {
  long long b = (total + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

void launch_yee_h(const GridDev &g, cudaStream_t st) {
  k_yee_h<<<grid_blocks((long long)g.nr * (g.nz - 1)), 256, 0, st>>>(g);
}

void launch_yee_e(const GridDev &g, cudaStream_t st) {
  k_yee_e<<<grid_blocks((long long)(g.nr - 1) * (g.nz - 1)), 256, 0, st>>>(g);
}

}  // namespace pdp3g
