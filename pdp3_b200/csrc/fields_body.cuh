// Per-node Yee updates of the axisymmetric (r, phi, z) grid, shared by the
// per-run kernels (fields.cu) and the ensemble's persistent kernel.
#pragma once

#include "pdp3g_internal.cuh"

namespace pdp3g {

#define FIDX(i, k) ((size_t)(i) * (size_t)nz + (size_t)(k))

// HField::calc_field, src/hField.cpp:93-157, node (i, k) with
// i in [0, nr-1], k in [0, nz-2]: H_r for every i, H_phi and H_z for
// i <= nr-2.  H_half = H_old + dH/2 (H_z: H_old - dH/2, upstream convention).
__device__ __forceinline__ void yee_h_node(const GridDev &g, int i, int k) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const double ephi_ik = g.ephi[FIDX(i, k)];
  const double ephi_ik1 = g.ephi[FIDX(i, k + 1)];
  const double a = dt * (ephi_ik1 - ephi_ik) / (dz * MAGN_CONST);
  const double hr = g.hr[FIDX(i, k)];
  const size_t ng = (size_t)nr * nz;
  g.hrh[FIDX(i, k)] = hr + a / 2;
  if (g.hh32) g.hh32[FIDX(i, k)] = (float)(hr + a / 2);
  g.hr[FIDX(i, k)] = hr + a;
  if (i < nr - 1) {
    const double b = dt * ((g.ez[FIDX(i + 1, k)] - g.ez[FIDX(i, k)]) / dr -
                           (g.er[FIDX(i, k + 1)] - g.er[FIDX(i, k)]) / dz) / MAGN_CONST;
    const double hphi = g.hphi[FIDX(i, k)];
    g.hphih[FIDX(i, k)] = hphi + b / 2;
    if (g.hh32) g.hh32[ng + FIDX(i, k)] = (float)(hphi + b / 2);
    g.hphi[FIDX(i, k)] = hphi + b;
    const double ephi_i1k = g.ephi[FIDX(i + 1, k)];
    const double c = dt * ((ephi_i1k + ephi_ik) / (2.0 * dr * (i + 0.5)) +
                           (ephi_i1k - ephi_ik) / dr) / MAGN_CONST;
    const double hz = g.hz[FIDX(i, k)];
    g.hzh[FIDX(i, k)] = hz - c / 2;
    if (g.hh32) g.hh32[2 * ng + FIDX(i, k)] = (float)(hz - c / 2);
    g.hz[FIDX(i, k)] = hz - c;
  }
}

// EField::calc_field, src/eField.cpp:85-170 (epsilon == 1), node (i, k)
// with i in [0, nr-2], k in [0, nz-2]:
//   E_r   i in [0, nr-2], k in [1, nz-2]
//   E_phi i in [1, nr-2], k in [1, nz-2]
//   E_z   i = 0 (on-axis form, 4/dr * H_phi), k in [0, nz-2];
//         i in [1, nr-2], k in [0, nz-2] (interior form, also the k = 0 row)
__device__ __forceinline__ void yee_e_node(const GridDev &g, int i, int k) {
  const int nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const double epsx2 = 2 * 1.0 * EPSILON0;
  const double sigma_t = g.sigma[FIDX(i, k)] * dt;
  const double koef_e = (epsx2 - sigma_t) / (epsx2 + sigma_t);
  const double koef_h = 2 * dt / (epsx2 + sigma_t);
  const double hphi_ik = g.hphi[FIDX(i, k)];
  const size_t ng = (size_t)g.nr * nz;
  if (k >= 1) {
    const double v = g.er[FIDX(i, k)] * koef_e -
                     (g.jr[FIDX(i, k)] + (hphi_ik - g.hphi[FIDX(i, k - 1)]) / dz) * koef_h;
    g.er[FIDX(i, k)] = v;
    if (g.e32) g.e32[FIDX(i, k)] = (float)v;
  }
  if (i == 0) {
    const double v =
        g.ez[FIDX(i, k)] * koef_e - (g.jz[FIDX(i, k)] - 4.0 / dr * hphi_ik) * koef_h;
    g.ez[FIDX(i, k)] = v;
    if (g.e32) g.e32[2 * ng + FIDX(i, k)] = (float)v;
  } else {
    const double hphi_m = g.hphi[FIDX(i - 1, k)];
    const double v = g.ez[FIDX(i, k)] * koef_e -
                     (g.jz[FIDX(i, k)] - (hphi_ik - hphi_m) / dr -
                      (hphi_ik + hphi_m) / (2.0 * dr * i)) * koef_h;
    g.ez[FIDX(i, k)] = v;
    if (g.e32) g.e32[2 * ng + FIDX(i, k)] = (float)v;
    if (k >= 1) {
      const double w = g.ephi[FIDX(i, k)] * koef_e -
                       (g.jphi[FIDX(i, k)] - (g.hr[FIDX(i, k)] - g.hr[FIDX(i, k - 1)]) / dz +
                        (g.hz[FIDX(i, k)] - g.hz[FIDX(i - 1, k)]) / dr) * koef_h;
      g.ephi[FIDX(i, k)] = w;
      if (g.e32) g.e32[ng + FIDX(i, k)] = (float)w;
    }
  }
}

#undef FIDX

}  // namespace pdp3g
