// Adjoint (vector-Jacobian product) of the FP32 cell-local PDP3 step.
//
// Reverse of one step s, given the adjoints of the state after it
// (lE, lH: FP64 grids; la, lb, lu: FP32 per particle):
//   1  E update   E' = ke E - kh (J + curl H')   (src/eField.cpp:85-170)
//        lJ = -kh lE',  lH' += curl^T(-kh lE'),  then lE = ke lE'
//   2  particles  (adjoint_particle.cuh reverse on each particle's tape,
//        recomputed from the stored post-injection state of step s)
//        la/lb/lu updated in place, lw += ..., lE += gather^T, lHh += gather^T
//   3  injection  slots injected at step s: their z and u_z were set from the
//        beam velocity, so lb/luz go to d/dv_beam and are then cleared
//   4  H update   H' = H + a(E), Hh = H + a(E)/2    (src/hField.cpp:93-157)
//        lE += a^T(lH' + lHh/2),  lH = lH' + lHh
// Stencil transposes scatter with FP64 atomics.
#include "adjoint_particle.cuh"
#include "pdp3g_internal.cuh"

namespace pdp3g {

#define AIDX(i, k) ((size_t)(i) * (size_t)nz + (size_t)(k))


// step 1a: lJ and the curl^T part into lH (reads lE)
__global__ void k_adj_e1(GridDev g, AdjGrids A) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const long long total = (long long)(nr - 1) * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1)), k = (int)(t - (long long)i * (nz - 1));
    const double epsx2 = 2 * 1.0 * EPSILON0;
    const double sigma_t = g.sigma[AIDX(i, k)] * dt;
    const double kh = 2 * dt / (epsx2 + sigma_t);
    if (k >= 1) {  // E_r
      const double gr = -kh * A.lEr[AIDX(i, k)];
      A.lJr[AIDX(i, k)] = gr;
      atomicAdd(&A.lHphi[AIDX(i, k)], gr / dz);
      atomicAdd(&A.lHphi[AIDX(i, k - 1)], -gr / dz);
    }
    if (i == 0) {  // E_z on axis
      const double gz = -kh * A.lEz[AIDX(i, k)];
      A.lJz[AIDX(i, k)] = gz;
      atomicAdd(&A.lHphi[AIDX(i, k)], -4.0 * gz / dr);
    } else {
      const double gz = -kh * A.lEz[AIDX(i, k)];
      A.lJz[AIDX(i, k)] = gz;
      atomicAdd(&A.lHphi[AIDX(i, k)], gz * (-1.0 / dr - 1.0 / (2.0 * dr * i)));
      atomicAdd(&A.lHphi[AIDX(i - 1, k)], gz * (1.0 / dr - 1.0 / (2.0 * dr * i)));
      if (k >= 1) {  // E_phi
        const double gp = -kh * A.lEphi[AIDX(i, k)];
        A.lJphi[AIDX(i, k)] = gp;
        atomicAdd(&A.lHr[AIDX(i, k)], -gp / dz);
        atomicAdd(&A.lHr[AIDX(i, k - 1)], gp / dz);
        atomicAdd(&A.lHz[AIDX(i, k)], gp / dr);
        atomicAdd(&A.lHz[AIDX(i - 1, k)], -gp / dr);
      }
    }
  }
}

// step 1b: lE = ke lE on the updated nodes
__global__ void k_adj_e2(GridDev g, AdjGrids A) {
  const int nr = g.nr, nz = g.nz;
  const double dt = g.dt;
  const long long total = (long long)(nr - 1) * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1)), k = (int)(t - (long long)i * (nz - 1));
    const double epsx2 = 2 * 1.0 * EPSILON0;
    const double sigma_t = g.sigma[AIDX(i, k)] * dt;
    const double ke = (epsx2 - sigma_t) / (epsx2 + sigma_t);
    if (k >= 1) A.lEr[AIDX(i, k)] *= ke;
    A.lEz[AIDX(i, k)] *= ke;
    if (i >= 1 && k >= 1) A.lEphi[AIDX(i, k)] *= ke;
  }
}

// step 4a: lE += a^T (lH + lHh/2)
__global__ void k_adj_h1(GridDev g, AdjGrids A) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const long long total = (long long)nr * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1)), k = (int)(t - (long long)i * (nz - 1));
    const double la = A.lHr[AIDX(i, k)] + 0.5 * A.lHhr[AIDX(i, k)];
    const double ca = dt / (dz * MAGN_CONST);
    atomicAdd(&A.lEphi[AIDX(i, k + 1)], la * ca);
    atomicAdd(&A.lEphi[AIDX(i, k)], -la * ca);
    if (i < nr - 1) {
      const double lb = A.lHphi[AIDX(i, k)] + 0.5 * A.lHhphi[AIDX(i, k)];
      atomicAdd(&A.lEz[AIDX(i + 1, k)], lb * dt / (dr * MAGN_CONST));
      atomicAdd(&A.lEz[AIDX(i, k)], -lb * dt / (dr * MAGN_CONST));
      atomicAdd(&A.lEr[AIDX(i, k + 1)], -lb * dt / (dz * MAGN_CONST));
      atomicAdd(&A.lEr[AIDX(i, k)], lb * dt / (dz * MAGN_CONST));
      // H_z -= c, Hh_z = H_z - c/2
      const double lc = -(A.lHz[AIDX(i, k)] + 0.5 * A.lHhz[AIDX(i, k)]);
      const double p = 1.0 / (2.0 * dr * (i + 0.5));
      atomicAdd(&A.lEphi[AIDX(i + 1, k)], lc * dt * (p + 1.0 / dr) / MAGN_CONST);
      atomicAdd(&A.lEphi[AIDX(i, k)], lc * dt * (p - 1.0 / dr) / MAGN_CONST);
    }
  }
}

// step 4b: lH += lHh on the updated nodes, lHh = 0
__global__ void k_adj_h2(GridDev g, AdjGrids A) {
  const int nr = g.nr, nz = g.nz;
  const long long total = (long long)nr * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nz), k = (int)(t - (long long)i * nz);
    if (k <= nz - 2) {
      A.lHr[t] += A.lHhr[t];
      if (i <= nr - 2) {
        A.lHphi[t] += A.lHhphi[t];
        A.lHz[t] += A.lHhz[t];
      }
    }
    A.lHhr[t] = 0.0;
    A.lHhphi[t] = 0.0;
    A.lHhz[t] = 0.0;
  }
}


__device__ __forceinline__ float node_val(const GridDev &g, const double *f, int i, int k) {
  return (float)f[(size_t)i * g.nz + k];
}

__device__ __forceinline__ float lget(const GridDev &g, const double *f, int i, int k) {
  if ((unsigned)i >= (unsigned)g.nr || (unsigned)k >= (unsigned)g.nz) return 0.0f;
  return (float)f[(size_t)i * g.nz + k];
}

__device__ __forceinline__ void ladd(const GridDev &g, double *f, int i, int k, float v) {
  if (v == 0.0f || (unsigned)i >= (unsigned)g.nr || (unsigned)k >= (unsigned)g.nz) return;
  atomicAdd(f + (size_t)i * g.nz + k, (double)v);
}

// step 2: particles.  Es = E of step s, Hh = H half-time of step s.
__global__ void __launch_bounds__(128) k_adj_particles(GridDev g, const double *E3,
                                                      const double *Hh3, AdjSpeciesDev S,
                                                      AdjGrids A, int face) {
  const int ncz = g.nz - 1;
  const size_t ng = (size_t)g.nr * g.nz;
  adj::Consts<float> C;
  C.ke = S.st.ke;
  C.kb = S.st.kb;
  C.cr = S.st.cr;
  C.cz = S.st.cz;
  C.kphi = S.st.kphi;
  C.kz = S.st.kz;
  C.kr = S.st.kr;
  C.nr = g.nr;
  C.nz = g.nz;
  C.bunch = S.st.kind == KIND_BUNCH;
  C.face = face;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < S.st.n;
       p += (long long)gridDim.x * blockDim.x) {
    if (S.st.alive != nullptr && !S.st.alive[p]) continue;
    adj::Tape<float> tp;
    const int c = S.st.cell[p];
    if (c < 0 || c >= (g.nr - 1) * ncz) continue;  // flagged by the forward step
    tp.i = c / ncz;
    tp.k = c - tp.i * ncz;
    tp.a = S.st.fr[p];
    tp.b = S.st.fz[p];
    tp.u[0] = S.st.ur[p];
    tp.u[1] = S.st.uphi[p];
    tp.u[2] = S.st.uz[p];
    tp.w = S.st.w[p];
    adj::gather_weights(tp);
    const double *fE[3] = {E3, E3 + ng, E3 + 2 * ng}, *fH[3] = {Hh3, Hh3 + ng, Hh3 + 2 * ng};
    int ri[2][3], zi[2][3];
    for (int fld = 0; fld < 2; fld++)
      for (int cc = 0; cc < 3; cc++) {
        int ir = adj::comp_rhalf(fld, cc) ? tp.ir_h : tp.i;
        int kz = adj::comp_zhalf(fld, cc) ? tp.kz_h : tp.k;
        ir = min(ir, g.nr - 2);
        kz = min(kz, g.nz - 2);
        ri[fld][cc] = ir;
        zi[fld][cc] = kz;
        const double *f = fld == 0 ? fE[cc] : fH[cc];
        float *dst = fld == 0 ? tp.fe[cc] : tp.fh[cc];
        dst[0] = node_val(g, f, ir, kz);
        dst[1] = node_val(g, f, ir + 1, kz);
        dst[2] = node_val(g, f, ir, kz + 1);
        dst[3] = node_val(g, f, ir + 1, kz + 1);
      }
    adj::forward(C, tp);
    float l_jphi[4] = {lget(g, A.lJphi, tp.i1, tp.k1), lget(g, A.lJphi, tp.i1 + 1, tp.k1),
                       lget(g, A.lJphi, tp.i1, tp.k1 + 1), lget(g, A.lJphi, tp.i1 + 1, tp.k1 + 1)};
    float l_piece[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
    if (tp.path_ok)
      for (int q = 0; q <= tp.np; q++) {
        const int ci = tp.pc_i[q], ck = tp.pc_k[q];
        l_piece[q][0] = lget(g, A.lJz, ci, ck);
        l_piece[q][1] = lget(g, A.lJz, ci + 1, ck);
        l_piece[q][2] = lget(g, A.lJr, ci, ck);
        l_piece[q][3] = lget(g, A.lJr, ci, ck + 1);
      }
    const float l_uout[3] = {S.lur[p], S.luphi[p], S.luz[p]};
    float l_a, l_b, l_u[3], l_w, l_fe[3][4], l_fh[3][4];
    adj::reverse(C, tp, S.la[p], S.lb[p], l_uout, l_jphi, l_piece, l_a, l_b, l_u, l_w, l_fe,
                 l_fh);
    S.la[p] = l_a;
    S.lb[p] = l_b;
    S.lur[p] = l_u[0];
    S.luphi[p] = l_u[1];
    S.luz[p] = l_u[2];
    S.lw[p] += (double)l_w;
    double *lEs[3] = {A.lEr, A.lEphi, A.lEz}, *lHs[3] = {A.lHhr, A.lHhphi, A.lHhz};
    for (int cc = 0; cc < 3; cc++) {
      for (int fld = 0; fld < 2; fld++) {
        const int ir = ri[fld][cc], kz = zi[fld][cc];
        double *dst = fld == 0 ? lEs[cc] : lHs[cc];
        const float *lv = fld == 0 ? l_fe[cc] : l_fh[cc];
        ladd(g, dst, ir, kz, lv[0]);
        ladd(g, dst, ir + 1, kz, lv[1]);
        ladd(g, dst, ir, kz + 1, lv[2]);
        ladd(g, dst, ir + 1, kz + 1, lv[3]);
      }
    }
  }
}

// step 3: injected slots [start, start+count): z = dl rr + dz/2 with
// dl = v dt and u_z = gamma(v) v / c.  Adds their d/dv into *lv and clears
// lb, luz (the values they replaced had no influence).
__global__ void k_adj_inject(AdjSpeciesDev S, long long start, long long count, double dt,
                             double dz, double velocity, const double *inv_pow11, double *lv) {
  double acc = 0;
  const double beta2 = velocity * velocity / LIGHT_SPEED_POW_2;
  const double duz_dv = 1.0 / (LIGHT_SPEED * pow(1.0 - beta2, 1.5));
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < count;
       j += (long long)gridDim.x * blockDim.x) {
    const long long idx = start + j;
    if (idx >= S.st.n) continue;
    int int_vel = (int)floor((double)(unsigned)idx);
    double ost = 0, rr = 0;
    int order = 1;
    while (int_vel >= 1 && order < 40) {
      ost = int_vel % 11;
      rr = rr + ost * inv_pow11[order];
      int_vel = (int)((int_vel - ost) / 11);
      order = order + 1;
    }
    acc += (double)S.lb[idx] * (dt * rr / dz) + (double)S.luz[idx] * duz_dv;
    S.lb[idx] = 0.0f;
    S.luz[idx] = 0.0f;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(lv, acc);
}

// loss = sum over the probe nodes of E_z^2 V (node volume); seeds lE_z = 2 E_z V
__global__ void k_adj_seed(GridDev g, AdjGrids A, int r0, int r1, int z0, int z1,
                           double *loss) {
  const int nz = g.nz;
  const double dr = g.dr, dz = g.dz;
  const long long w = (long long)(z1 - z0), total = (long long)(r1 - r0) * w;
  double acc = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = r0 + (int)(t / w), k = z0 + (int)(t - (t / w) * w);
    const double vol = i == 0 ? PI * dz * dr * dr / 4. : 2.0 * PI * dz * dr * dr * i;
    const double ez = g.ez[AIDX(i, k)];
    acc += ez * ez * vol;
    A.lEz[AIDX(i, k)] = 2.0 * ez * vol;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

static int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

void adj_launch_e(const GridDev &g, const AdjGrids &A, cudaStream_t st) {
  const long long n = (long long)(g.nr - 1) * (g.nz - 1);
  k_adj_e1<<<blocks_for(n, 256), 256, 0, st>>>(g, A);
  k_adj_e2<<<blocks_for(n, 256), 256, 0, st>>>(g, A);
}

void adj_launch_h(const GridDev &g, const AdjGrids &A, cudaStream_t st) {
  k_adj_h1<<<blocks_for((long long)g.nr * (g.nz - 1), 256), 256, 0, st>>>(g, A);
  k_adj_h2<<<blocks_for((long long)g.nr * g.nz, 256), 256, 0, st>>>(g, A);
}

void adj_launch_particles(const GridDev &g, const double *E3, const double *Hh3,
                          const AdjSpeciesDev &S, const AdjGrids &A, int face, cudaStream_t st) {
  if (S.st.n <= 0) return;
  k_adj_particles<<<blocks_for(S.st.n, 128), 128, 0, st>>>(g, E3, Hh3, S, A, face);
}

void adj_launch_inject(const AdjSpeciesDev &S, long long start, long long count, double dt,
                       double dz, double velocity, const double *inv_pow11, double *lv,
                       cudaStream_t st) {
  if (count <= 0) return;
  k_adj_inject<<<blocks_for(count, 256), 256, 0, st>>>(S, start, count, dt, dz, velocity,
                                                        inv_pow11, lv);
}

void adj_launch_seed(const GridDev &g, const AdjGrids &A, int r0, int r1, int z0, int z1,
                     double *loss, cudaStream_t st) {
  const long long n = (long long)(r1 - r0) * (z1 - z0);
  k_adj_seed<<<blocks_for(n, 256), 256, 0, st>>>(g, A, r0, r1, z0, z1, loss);
}

}  // namespace pdp3g
