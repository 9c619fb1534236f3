// Adjoint (vector-Jacobian product) of the FP32 cell-local PDP3 step.
//
// Reverse of one step s, given the adjoints of the state after it
// (lE, lH: FP64 grids; la, lb, lu: FP32 per particle):
//   1  E update   E' = ke E - kh (J + curl H')   (src/eField.cpp:85-170)
//        lJ = -kh lE',  lH' += curl^T(-kh lE'),  lE = ke lE'
//   2  particles  (adjoint_particle.cuh reverse on each particle's tape,
//        recomputed from the stored post-injection state of step s)
//        la/lb/lu updated in place, lw += ..., lE += gather^T, lHh += gather^T
//   3  injection  slots injected at step s: their z and u_z were set from the
//        beam velocity, so lb/luz go to d/dv_beam and are then cleared
//   4  H update   H' = H + a(E), Hh = H + a(E)/2    (src/hField.cpp:93-157)
//        lE += a^T(lH' + lHh/2),  lH = lH' + lHh
// Stencil transposes scatter with FP64 atomics.
#include <algorithm>
#include <climits>

#include "adjoint_particle.cuh"
#include "pdp3g_internal.cuh"

namespace pdp3g {

#define AIDX(i, k) ((size_t)(i) * (size_t)nz + (size_t)(k))


// step 1: E update transposed, node (i, k) of the E update's range:
// lJ = -kh lE', lH += curl^T(-kh lE'), lE = ke lE' (the scatter goes to lH
// only, so each thread can scale its own lE in place)
__global__ void k_adj_e(GridDev g, AdjGrids A) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const long long total = (long long)(nr - 1) * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1)), k = (int)(t - (long long)i * (nz - 1));
    const double epsx2 = 2 * 1.0 * EPSILON0;
    const double sigma_t = g.sigma[AIDX(i, k)] * dt;
    const double kh = 2 * dt / (epsx2 + sigma_t);
    const double ke = (epsx2 - sigma_t) / (epsx2 + sigma_t);
    if (k >= 1) {  // E_r
      const double gr = -kh * A.lEr[AIDX(i, k)];
      A.lJr[AIDX(i, k)] = (float)gr;
      atomicAdd(&A.lHphi[AIDX(i, k)], gr / dz);
      atomicAdd(&A.lHphi[AIDX(i, k - 1)], -gr / dz);
      A.lEr[AIDX(i, k)] *= ke;
    }
    const double gz = -kh * A.lEz[AIDX(i, k)];
    A.lJz[AIDX(i, k)] = (float)gz;
    A.lEz[AIDX(i, k)] *= ke;
    if (i == 0) {  // on-axis E_z: 4/dr H_phi
      atomicAdd(&A.lHphi[AIDX(i, k)], -4.0 * gz / dr);
    } else {
      atomicAdd(&A.lHphi[AIDX(i, k)], gz * (-1.0 / dr - 1.0 / (2.0 * dr * i)));
      atomicAdd(&A.lHphi[AIDX(i - 1, k)], gz * (1.0 / dr - 1.0 / (2.0 * dr * i)));
      if (k >= 1) {  // E_phi
        const double gp = -kh * A.lEphi[AIDX(i, k)];
        A.lJphi[AIDX(i, k)] = (float)gp;
        atomicAdd(&A.lHr[AIDX(i, k)], -gp / dz);
        atomicAdd(&A.lHr[AIDX(i, k - 1)], gp / dz);
        atomicAdd(&A.lHz[AIDX(i, k)], gp / dr);
        atomicAdd(&A.lHz[AIDX(i - 1, k)], -gp / dr);
        A.lEphi[AIDX(i, k)] *= ke;
      }
    }
  }
}

// Between steps 1 and 2: cell (i, k) is active when any adjoint of J that
// the particles starting in it read is nonzero.  A particle's step moves it
// at most half a cell (Courant 0.5), so its mid-step and path cells lie
// within one cell of its start cell and the nodes it reads adjoints of J at
// within i-1..i+2, k-1..k+2.  The adjoints of the fields spread from the
// probe by one node per step (the Yee stencil), so early in the reverse most
// cells are inactive; a particle whose own adjoints are zero in an inactive
// cell has a reverse whose every output is zero (the reverse is linear in
// them) and is skipped.
__global__ void k_adj_active(GridDev g, AdjGrids A, uint8_t *active) {
  const int nr = g.nr, nz = g.nz, ncz = nz - 1;
  const long long total = (long long)(nr - 1) * ncz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / ncz), k = (int)(t - (long long)i * ncz);
    const int i0 = max(i - 1, 0), i1 = min(i + 2, nr - 1);
    const int k0 = max(k - 1, 0), k1 = min(k + 2, nz - 1);
    bool any = false;
    for (int ii = i0; ii <= i1 && !any; ii++)
      for (int kk = k0; kk <= k1; kk++) {
        const size_t n = AIDX(ii, kk);
        if (A.lJr[n] != 0.0f || A.lJphi[n] != 0.0f || A.lJz[n] != 0.0f) {
          any = true;
          break;
        }
      }
    active[t] = any ? 1 : 0;
  }
}

// step 4: H update transposed, every node: where the H update ran,
// lE += a^T(lH + lHh/2) and lH += lHh; everywhere lHh = 0 (the half-step
// values the update did not write never change, so their adjoints are
// dropped).  The scatter goes to lE only.
__global__ void k_adj_h(GridDev g, AdjGrids A) {
  const int nr = g.nr, nz = g.nz;
  const double dr = g.dr, dz = g.dz, dt = g.dt;
  const long long total = (long long)nr * nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / nz), k = (int)(t - (long long)i * nz);
    if (k <= nz - 2) {
      const double la = A.lHr[t] + 0.5 * A.lHhr[t];
      const double ca = dt / (dz * MAGN_CONST);
      atomicAdd(&A.lEphi[AIDX(i, k + 1)], la * ca);
      atomicAdd(&A.lEphi[AIDX(i, k)], -la * ca);
      A.lHr[t] += A.lHhr[t];
      if (i < nr - 1) {
        const double lb = A.lHphi[t] + 0.5 * A.lHhphi[t];
        atomicAdd(&A.lEz[AIDX(i + 1, k)], lb * dt / (dr * MAGN_CONST));
        atomicAdd(&A.lEz[AIDX(i, k)], -lb * dt / (dr * MAGN_CONST));
        atomicAdd(&A.lEr[AIDX(i, k + 1)], -lb * dt / (dz * MAGN_CONST));
        atomicAdd(&A.lEr[AIDX(i, k)], lb * dt / (dz * MAGN_CONST));
        // H_z -= c, Hh_z = H_z - c/2
        const double lc = -(A.lHz[t] + 0.5 * A.lHhz[t]);
        const double p = 1.0 / (2.0 * dr * (i + 0.5));
        atomicAdd(&A.lEphi[AIDX(i + 1, k)], lc * dt * (p + 1.0 / dr) / MAGN_CONST);
        atomicAdd(&A.lEphi[AIDX(i, k)], lc * dt * (p - 1.0 / dr) / MAGN_CONST);
        A.lHphi[t] += A.lHhphi[t];
        A.lHz[t] += A.lHhz[t];
      }
    }
    A.lHhr[t] = 0.0;
    A.lHhphi[t] = 0.0;
    A.lHhz[t] = 0.0;
  }
}

// adjoint of J at (i, k), 0 outside the grid
__device__ __forceinline__ float lget(const GridDev &g, const float *f, int i, int k) {
  if ((unsigned)i >= (unsigned)g.nr || (unsigned)k >= (unsigned)g.nz) return 0.0f;
  return __ldg(f + (size_t)i * g.nz + k);
}

__device__ __forceinline__ void ladd(const GridDev &g, double *f, int i, int k, float v) {
  if (v == 0.0f || (unsigned)i >= (unsigned)g.nr || (unsigned)k >= (unsigned)g.nz) return;
  atomicAdd(f + (size_t)i * g.nz + k, (double)v);
}

#ifndef ADJ_THREADS_PER_CTA
#define ADJ_THREADS_PER_CTA 128
#endif
#ifndef ADJ_MIN_BLOCKS
#define ADJ_MIN_BLOCKS 4  // CTAs per SM the register budget is sized for (128 registers)
#endif
// the particle reverse keeps its tape in registers: with the warp-level
// reduction of the field-node adjoints (no shared tile, no barrier), 512
// resident threads of 128 registers beat 1024 of 64 with the tape spilled;
// 128-thread CTAs (4 per SM) end the grid-stride loop with a shorter tail
// than 256-thread ones (2 per SM)
constexpr int ADJ_THREADS = ADJ_THREADS_PER_CTA;
static_assert(ADJ_THREADS % 16 == 0, "prefetch sizes are multiples of 16 bytes");
#ifndef ADJ_PREFETCH_AHEAD
#define ADJ_PREFETCH_AHEAD 1  // CTA iterations between a chunk's prefetch and its use
#endif
// Warp-level segmented sum over runs of consecutive lanes with the same key
// (particles sorted by cell, with the same half-cell quadrant, share their
// 24 gather nodes); the last lane of each run holds the run's totals.
// One lane asks L2 for the particle chunk that this CTA steps after the
// current one (the reverse is latency-bound: 16 warps per SM), when that
// chunk is a full one: every prefetched byte lies inside the arrays.
__device__ __forceinline__ void prefetch_chunk(const AdjSpeciesDev &S, long long next) {
  if ((next + 1) * ADJ_THREADS > S.st.n) return;
  const long long q = next * ADJ_THREADS;
  constexpr unsigned B4 = 4u * ADJ_THREADS;
  prefetch_l2(S.st.cell + q, B4);
  prefetch_l2(S.st.fr + q, B4);
  prefetch_l2(S.st.fz + q, B4);
  prefetch_l2(S.st.ur + q, B4);
  prefetch_l2(S.st.uphi + q, B4);
  prefetch_l2(S.st.uz + q, B4);
  prefetch_l2(S.st.w + q, B4);
  if (S.st.alive) prefetch_l2(S.st.alive + q, ADJ_THREADS);
  prefetch_l2(S.la + q, B4);
  prefetch_l2(S.lb + q, B4);
  prefetch_l2(S.lur + q, B4);
  prefetch_l2(S.luphi + q, B4);
  prefetch_l2(S.luz + q, B4);
  prefetch_l2(S.lw + q, 2 * B4);
}

template <int N>
__device__ __forceinline__ bool warp_seg_sum(int key, float (&v)[N]) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int prev = __shfl_up_sync(FULL, key, 1);
  const int next = __shfl_down_sync(FULL, key, 1);
  const bool head = lane == 0 || prev != key;
  const bool tail = lane == 31 || next != key;
  const unsigned heads = __ballot_sync(FULL, head);
  const unsigned le = lane == 31 ? FULL : ((2u << lane) - 1u);
  const int seg_start = 31 - __clz(heads & le);
#pragma unroll
  for (int j = 0; j < N; j++) {
    float x = v[j];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const float y = __shfl_up_sync(FULL, x, off);
      if (lane >= seg_start + off) x += y;
    }
    v[j] = x;
  }
  return tail && key >= 0;
}

// step 2: particles.  Q = E and the half-step H of step s as per-cell quads
// (the 2x2 nodes of a cell, GridDev::q32's layout, as the forward step
// gathered them).  Each thread takes one particle; the 24
// field-node adjoints of a warp's particles are summed over runs of lanes
// that share their gather nodes (particles sorted by cell) and each run adds
// its totals to the FP64 grids.  Warps are independent.  WALLS: whether the
// wall-reflection jump terms (face bit 1) are compiled in.
template <bool WALLS>
__global__ void __launch_bounds__(ADJ_THREADS, ADJ_MIN_BLOCKS) k_adj_particles(
    GridDev g, const float4 *Q, AdjSpeciesDev S, AdjGrids A, const uint8_t *active, int face,
    float face_h) {
  const int ncz = g.nz - 1;
  const size_t ncells = (size_t)(g.nr - 1) * ncz;
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
  C.face_h = face_h;
  const long long nchunks = (S.st.n + ADJ_THREADS - 1) / ADJ_THREADS;
  for (long long chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    if (threadIdx.x == 0) prefetch_chunk(S, chunk + ADJ_PREFETCH_AHEAD * (long long)gridDim.x);
    const long long p = chunk * ADJ_THREADS + threadIdx.x;
    bool live = p < S.st.n && (S.st.alive == nullptr || S.st.alive[p]);
    const int c = live ? S.st.cell[p] : 0;
    if (c < 0 || c >= (g.nr - 1) * ncz) live = false;  // flagged by the forward step
    // zero adjoints of the particle and none of J within its reach (k_adj_active):
    // every output of its reverse is zero, nothing to do.  The five loads are
    // issued together and tested bitwise (a sign-only -0.0f counts as
    // nonzero, which only costs a reverse that adds zeros).
    if (live) {
      const unsigned bits = __float_as_uint(S.la[p]) | __float_as_uint(S.lb[p]) |
                            __float_as_uint(S.lur[p]) | __float_as_uint(S.luphi[p]) |
                            __float_as_uint(S.luz[p]);
      if (bits == 0u && !active[c]) live = false;
    }
    if (__all_sync(0xffffffffu, !live)) continue;  // the whole warp: no sums to add either
    const int ci = c / ncz, ck = c - (c / ncz) * ncz;
    float lf[24];  // this lane's field-node adjoints, reduced across the warp
    int key = -1, q_ir_h = 0, q_kz_h = 0;
    if (!live) {
#pragma unroll
      for (int j = 0; j < 24; j++) lf[j] = 0.0f;
    } else {
      adj::Tape<float> tp;
      tp.i = ci;
      tp.k = ck;
      tp.a = S.st.fr[p];
      tp.b = S.st.fz[p];
      tp.u[0] = S.st.ur[p];
      tp.u[1] = S.st.uphi[p];
      tp.u[2] = S.st.uz[p];
      tp.w = S.st.w[p];
      adj::gather_weights(tp);
      // node rows/columns of the two weightings (clamped as the forward gather)
      const int ir_h = min(tp.ir_h, g.nr - 2), ir_n = min(tp.i, g.nr - 2);
      const int kz_h = min(tp.kz_h, g.nz - 2), kz_n = min(tp.k, g.nz - 2);
#pragma unroll
      for (int cc = 0; cc < 3; cc++) {
        {
          const int ir = adj::comp_rhalf(0, cc) ? ir_h : ir_n;
          const int kz = adj::comp_zhalf(0, cc) ? kz_h : kz_n;
          const float4 v = __ldg(Q + cc * ncells + (size_t)ir * ncz + kz);
          tp.fe[cc][0] = v.x;
          tp.fe[cc][1] = v.y;
          tp.fe[cc][2] = v.z;
          tp.fe[cc][3] = v.w;
        }
        {
          const int ir = adj::comp_rhalf(1, cc) ? ir_h : ir_n;
          const int kz = adj::comp_zhalf(1, cc) ? kz_h : kz_n;
          const float4 v = __ldg(Q + (3 + cc) * ncells + (size_t)ir * ncz + kz);
          tp.fh[cc][0] = v.x;
          tp.fh[cc][1] = v.y;
          tp.fh[cc][2] = v.z;
          tp.fh[cc][3] = v.w;
        }
      }
      adj::forward(C, tp);
      float l_jphi[4] = {lget(g, A.lJphi, tp.i1, tp.k1), lget(g, A.lJphi, tp.i1 + 1, tp.k1),
                         lget(g, A.lJphi, tp.i1, tp.k1 + 1),
                         lget(g, A.lJphi, tp.i1 + 1, tp.k1 + 1)};
      float l_piece[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
      if (tp.path_ok) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
          if (q > tp.np) continue;
          const int qi = tp.pci(q), qk = tp.pck(q);
          l_piece[q][0] = lget(g, A.lJz, qi, qk);
          l_piece[q][1] = lget(g, A.lJz, qi + 1, qk);
          l_piece[q][2] = lget(g, A.lJr, qi, qk);
          l_piece[q][3] = lget(g, A.lJr, qi, qk + 1);
        }
      }
      const float l_uout[3] = {S.lur[p], S.luphi[p], S.luz[p]};
      float l_a, l_b, l_u[3], l_w, l_fe[3][4], l_fh[3][4];
      adj::reverse<float, WALLS>(C, tp, S.la[p], S.lb[p], l_uout, l_jphi, l_piece, l_a, l_b,
                                 l_u, l_w, l_fe, l_fh);
      S.la[p] = l_a;
      S.lb[p] = l_b;
      S.lur[p] = l_u[0];
      S.luphi[p] = l_u[1];
      S.luz[p] = l_u[2];
      S.lw[p] += (double)l_w;
#pragma unroll
      for (int cc = 0; cc < 3; cc++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
          lf[cc * 4 + q] = l_fe[cc][q];
          lf[12 + cc * 4 + q] = l_fh[cc][q];
        }
      // lanes with the same cell and half-cell quadrant share the 24 nodes
      key = ((ci * ncz + ck) * 2 + (tp.ir_h == ci ? 1 : 0)) * 2 + (tp.kz_h == ck ? 1 : 0);
      q_ir_h = ir_h;
      q_kz_h = kz_h;
    }
    if (warp_seg_sum<24>(key, lf)) {
      const int ir_n = ci, kz_n = ck;
#pragma unroll
      for (int cc = 0; cc < 3; cc++) {
        {
          const int ir = adj::comp_rhalf(0, cc) ? q_ir_h : ir_n;
          const int kz = adj::comp_zhalf(0, cc) ? q_kz_h : kz_n;
          double *grid = cc == 0 ? A.lEr : (cc == 1 ? A.lEphi : A.lEz);
          ladd(g, grid, ir, kz, lf[cc * 4 + 0]);
          ladd(g, grid, ir + 1, kz, lf[cc * 4 + 1]);
          ladd(g, grid, ir, kz + 1, lf[cc * 4 + 2]);
          ladd(g, grid, ir + 1, kz + 1, lf[cc * 4 + 3]);
        }
        {
          const int ir = adj::comp_rhalf(1, cc) ? q_ir_h : ir_n;
          const int kz = adj::comp_zhalf(1, cc) ? q_kz_h : kz_n;
          double *grid = cc == 0 ? A.lHhr : (cc == 1 ? A.lHhphi : A.lHhz);
          ladd(g, grid, ir, kz, lf[12 + cc * 4 + 0]);
          ladd(g, grid, ir + 1, kz, lf[12 + cc * 4 + 1]);
          ladd(g, grid, ir, kz + 1, lf[12 + cc * 4 + 2]);
          ladd(g, grid, ir + 1, kz + 1, lf[12 + cc * 4 + 3]);
        }
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
  k_adj_e<<<blocks_for((long long)(g.nr - 1) * (g.nz - 1), 256), 256, 0, st>>>(g, A);
}

void adj_launch_h(const GridDev &g, const AdjGrids &A, cudaStream_t st) {
  k_adj_h<<<blocks_for((long long)g.nr * g.nz, 256), 256, 0, st>>>(g, A);
}

void adj_launch_active(const GridDev &g, const AdjGrids &A, uint8_t *active, cudaStream_t st) {
  k_adj_active<<<blocks_for((long long)(g.nr - 1) * (g.nz - 1), 256), 256, 0, st>>>(g, A, active);
}

void adj_launch_particles(const GridDev &g, const float4 *Q, const AdjSpeciesDev &S,
                          const AdjGrids &A, const uint8_t *active, int face, float face_h,
                          cudaStream_t st) {
  if (S.st.n <= 0) return;
  const long long nchunks = (S.st.n + ADJ_THREADS - 1) / ADJ_THREADS;
  auto kernel = (face & 2) ? k_adj_particles<true> : k_adj_particles<false>;
  int bpsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, kernel, ADJ_THREADS, 0) !=
          cudaSuccess || bpsm < 1)
    bpsm = 1;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long blocks = std::min<long long>(nchunks, (long long)bpsm * nsm);
  kernel<<<(int)std::max<long long>(blocks, 1), ADJ_THREADS, 0, st>>>(g, Q, S, A, active,
                                                                         face, face_h);
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
