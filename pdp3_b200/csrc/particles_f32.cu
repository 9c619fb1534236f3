// FP32 cell-local form of the particle phase of one PDP3 step.
//
// Particle state (structure of arrays, 28 B read / 24 B written per step):
//   cell   int32   i * (n_grid_z - 1) + k, the upstream cell
//                  (CELL_NUMBER, include/geometry.h:44: r in (i dr, (i+1) dr])
//   fr, fz float   in-cell offsets r/dr - i and z/dz - k, in (0, 1]
//   ur, uphi, uz float   momentum per mass over c, u = gamma v / c
//   w      float   macroparticle weight (physical particles carried)
//   alive  uint8   bunch species only
//
// The step is the upstream one (gather, relativistic Boris or the upstream
// Vay, two half moves with the rz rotation, azimuthal deposition at the
// mid-step position, reflection or loss at the walls, r-z deposition along
// the step, velocity rotation), written in cell-local units so that every
// quantity that the upstream code forms as a difference of two large
// numbers is formed from offsets instead:
//
// * gather weights: (r2^2 - r1^2) = (r2 - r1)(r2 + r1) with r2 - r1 an exact
//   small offset (EField::get_field src/eField.cpp:204-316, including its
//   CELL_VOLUME(i+3) and CELL_VOLUME(i+2) normalisation);
// * rz rotation: r' - x = y^2 / (x + r') instead of sqrt(x^2+y^2) - x;
// * r-z deposition (Particles::simple_current_distribution,
//   src/particles.cpp:333-474): with rho_m the segment's mid radius in
//   cells, f_m its offset and s = (d_rho/2)/rho_m, the closed forms reduce to
//     j_z(i)   ~ d_zeta [(1 - f_m)(2i + f_m) + i(i+1) eps] / (i rho_m)
//     j_z(i+1) ~ d_zeta [f_m (2i + 1 + f_m) - i(i+1) eps] / ((i+1) rho_m)
//     j_r(i,k) ~ d_rho beta/2 - d_zeta d_rho/4 + i(i+1)/2 [d_rho beta/(rho_o rho_n)
//                - d_zeta d_rho/(2 rho_n rho_m) - d_zeta eps/rho_m]    / (i + 1/2)
//   (j_r(i,k+1) the same with beta -> 1 - beta, d_zeta -> -d_zeta), where
//   eps = atanh(s)/s - 1 carries the upstream log((r_o+dr)/r_o) term.  These
//   are the upstream integrals rearranged; they are smooth in d_rho -> 0 and
//   d_zeta -> 0, where the upstream switches to strict_motion_weighting
//   (src/particles.cpp:786-988), whose z-only and i = 0 forms they equal.
//
// Each warp stages 128 consecutive particles through shared memory (16-byte
// coalesced loads and stores), each lane steps 4 consecutive particles and
// keeps FP32 running sums of their deposits while the cell stays the same;
// one segmented warp reduction per 128 particles then adds the runs into the
// FP64 grid currents with FP64 atomics (particles sorted by cell make the
// runs long).  Warps are independent: no CTA-wide synchronisation.
#include "particles_f32.cuh"

namespace pdp3g {

// One thread of the CTA asks L2 for the input state of the CTA's next chunk
// (when that chunk is a full one: every prefetched byte lies inside the
// arrays) while its warps step the current one: 1.92 -> 1.87 ms per 64-ppc
// wake step.
__device__ __forceinline__ void prefetch_f32_chunk(const SpeciesF32 &s, long long next) {
  if ((next + 1) * F32_CHUNK > s.n) return;
  const long long q = next * F32_CHUNK;
  constexpr unsigned B4 = 4u * F32_CHUNK;
  prefetch_l2(s.cell + q, B4);
  prefetch_l2(s.fr + q, B4);
  prefetch_l2(s.fz + q, B4);
  prefetch_l2(s.ur + q, B4);
  prefetch_l2(s.uphi + q, B4);
  prefetch_l2(s.uz + q, B4);
  prefetch_l2(s.w + q, B4);
  if (s.alive) prefetch_l2(s.alive + q, F32_CHUNK);
}

template <bool OUT, int PUSHER>
__global__ void __launch_bounds__(F32_THREADS, F32_MIN_BLOCKS)
    k_push_deposit_f32(GridDev g, SpeciesF32 s, SpeciesOut o) {
  __shared__ F32Shared sm;
  const long long nchunks = (s.n + F32_CHUNK - 1) / F32_CHUNK;
  for (long long chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    if (threadIdx.x == 0) prefetch_f32_chunk(s, chunk + (long long)gridDim.x);
    f32_chunk<OUT, PUSHER>(g, s, o, PUSHER, chunk, sm);
  }
}

// one kernel per pusher (0 relativistic Boris, 1 upstream Vay, 2 classic Boris)
template <bool OUT>
static void launch_f32_kernel(const GridDev &g, const SpeciesF32 &s, const SpeciesOut &o,
                              int pusher, int blocks, cudaStream_t st) {
  if (pusher == 1)
    k_push_deposit_f32<OUT, 1><<<blocks, F32_THREADS, 0, st>>>(g, s, o);
  else if (pusher == 2)
    k_push_deposit_f32<OUT, 2><<<blocks, F32_THREADS, 0, st>>>(g, s, o);
  else
    k_push_deposit_f32<OUT, 0><<<blocks, F32_THREADS, 0, st>>>(g, s, o);
}

// Bunch::bunch_inject in the cell-local form: z = dl * random_reverse(idx, 11)
// + dz/2 (computed in FP64 as upstream), v_z = v_beam (u_z = gamma v / c).
__device__ __forceinline__ void inject_slot_f32(const SpeciesF32 &s, long long idx, double dl,
                                                double half_dz, double dz, int ncz, float uz,
                                                const double *inv_pow11) {
  int int_vel = (int)floor((double)(unsigned)idx);
  double ost = 0, rr = 0;
  int order = 1;
  while (int_vel >= 1 && order < 40) {
    ost = int_vel % 11;
    rr = rr + ost * inv_pow11[order];
    int_vel = (int)((int_vel - ost) / 11);
    order = order + 1;
  }
  if (idx < s.n) {
    const double z = dl * rr + half_dz;
    int k = (int)ceil(z / dz) - 1;
    if (k < 0) k = 0;
    if (k > ncz - 1) k = ncz - 1;
    const int c = s.cell[idx];
    const int i = c / ncz;
    s.cell[idx] = i * ncz + k;
    s.fz[idx] = (float)(z / dz - k);
    s.uz[idx] = uz;
    s.alive[idx] = 1;
  }
}

__global__ void k_bunch_inject_f32(SpeciesF32 s, long long start, long long count, double dl,
                                   double half_dz, double dz, int ncz, float uz,
                                   const double *inv_pow11) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < count;
       j += (long long)gridDim.x * blockDim.x)
    inject_slot_f32(s, start + j, dl, half_dz, dz, ncz, uz, inv_pow11);
}

// the same with the schedule evaluated from the device time (a captured step)
__global__ void k_bunch_inject_f32_dev(SpeciesF32 s, const double *d_t, double begin, double end,
                                       double dt, unsigned pis, double dl, double half_dz,
                                       double dz, int ncz, float uz, const double *inv_pow11) {
  long long start, count;
  if (!inject_window(*d_t, begin, end, dt, pis, (unsigned)s.n, start, count)) return;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < count;
       j += (long long)gridDim.x * blockDim.x)
    inject_slot_f32(s, start + j, dl, half_dz, dz, ncz, uz, inv_pow11);
}

// Particles::charge_weighting (src/particles.cpp:101-226) for the cell-local
// form: positions are rebuilt in FP64 from (cell, offsets) and weighted with
// the upstream formulas; runs of lanes on the same node block are summed in
// the warp before the atomics (charge_run_add).  The loop runs whole warps
// (every lane takes part in the warp sums).
__global__ void k_charge_density_f32(GridDev g, SpeciesF32 s, double charge, double *rho) {
  const int ncz = g.nz - 1;
  const double dr = g.dr, dz = g.dz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p0 = blockIdx.x * (long long)blockDim.x + (threadIdx.x & ~31); p0 < s.n;
       p0 += stride) {
    const long long p = p0 + (threadIdx.x & 31);
    const bool live = p < s.n && (s.alive == nullptr || s.alive[p]);
    int r_i = 0, z_k = 0;
    double w[4] = {0, 0, 0, 0};
    if (live) {
      const int c = s.cell[p];
      const int ci = c / ncz, ck = c - ci * ncz;
      const double r = (ci + (double)s.fr[p]) * dr, z = (ck + (double)s.fz[p]) * dz;
      charge_weights(g, r, z, charge * (double)s.w[p], r_i, z_k, w);
    }
    charge_run_add(g, rho, live, r_i, z_k, w);
  }
}

// v0: sum m c^2 (gamma - 1) = m c^2 u^2 / (gamma + 1), v1: alive count
__global__ void k_kinetic_f32(SpeciesF32 s, double mass, double *partials) {
  double v[2] = {0, 0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x) {
    if (s.alive != nullptr && !s.alive[p]) continue;
    const double ur = s.ur[p], up = s.uphi[p], uz = s.uz[p];
    const double u2 = ur * ur + up * up + uz * uz;
    v[0] += mass * (double)s.w[p] * LIGHT_SPEED_POW_2 * u2 / (sqrt(1.0 + u2) + 1.0);
    v[1] += 1.0;
  }
  __shared__ double sh[2][F32_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = 0; j < 2; j++) {
    double x = v[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[j][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double sum = 0;
    for (int w = 0; w < F32_THREADS / 32; w++) sum += sh[threadIdx.x][w];
    partials[(size_t)blockIdx.x * 2 + threadIdx.x] = sum;
  }
}

// cell-local FP32 state -> FP64 r, z, v (and w when w_out is given)
__global__ void k_cell_to_f64(SpeciesF32 s, double dr, double dz, int ncz, double *r, double *z,
                              double *vr, double *vphi, double *vz, double *w_out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x) {
    const int c = s.cell[p];
    const int i = c / ncz, k = c - (c / ncz) * ncz;
    r[p] = (i + (double)s.fr[p]) * dr;
    z[p] = (k + (double)s.fz[p]) * dz;
    const double ur = s.ur[p], up = s.uphi[p], uz = s.uz[p];
    const double c_over_g = LIGHT_SPEED / sqrt(1.0 + (ur * ur + up * up + uz * uz));
    vr[p] = ur * c_over_g;
    vphi[p] = up * c_over_g;
    vz[p] = uz * c_over_g;
    if (w_out) w_out[p] = s.w[p];
  }
}

// FP64 r, z, v (and w when given) -> cell-local FP32 state; a NaN position,
// a cell outside the grid or v >= c raises the matching error flag.
__global__ void k_f64_to_cell(SpeciesF32 s, const double *r, const double *z, const double *vr,
                              const double *vphi, const double *vz, const double *w_in,
                              double dr, double dz, int nr, int nz, unsigned *err) {
  const int ncz = nz - 1;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x) {
    const double rp = r[p], zp = z[p];
    if (!isfinite(rp) || !isfinite(zp)) {
      atomicOr(err, ERR_NAN);
      continue;
    }
    int i = (int)ceil(rp / dr) - 1, k = (int)ceil(zp / dz) - 1;
    if (i < 0) i = 0;
    if (k < 0) k = 0;
    if (i > nr - 2 || k > nz - 2) {
      atomicOr(err, ERR_OUT_OF_GRID);
      i = min(i, nr - 2);
      k = min(k, nz - 2);
    }
    s.cell[p] = i * ncz + k;
    s.fr[p] = (float)(rp / dr - i);
    s.fz[p] = (float)(zp / dz - k);
    const double v2 = __dadd_rn(__dadd_rn(__dmul_rn(vr[p], vr[p]), __dmul_rn(vphi[p], vphi[p])),
                                __dmul_rn(vz[p], vz[p]));
    if (!(v2 < LIGHT_SPEED_POW_2)) {
      atomicOr(err, ERR_V_GE_C);
      continue;
    }
    const double gc = 1.0 / (LIGHT_SPEED * sqrt(1.0 - v2 / LIGHT_SPEED_POW_2));
    s.ur[p] = (float)(vr[p] * gc);
    s.uphi[p] = (float)(vphi[p] * gc);
    s.uz[p] = (float)(vz[p] * gc);
    if (w_in) ((float *)s.w)[p] = (float)w_in[p];
  }
}

void launch_cell_to_f64(const SpeciesF32 &s, double dr, double dz, int ncz, double *r, double *z,
                        double *vr, double *vphi, double *vz, double *w_out, cudaStream_t st) {
  if (s.n <= 0) return;
  long long blocks = (s.n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_cell_to_f64<<<(int)blocks, 256, 0, st>>>(s, dr, dz, ncz, r, z, vr, vphi, vz, w_out);
}

void launch_f64_to_cell(const SpeciesF32 &s, const double *r, const double *z, const double *vr,
                        const double *vphi, const double *vz, const double *w_in, double dr,
                        double dz, int nr, int nz, unsigned *err, cudaStream_t st) {
  if (s.n <= 0) return;
  long long blocks = (s.n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_f64_to_cell<<<(int)blocks, 256, 0, st>>>(s, r, z, vr, vphi, vz, w_in, dr, dz, nr, nz, err);
}

void launch_push_deposit_f32(const GridDev &g, const SpeciesF32 &s, int pusher, int n_sm,
                             int blocks_per_sm, cudaStream_t st) {
  if (s.n <= 0) return;
  long long chunks = (s.n + F32_CHUNK - 1) / F32_CHUNK;
  long long blocks = (long long)n_sm * (blocks_per_sm > 0 ? blocks_per_sm : F32_MIN_BLOCKS);
  if (blocks > chunks) blocks = chunks;
  launch_f32_kernel<false>(g, s, in_place(s), pusher, (int)blocks, st);
}

void launch_push_deposit_f32_to(const GridDev &g, const SpeciesF32 &s, const SpeciesOut &o,
                                int pusher, int n_sm, int blocks_per_sm, cudaStream_t st) {
  if (s.n <= 0) return;
  long long chunks = (s.n + F32_CHUNK - 1) / F32_CHUNK;
  long long blocks = (long long)n_sm * (blocks_per_sm > 0 ? blocks_per_sm : F32_MIN_BLOCKS);
  if (blocks > chunks) blocks = chunks;
  launch_f32_kernel<true>(g, s, o, pusher, (int)blocks, st);
}

void launch_bunch_inject_f32(const SpeciesF32 &s, long long start, long long count, double dl,
                             double half_dz, double dz, int ncz, float uz,
                             const double *inv_pow11, cudaStream_t st) {
  if (count <= 0) return;
  long long blocks = (count + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  k_bunch_inject_f32<<<(int)blocks, 256, 0, st>>>(s, start, count, dl, half_dz, dz, ncz, uz,
                                                  inv_pow11);
}

void launch_bunch_inject_f32_dev(const SpeciesF32 &s, const double *d_t, double begin,
                                 double end, double dt, unsigned pis, double dl, double half_dz,
                                 double dz, int ncz, float uz, const double *inv_pow11,
                                 cudaStream_t st) {
  if (pis == 0) return;
  long long blocks = ((long long)pis + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  k_bunch_inject_f32_dev<<<(int)blocks, 256, 0, st>>>(s, d_t, begin, end, dt, pis, dl, half_dz,
                                                      dz, ncz, uz, inv_pow11);
}

void launch_charge_density_f32(const GridDev &g, const SpeciesF32 &s, double charge,
                               double *rho, cudaStream_t st) {
  if (s.n <= 0) return;
  long long blocks = (s.n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_charge_density_f32<<<(int)blocks, 256, 0, st>>>(g, s, charge, rho);
}

void launch_kinetic_f32(const SpeciesF32 &s, double mass, double *partials, double *out,
                        cudaStream_t st) {
  const int nb = diag_blocks();
  k_kinetic_f32<<<nb, F32_THREADS, 0, st>>>(s, mass, partials);
  launch_finalize(partials, nb, 2, out, st);
}

}  // namespace pdp3g
