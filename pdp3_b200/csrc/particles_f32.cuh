// Device code of the FP32 cell-local particle phase (see particles_f32.cu).
#pragma once

#include "pdp3g_internal.cuh"

namespace pdp3g {

// node offset i * n_grid_z + k in 32-bit arithmetic (FP32 contexts hold
// fewer than 2^31 nodes, checked at creation): one multiply-add instead of
// a 64-bit one per address
#define GIDX(i, k) ((unsigned)(i) * (unsigned)g.nz + (unsigned)(k))

constexpr int F32_THREADS = 256;
constexpr int F32_MIN_BLOCKS = 4;                     // CTAs per SM (64 registers)
constexpr int F32_WARPS = F32_THREADS / 32;
constexpr int F32_PER_LANE = 4;                       // consecutive particles per thread
constexpr int F32_WARP_CHUNK = 32 * F32_PER_LANE;     // particles per warp
static_assert(F32_CHUNK == F32_WARPS * F32_WARP_CHUNK, "CTA chunk = its warps' chunks");

__device__ __forceinline__ void flag32(const GridDev &g, unsigned bit) { atomicOr(g.err, bit); }

// moves (i, f) so that f is in (0, 1] (CELL_NUMBER semantics); cells below
// 0 clamp to 0 like the upstream "sometimes it gives -1" workaround.  c =
// ceil(f) - 1 cells in one step, branch-free; for a move of at most one cell
// (all that a step at Courant 0.5 makes) f - c is the same subtraction of 1
// as a cell-by-cell loop would make.
__device__ __forceinline__ void renorm(int &i, float &f) {
  const float c = ceilf(f) - 1.0f;
  i += (int)c;
  f -= c;
  if (i < 0) { f = f + (float)i; i = 0; }
}

// adds v into the FP64 grid current `base` at node (i, k), flagging nodes
// outside the grid.  Arguments by value: the out-of-line callers below take
// no pointer to the kernel's parameters or locals.
__device__ __forceinline__ void dep_node(unsigned *err, double *base, int nr, int nz, int i, int k,
                                         float v) {
  if ((unsigned)i >= (unsigned)nr || (unsigned)k >= (unsigned)nz) {
    atomicOr(err, ERR_OUT_OF_GRID);
    return;
  }
  atomicAdd(base + (unsigned)i * (unsigned)nz + (unsigned)k, (double)v);
}

// the per-node tested deposits of a 2x2 block at the grid edge (dep_block's
// rare path, kept out of line so that the inlined copies of dep_block stay
// small); mode as MODE in dep_block
static __device__ __noinline__ void dep_block_edge(double *jr, double *jphi, double *jz,
                                                   unsigned *err, int nr, int nz, int mode, int i,
                                                   int k, float v0, float v1, float v2, float v3) {
  if (mode == 0) {
    dep_node(err, jphi, nr, nz, i, k, v0);
    dep_node(err, jphi, nr, nz, i + 1, k, v1);
    dep_node(err, jphi, nr, nz, i, k + 1, v2);
    dep_node(err, jphi, nr, nz, i + 1, k + 1, v3);
  } else {
    dep_node(err, jz, nr, nz, i, k, v0);
    dep_node(err, jz, nr, nz, i + 1, k, v1);
    dep_node(err, jr, nr, nz, i, k, v2);
    dep_node(err, jr, nr, nz, i, k + 1, v3);
  }
}

// atanh(s)/s - 1 away from 0: rare in a step (|s| >= 0.1 is a radial move of
// a fifth of the radius), and out of line, so the hot loop keeps no copy of
// atanhf's code
static __device__ __noinline__ float atanh_ratio_m1_far(float s) { return atanhf(s) / s - 1.0f; }

// eps(s) = atanh(s)/s - 1
__device__ __forceinline__ float atanh_ratio_m1(float s) {
  const float s2 = s * s;
  if (s2 < 0.01f) return s2 * (1.0f / 3.0f + s2 * (0.2f + s2 * (1.0f / 7.0f + s2 * (1.0f / 9.0f))));
  return atanh_ratio_m1_far(s);
}

// One straight piece of the step inside cell (ci, ck), endpoints given as
// offsets (ao, co) -> (an, cn) relative to that cell (each in [0, 1]).
// out = {j_z(ci, ck), j_z(ci+1, ck), j_r(ci, ck), j_r(ci, ck+1)}.
__device__ __forceinline__ void piece_values(int ci, float ao, float co, float an, float cn,
                                             float kz, float kr, float out[4]) {
  const float drho = an - ao, dzeta = cn - co;
  const float fi = (float)ci;
  const float fm = 0.5f * (ao + an);
  const float rho_m = fi + fm;
  const float beta = 1.0f - co;  // ((k+1) dz - z_o)/dz
  if (ci >= 1) {
    const float inv_rm = 1.0f / rho_m;
    const float s = 0.5f * drho * inv_rm;
    const float eps = atanh_ratio_m1(s);
    const float ii1 = fi * (fi + 1.0f);
    out[0] = kz * dzeta * ((1.0f - fm) * (2.0f * fi + fm) + ii1 * eps) * inv_rm / fi;
    out[1] = kz * dzeta * (fm * (2.0f * fi + 1.0f + fm) - ii1 * eps) * inv_rm / (fi + 1.0f);
    const float rho_o = fi + ao, rho_n = fi + an;
    const float q1 = drho / (rho_o * rho_n);
    const float q2 = dzeta * drho * 0.5f * inv_rm / rho_n;
    const float q3 = dzeta * eps * inv_rm;
    const float h = 0.5f * ii1;
    const float inv_r0 = kr / (fi + 0.5f);
    out[2] = inv_r0 * (0.5f * drho * beta - 0.25f * dzeta * drho + h * (q1 * beta - q2 - q3));
    // beta + co = 1, so out[2] + out[3] = inv_r0 (drho / 2 + h q1)
    out[3] = inv_r0 * (0.5f * drho + h * q1) - out[2];
  } else {
    // i = 0: src/particles.cpp:415-473 (no log terms; i(i+1) = 0)
    out[0] = 8.0f * kz * dzeta * (1.0f - fm);
    out[1] = kz * dzeta * (1.0f + fm);
    out[2] = 2.0f * kr * (0.5f * drho * beta - 0.25f * dzeta * drho);
    out[3] = 2.0f * kr * (0.5f * drho * co + 0.25f * dzeta * drho);
  }
}

// the 4 deposits of a cell (i, k) into the nodes (i..i+1, k..k+1):
// MODE 0 = j_phi at (i,k), (i+1,k), (i,k+1), (i+1,k+1);
// MODE 1 = j_z at (i,k), (i+1,k), j_r at (i,k), (i,k+1).
// One bounds test for the block; the per-node tests only at the grid edge.
template <int MODE>
__device__ __forceinline__ void dep_block(const GridDev &g, int i, int k, const float v[4]) {
  if ((unsigned)i < (unsigned)(g.nr - 1) && (unsigned)k < (unsigned)(g.nz - 1)) {
    const size_t n0 = GIDX(i, k);
    if (MODE == 0) {
      atomicAdd(g.jphi + n0, (double)v[0]);
      atomicAdd(g.jphi + n0 + g.nz, (double)v[1]);
      atomicAdd(g.jphi + n0 + 1, (double)v[2]);
      atomicAdd(g.jphi + n0 + g.nz + 1, (double)v[3]);
    } else {
      atomicAdd(g.jz + n0, (double)v[0]);
      atomicAdd(g.jz + n0 + g.nz, (double)v[1]);
      atomicAdd(g.jr + n0, (double)v[2]);
      atomicAdd(g.jr + n0 + 1, (double)v[3]);
    }
    return;
  }
  dep_block_edge(g.jr, g.jphi, g.jz, g.err, g.nr, g.nz, MODE, i, k, v[0], v[1], v[2], v[3]);
}

// The step's straight path from (i, a, k, b) to (in, an, kn, bn) split at the
// cell faces it crosses (at most one r face and one z face), each piece
// deposited into j_z and j_r.  Nothing is deposited when the path spans more
// than one cell in r or z (as upstream).  Only steps that leave their cell
// come here (about one in a thousand at thermal speeds): out of line, with
// its arguments by value and no results, so that the hot loop keeps neither
// its code nor a local array for it.
static __device__ __noinline__ void deposit_path(double *jr, double *jz, unsigned *err, int nr,
                                                 int nz, int i, float a, int k, float b, int in,
                                                 float an, int kn, float bn, float kz, float kr) {
  const int di = in - i, dk = kn - k;
  if (di < -1 || di > 1 || dk < -1 || dk > 1) return;
  // end point relative to the start cell
  const float A = (float)di + an, B = (float)dk + bn;
  float tr = 2.0f, tz = 2.0f;
  if (di != 0) tr = ((di > 0 ? 1.0f : 0.0f) - a) / (A - a);
  if (dk != 0) tz = ((dk > 0 ? 1.0f : 0.0f) - b) / (B - b);
  // crossings in path order: (t0, kind0), (t1, kind1); kind 0 r face, 1 z face
  const bool cr_r = tr <= 1.0f, cr_z = tz <= 1.0f;
  const int np = (cr_r ? 1 : 0) + (cr_z ? 1 : 0);
  const bool r_first = cr_r && (!cr_z || tr <= tz);
  const float t0 = r_first ? tr : tz, t1 = r_first ? tz : tr;
  const int kind0 = r_first ? 0 : 1;
  int ci = i, ck = k;
  float pa = a, pb = b;  // current point relative to (i, k)
#pragma unroll 1
  for (int p = 0; p <= np; p++) {
    float qa, qb;
    const int kind = (p == 0) ? kind0 : 1 - kind0;
    if (p < np) {
      // crossing point: the crossed coordinate sits exactly on the face
      const float tt = p == 0 ? t0 : t1;
      if (kind == 0) {
        qa = di > 0 ? 1.0f : 0.0f;
        qb = b + tt * (B - b);
      } else {
        qa = a + tt * (A - a);
        qb = dk > 0 ? 1.0f : 0.0f;
      }
    } else {
      qa = A;
      qb = B;
    }
    const float oi = (float)(ci - i), ok = (float)(ck - k);
    float v[4];
    piece_values(ci, pa - oi, pb - ok, qa - oi, qb - ok, kz, kr, v);
    dep_node(err, jz, nr, nz, ci, ck, v[0]);
    dep_node(err, jz, nr, nz, ci + 1, ck, v[1]);
    dep_node(err, jr, nr, nz, ci, ck, v[2]);
    dep_node(err, jr, nr, nz, ci, ck + 1, v[3]);
    if (p < np) {
      if (kind == 0) ci += di; else ck += dk;
    }
    pa = qa;
    pb = qb;
  }
}

// A lane's running sum of the 4 deposits of consecutive particles with the
// same key (node layout as in warp_run_deposit); key < 0: empty.
struct RunAcc {
  int key;  // node index i * n_grid_z + k of the run's cell
  float v[4];
};

template <int MODE>
__device__ __forceinline__ void acc_flush(const GridDev &g, const RunAcc &A) {
  const int i = A.key / g.nz, k = A.key - i * g.nz;
  dep_block<MODE>(g, i, k, A.v);
}

// adds one particle's deposit; a new key flushes the previous run (runs end
// inside a lane rarely when the particles are sorted by cell)
template <int MODE>
__device__ __forceinline__ void acc_add(const GridDev &g, RunAcc &A, int key, const float v[4]) {
  if (key < 0) return;
  if (key == A.key) {
#pragma unroll
    for (int j = 0; j < 4; j++) A.v[j] += v[j];
    return;
  }
  if (A.key >= 0) acc_flush<MODE>(g, A);
  A.key = key;
#pragma unroll
  for (int j = 0; j < 4; j++) A.v[j] = v[j];
}

// Warp-level segmented sum of the lanes' running sums: each run of
// consecutive lanes with the same key (particles sorted by cell form long
// runs) is added up and its last lane adds the totals into the FP64 grid.
// Lanes with key < 0 hold nothing.
// node layout: MODE 0 = j_phi at (i,k), (i+1,k), (i,k+1), (i+1,k+1);
//              MODE 1 = j_z at (i,k), (i+1,k), j_r at (i,k), (i,k+1).
template <int MODE>
__device__ __forceinline__ void warp_run_deposit(const GridDev &g, const RunAcc &A) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int key = A.key;
  const int prev = __shfl_up_sync(FULL, key, 1);
  const int next = __shfl_down_sync(FULL, key, 1);
  const bool head = lane == 0 || prev != key;
  const bool tail = lane == 31 || next != key;
  const unsigned heads = __ballot_sync(FULL, head);
  const unsigned le = lane == 31 ? FULL : ((2u << lane) - 1u);
  const int seg_start = 31 - __clz(heads & le);
  RunAcc R = A;
#pragma unroll
  for (int j = 0; j < 4; j++) {
    float x = R.v[j];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const float y = __shfl_up_sync(FULL, x, off);
      if (lane >= seg_start + off) x += y;
    }
    R.v[j] = x;
  }
  if (tail && key >= 0) acc_flush<MODE>(g, R);
}

__device__ __forceinline__ void weights_rhalf(int i, float a, int &ir, float &w0, float &w1) {
  // E_r / H_z / H_phi radial part: i_r = CELL_NUMBER(r - dr/2), volumes
  // CELL_VOLUME(i_r+1), CELL_VOLUME(i_r+3) (src/eField.cpp:225-248)
  ir = a > 0.5f ? i : i - 1;
  if (ir < 0) ir = 0;
  const float d21 = (float)(ir - i) + 1.5f - a;
  const float s21 = (float)(ir + i) + 0.5f + a;
  const float d32 = (float)(i - ir) + a - 0.5f;
  const float s32 = (float)(i + ir) + 1.5f + a;
  w0 = d21 * s21 / (2.0f * (float)(ir + 1));
  w1 = d32 * s32 / (2.0f * (float)(ir + 3));
}

__device__ __forceinline__ void weights_rnode(int i, float a, float &w0, float &w1) {
  // E_z / E_phi / H_r radial part: i_r = CELL_NUMBER(r), volume CELL_VOLUME(i)
  // or CYL_VOL for r <= dr, and CELL_VOLUME(i+2) (src/eField.cpp:252-279)
  const float fi = (float)i;
  const float v1 = i >= 1 ? 2.0f * fi : 0.25f;
  w0 = (1.0f - a) * (2.0f * fi + a) / v1;
  w1 = a * (2.0f * fi + 1.0f + a) / (2.0f * (fi + 2.0f));
}

__device__ __forceinline__ void weights_zhalf(int k, float b, int &kz, float &w0, float &w1) {
  kz = b > 0.5f ? k : k - 1;
  if (kz < 0) kz = 0;
  w0 = (float)(kz - k) + 1.5f - b;
  w1 = (float)(k - kz) + b - 0.5f;
}

// f: the FP32 copy of the component (GridDev::e32 / hh32), the same values
// the FP64 grid rounds to.  No bounds test: the caller gathers only for a
// valid cell (0 <= i <= n_grid_r-2, 0 <= k <= n_grid_z-2), and every ir, kz
// it passes is i or k, or one less clamped at 0, so the four nodes lie in the
// grid.
__device__ __forceinline__ float gather4(const GridDev &g, const float *__restrict__ f, int ir,
                                         int kz, float wr0, float wr1, float wz0, float wz1) {
  const float f00 = __ldg(f + GIDX(ir, kz)), f10 = __ldg(f + GIDX(ir + 1, kz));
  const float f01 = __ldg(f + GIDX(ir, kz + 1));
  const float f11 = __ldg(f + GIDX(ir + 1, kz + 1));
  return wz0 * (f00 * wr0 + f10 * wr1) + wz1 * (f01 * wr0 + f11 * wr1);
}

// The same from the cell's packed quad (GridDev::q32): one 16-byte load.
__device__ __forceinline__ float gather_quad(const float4 *__restrict__ q, float wr0, float wr1,
                                             float wz0, float wz1) {
  const float4 v = __ldg(q);
  return wz0 * (v.x * wr0 + v.y * wr1) + wz1 * (v.z * wr0 + v.w * wr1);
}


// Per-warp staging of a warp chunk in shared memory: element e of the chunk
// (particle base + e, lane e / F32_PER_LANE's j-th particle with
// j = e % F32_PER_LANE) sits at slot j * 32 + e / F32_PER_LANE, so a lane
// reads its j-th particle at j * 32 + lane and the 16-byte loads and stores
// of a lane's consecutive elements land on consecutive slots across the
// warp: both are free of bank conflicts.  Results overwrite the particle's
// own slots.
struct WarpStage {
  int cell[F32_WARP_CHUNK];
  float fr[F32_WARP_CHUNK], fz[F32_WARP_CHUNK];
  float ur[F32_WARP_CHUNK], uphi[F32_WARP_CHUNK], uz[F32_WARP_CHUNK];
  float w[F32_WARP_CHUNK];
  uint8_t alive[F32_WARP_CHUNK];
};

// Shared memory of one CTA of the FP32 particle phase.
struct F32Shared {
  WarpStage stage[F32_WARPS];
};

static_assert(F32_PER_LANE % 4 == 0, "16-byte staging loads");
constexpr int F32_Q = F32_PER_LANE / 4;  // 16-byte vectors per lane and array

template <typename T>
__device__ __forceinline__ void stage_in(T *dst, const T *src, long long base, long long n,
                                         int lane) {
  const long long e0 = base + F32_PER_LANE * lane;
  if (base + F32_WARP_CHUNK <= n && ((uintptr_t)(src + base) & 15) == 0) {
#pragma unroll
    for (int q = 0; q < F32_Q; q++) {
      const int4 v = reinterpret_cast<const int4 *>(src + base)[F32_Q * lane + q];
      dst[(4 * q + 0) * 32 + lane] = reinterpret_cast<const T &>(v.x);
      dst[(4 * q + 1) * 32 + lane] = reinterpret_cast<const T &>(v.y);
      dst[(4 * q + 2) * 32 + lane] = reinterpret_cast<const T &>(v.z);
      dst[(4 * q + 3) * 32 + lane] = reinterpret_cast<const T &>(v.w);
    }
  } else {
#pragma unroll
    for (int j = 0; j < F32_PER_LANE; j++) dst[32 * j + lane] = e0 + j < n ? src[e0 + j] : T();
  }
}

template <typename T>
__device__ __forceinline__ void stage_out(T *dst, const T *src, long long base, long long n,
                                          int lane) {
  const long long e0 = base + F32_PER_LANE * lane;
  if (base + F32_WARP_CHUNK <= n && ((uintptr_t)(dst + base) & 15) == 0) {
#pragma unroll
    for (int q = 0; q < F32_Q; q++) {
      int4 v;
      v.x = reinterpret_cast<const int &>(src[(4 * q + 0) * 32 + lane]);
      v.y = reinterpret_cast<const int &>(src[(4 * q + 1) * 32 + lane]);
      v.z = reinterpret_cast<const int &>(src[(4 * q + 2) * 32 + lane]);
      v.w = reinterpret_cast<const int &>(src[(4 * q + 3) * 32 + lane]);
      reinterpret_cast<int4 *>(dst + base)[F32_Q * lane + q] = v;
    }
  } else {
#pragma unroll
    for (int j = 0; j < F32_PER_LANE; j++)
      if (e0 + j < n) dst[e0 + j] = src[32 * j + lane];
  }
}

// One warp chunk (F32_WARP_CHUNK consecutive particles of species s, lane l
// taking particles 4 l .. 4 l + 3 in order): push, deposit and store.  Each
// lane keeps running sums of its particles' deposits while their key (cell)
// stays the same, and the warp adds the lanes' sums up with one segmented
// reduction per chunk before the FP64 atomics.
// OUT = false: the step in place (o unused); OUT = true: results go to o.
// QUAD: gather from the packed quads (GridDev::q32) instead of the node
// copies (the persistent ensemble kernel, which does not pack them).
template <bool OUT, int PUSHER, bool QUAD>
__device__ __forceinline__ void f32_warp_chunk(const GridDev &g, const SpeciesF32 &s,
                                               const SpeciesOut &o, int pusher_rt,
                                               long long wchunk, WarpStage &ws) {
  // PUSHER >= 0 fixes the pusher at compile time (one kernel per pusher keeps
  // the code small); -1 takes it from pusher_rt
  const int pusher = PUSHER >= 0 ? PUSHER : pusher_rt;
  const int lane = threadIdx.x & 31;
  const int ncz = g.nz - 1;
  const long long base = wchunk * F32_WARP_CHUNK;
  if (base >= s.n) return;
  const bool has_alive = s.alive != nullptr;
  // cells per radial row a power of two (every benchmarked grid): the cell
  // index splits into (i, k) by a shift and a mask
  const bool row_pow2 = (ncz & (ncz - 1)) == 0;
  const int row_shift = __ffs(ncz) - 1;
  // OUT: the chunk is staged in shared memory and written out whole (slots
  // of skipped particles carry their input over); in place: each particle
  // is read and written where it lies (a lane's four consecutive particles
  // share 16-byte segments, which L1 keeps between the lane's four passes)
  constexpr bool STAGE = OUT;
  if (STAGE) {
    stage_in(ws.cell, s.cell, base, s.n, lane);
    stage_in(ws.fr, s.fr, base, s.n, lane);
    stage_in(ws.fz, s.fz, base, s.n, lane);
    stage_in(ws.ur, s.ur, base, s.n, lane);
    stage_in(ws.uphi, s.uphi, base, s.n, lane);
    stage_in(ws.uz, s.uz, base, s.n, lane);
    stage_in(ws.w, s.w, base, s.n, lane);
  }
  if (STAGE && has_alive) {
#pragma unroll
    for (int j = 0; j < F32_PER_LANE; j++) {
      const long long e = base + F32_PER_LANE * lane + j;
      ws.alive[32 * j + lane] = e < s.n ? s.alive[e] : 0;
    }
  }
  __syncwarp();
  RunAcc acc_phi, acc_rz;
  acc_phi.key = -1;
  acc_rz.key = -1;
#pragma unroll
  for (int j = 0; j < 4; j++) acc_phi.v[j] = acc_rz.v[j] = 0.0f;
#pragma unroll 1
  for (int jp = 0; jp < F32_PER_LANE; jp++) {
    const int slot = 32 * jp + lane;
    const long long p = base + F32_PER_LANE * lane + jp;
    bool live = p < s.n;
    if (live && has_alive && !(STAGE ? ws.alive[slot] : s.alive[p])) live = false;
    int c = live ? (STAGE ? ws.cell[slot] : s.cell[p]) : 0;
    if (live && (c < 0 || c >= (g.nr - 1) * ncz)) {
      flag32(g, ERR_OUT_OF_GRID);
      live = false;
    }
    // otherwise c / ncz through the FP32 reciprocal (exact for c < 2^24),
    // corrected to the exact quotient
    int i;
    if (row_pow2) {
      i = c >> row_shift;
    } else if (c < (1 << 24)) {
      i = (int)((float)c * (1.0f / (float)ncz));
      if (i * ncz > c) i--;
      if ((i + 1) * ncz <= c) i++;
    } else {
      i = c / ncz;
    }
    const int k = c - i * ncz;
    if (live) {
      const float a = STAGE ? ws.fr[slot] : s.fr[p], b = STAGE ? ws.fz[slot] : s.fz[p];
      float u[3];
      if (STAGE) {
        u[0] = ws.ur[slot];
        u[1] = ws.uphi[slot];
        u[2] = ws.uz[slot];
      } else {
        u[0] = s.ur[p];
        u[1] = s.uphi[p];
        u[2] = s.uz[p];
      }
      const float w = STAGE ? ws.w[slot] : s.w[p];
      // ---- gather E (time n) and H (time n+1/2)
      int ir_h, kz_h;
      float wrh0, wrh1, wrn0, wrn1, wzh0, wzh1;
      weights_rhalf(i, a, ir_h, wrh0, wrh1);
      weights_rnode(i, a, wrn0, wrn1);
      weights_zhalf(k, b, kz_h, wzh0, wzh1);
      const float wzn0 = 1.0f - b, wzn1 = b;
      const int ir_n = i, kz_n = k;
      float e[3], h[3];
      if (QUAD) {
        // quads of the cells (ir, kz): the particle's own cell c for the
        // node weights, one row (ncz) and/or one column lower for the half
        // weights when the particle sits in the lower half
        const size_t ncells = (size_t)(g.nr - 1) * (size_t)ncz;
        const unsigned q_nn = (unsigned)c, q_hn = q_nn - (unsigned)(i - ir_h) * (unsigned)ncz;
        const unsigned q_nh = q_nn - (unsigned)(k - kz_h), q_hh = q_hn - (unsigned)(k - kz_h);
        e[0] = gather_quad(g.q32 + q_hn, wrh0, wrh1, wzn0, wzn1);
        e[1] = gather_quad(g.q32 + ncells + q_nn, wrn0, wrn1, wzn0, wzn1);
        e[2] = gather_quad(g.q32 + 2 * ncells + q_nh, wrn0, wrn1, wzh0, wzh1);
        h[0] = gather_quad(g.q32 + 3 * ncells + q_nh, wrn0, wrn1, wzh0, wzh1);
        h[1] = gather_quad(g.q32 + 4 * ncells + q_hh, wrh0, wrh1, wzh0, wzh1);
        h[2] = gather_quad(g.q32 + 5 * ncells + q_hn, wrh0, wrh1, wzn0, wzn1);
      } else {
        const size_t ng = (size_t)g.nr * g.nz;
        e[0] = gather4(g, g.e32, ir_h, kz_n, wrh0, wrh1, wzn0, wzn1);
        e[1] = gather4(g, g.e32 + ng, ir_n, kz_n, wrn0, wrn1, wzn0, wzn1);
        e[2] = gather4(g, g.e32 + 2 * ng, ir_n, kz_h, wrn0, wrn1, wzh0, wzh1);
        h[0] = gather4(g, g.hh32, ir_n, kz_h, wrn0, wrn1, wzh0, wzh1);
        h[1] = gather4(g, g.hh32 + ng, ir_h, kz_h, wrh0, wrh1, wzh0, wzh1);
        h[2] = gather4(g, g.hh32 + 2 * ng, ir_h, kz_n, wrh0, wrh1, wzn0, wzn1);
      }
      // ---- push
      float inv_g = 1.0f;
      if (pusher == 1) {
        // Vay as the upstream code writes it (src/particles.cpp:1152-1254), in
        // SI velocity units (gamma v in m/s) because its alpha/us2 terms mix
        // units and so depend on them.
        const float C = (float)LIGHT_SPEED;
        float vel[3] = {u[0] * C, u[1] * C, u[2] * C};
        float ee[3], bb[3], vt[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
          ee[j] = e[j] * s.vay_e;
          bb[j] = h[j] * s.vay_b;
          vt[j] = vel[j];
          vel[j] += ee[j];
        }
        float gm = rsqrtf(1.0f + (vt[0] * vt[0] + vt[1] * vt[1] + vt[2] * vt[2]) * s.inv_c2);
        vel[0] += gm * (vt[1] * bb[2] - vt[2] * bb[1]);
        vel[1] += gm * (vt[2] * bb[0] - vt[0] * bb[2]);
        vel[2] += gm * (vt[0] * bb[1] - vt[1] * bb[0]);
        gm = rsqrtf(1.0f + (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]) * s.inv_c2);
        float alpha = 1.0f / gm / gm;
        const float B2 = bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2];
        float sg = alpha - B2;
        const float vb = vel[0] * bb[0] + vel[1] * bb[1] + vel[2] * bb[2];
        alpha = rsqrtf(0.5f * (sg + sqrtf(sg * sg + 4.0f * (B2 + vb * vb))));
#pragma unroll
        for (int j = 0; j < 3; j++) bb[j] *= alpha;
        sg = 1.0f / (1.0f + bb[0] * bb[0] + bb[1] * bb[1] + bb[2] * bb[2]);
        alpha = vel[0] * bb[0] + vel[1] * bb[1] + vel[2] * bb[2];
        vt[0] = sg * (vel[0] + alpha * bb[0] + bb[2] * vel[1] - bb[1] * vel[2]);
        vt[1] = sg * (vel[1] + alpha * bb[1] + bb[0] * vel[2] - bb[2] * vel[0]);
        vt[2] = sg * (vel[2] + alpha * bb[2] + bb[1] * vel[0] - bb[0] * vel[1]);
#pragma unroll
        for (int j = 0; j < 3; j++) u[j] = vt[j] / C;
        inv_g = rsqrtf(1.0f + u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      } else {
        // Boris (src/particles.cpp:1025-1150) on u = gamma v / c
        float um[3];
#pragma unroll
        for (int j = 0; j < 3; j++) um[j] = u[j] + s.ke * e[j];
        const float gi = pusher == 0 ? rsqrtf(1.0f + um[0] * um[0] + um[1] * um[1] + um[2] * um[2])
                                     : 1.0f;
        float tb[3];
#pragma unroll
        for (int j = 0; j < 3; j++) tb[j] = s.kb * h[j] * gi;
        const float c2 = 2.0f / (1.0f + tb[0] * tb[0] + tb[1] * tb[1] + tb[2] * tb[2]);
        const float w0 = um[0] + (um[1] * tb[2] - um[2] * tb[1]);
        const float w1 = um[1] + (um[2] * tb[0] - um[0] * tb[2]);
        const float w2 = um[2] + (um[0] * tb[1] - um[1] * tb[0]);
        u[0] = um[0] + c2 * (w1 * tb[2] - w2 * tb[1]) + s.ke * e[0];
        u[1] = um[1] + c2 * (w2 * tb[0] - w0 * tb[2]) + s.ke * e[1];
        u[2] = um[2] + c2 * (w0 * tb[1] - w1 * tb[0]) + s.ke * e[2];
        inv_g = pusher == 0 ? rsqrtf(1.0f + u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) : 1.0f;
      }
      if (!(inv_g == inv_g)) flag32(g, ERR_NAN);
      // ---- first half move and rz rotation (cells of r and z units)
      const float dr_h = u[0] * inv_g * s.cr, dy = u[1] * inv_g * s.cr;
      const float dz_h = u[2] * inv_g * s.cz;
      float xa = a + dr_h;
      float x = (float)i + xa;
      float rr = sqrtf(x * x + dy * dy);
      float a1 = xa + (x > 0.0f ? dy * dy / (x + rr) : rr - x);
      float b1 = b + dz_h;
      // ---- azimuthal current at the mid-step position (src/particles.cpp:688-784)
      {
        int i1 = i, k1 = k;
        float f1 = a1, g1 = b1;
        renorm(i1, f1);
        renorm(k1, g1);
        const float fi1 = (float)i1;
        const float rho1 = fi1 + f1;
        const float v1 = i1 >= 1 ? 2.0f * fi1 : 0.25f;
        const float wa = (1.0f - f1) * (2.0f * fi1 + f1) / (rho1 * v1);
        const float wb = f1 * (2.0f * fi1 + 1.0f + f1) / (rho1 * 2.0f * (fi1 + 1.0f));
        const float pref = s.kphi * w * u[1] * inv_g;
        const float vphi4[4] = {pref * (1.0f - g1) * wa, pref * (1.0f - g1) * wb,
                                pref * g1 * wa, pref * g1 * wb};
        acc_add<0>(g, acc_phi, i1 * g.nz + k1, vphi4);
      }
      // ---- second half move, walls, rz rotation (src/particles.cpp:1355-1365)
      float xa2 = a1 + dr_h;
      float b2 = b1 + dz_h;
      bool alive_now = true;
      const float wr_rel = (float)(g.nr - 1) - 0.5f - (float)i;
      const float wz_rel = (float)(g.nz - 1) - 0.5f - (float)k;
      if (s.kind == KIND_PLASMA) {
        if (xa2 > wr_rel) { xa2 = 2.0f * wr_rel - xa2; u[0] = -u[0]; }
        if (b2 > wz_rel) { b2 = 2.0f * wz_rel - b2; u[2] = -u[2]; }
      } else {
        if (xa2 > wr_rel) alive_now = false;
        if (b2 > wz_rel) alive_now = false;
      }
      if (xa2 < 0.5f - (float)i) { xa2 = 1.0f - 2.0f * (float)i - xa2; u[0] = -u[0]; }
      if (b2 < 0.5f - (float)k) { b2 = 1.0f - 2.0f * (float)k - b2; u[2] = -u[2]; }
      const float x2 = (float)i + xa2;
      const float r2 = sqrtf(x2 * x2 + dy * dy);
      float an = xa2 + (x2 > 0.0f ? dy * dy / (x2 + r2) : r2 - x2);
      float bn = b2;
      int in = i, kn = k;
      renorm(in, an);
      renorm(kn, bn);
      if (alive_now) {
        if (in == i && kn == k) {
          // the step stays in its cell (all but about one particle-step in
          // a thousand at thermal speeds): the one piece deposit_path would
          // make, without its face-crossing logic, into the running sums
          float vrz4[4];
          piece_values(i, a, b, an, bn, s.kz * w, s.kr * w, vrz4);
          acc_add<1>(g, acc_rz, i * g.nz + k, vrz4);
        } else {
          deposit_path(g.jr, g.jz, g.err, g.nr, g.nz, i, a, k, b, in, an, kn, bn, s.kz * w,
                       s.kr * w);
        }
        // back_velocity_to_rz (src/particles.cpp:1005-1015): cos = x/r, sin = y/r
        const float inv_r2 = 1.0f / r2;
        const float st = dy * inv_r2, ct = x2 * inv_r2;
        const float u0 = ct * u[0] - st * u[1];
        const float u1 = st * u[0] + ct * u[1];
        u[0] = u0;
        u[1] = u1;
      }
      if (has_alive) {
        if (STAGE)
          ws.alive[slot] = alive_now ? 1 : 0;
        else
          s.alive[p] = alive_now ? 1 : 0;
      }
      if (in > g.nr - 2 || kn > g.nz - 2) {
        flag32(g, ERR_OUT_OF_GRID);
        in = min(in, g.nr - 2);
        kn = min(kn, g.nz - 2);
      }
      if (STAGE) {
        ws.cell[slot] = in * ncz + kn;
        ws.fr[slot] = an;
        ws.fz[slot] = bn;
        ws.ur[slot] = u[0];
        ws.uphi[slot] = u[1];
        ws.uz[slot] = u[2];
      } else {
        s.cell[p] = in * ncz + kn;
        s.fr[p] = an;
        s.fz[p] = bn;
        s.ur[p] = u[0];
        s.uphi[p] = u[1];
        s.uz[p] = u[2];
      }
    }
  }
  warp_run_deposit<0>(g, acc_phi);
  warp_run_deposit<1>(g, acc_rz);
  if (!STAGE) return;
  __syncwarp();
  // particles skipped above (dead, not yet injected) keep their staged state
  int *cell_o = OUT ? o.cell : s.cell;
  float *fr_o = OUT ? o.fr : s.fr, *fz_o = OUT ? o.fz : s.fz;
  float *ur_o = OUT ? o.ur : s.ur, *uphi_o = OUT ? o.uphi : s.uphi, *uz_o = OUT ? o.uz : s.uz;
  stage_out(cell_o, ws.cell, base, s.n, lane);
  stage_out(fr_o, ws.fr, base, s.n, lane);
  stage_out(fz_o, ws.fz, base, s.n, lane);
  stage_out(ur_o, ws.ur, base, s.n, lane);
  stage_out(uphi_o, ws.uphi, base, s.n, lane);
  stage_out(uz_o, ws.uz, base, s.n, lane);
  if (has_alive) {
    uint8_t *alive_o = OUT ? o.alive : s.alive;
#pragma unroll
    for (int j = 0; j < F32_PER_LANE; j++) {
      const long long e = base + F32_PER_LANE * lane + j;
      if (e < s.n) alive_o[e] = ws.alive[32 * j + lane];
    }
  }
  __syncwarp();
}

// One CTA chunk of F32_CHUNK consecutive particles: warp w takes the w-th
// warp chunk.  No CTA-wide synchronisation: warps are independent.
template <bool OUT, int PUSHER = -1, bool QUAD = true>
__device__ __forceinline__ void f32_chunk(const GridDev &g, const SpeciesF32 &s,
                                          const SpeciesOut &o, int pusher, long long chunk,
                                          F32Shared &sm) {
  const int warp = threadIdx.x >> 5;
  f32_warp_chunk<OUT, PUSHER, QUAD>(g, s, o, pusher, chunk * F32_WARPS + warp, sm.stage[warp]);
}

}  // namespace pdp3g
