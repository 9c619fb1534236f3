// Stable integer sort of particles by cell: a least-significant-digit radix
// sort of (cell, index) pairs with 8-bit digits, followed by a gather of
// every particle array through the resulting permutation.
//
// Stability and determinism: every pass splits the items into fixed
// sub-ranges of SUB consecutive items, one per warp; a warp walks its
// sub-range in order, ranking equal digits inside each 32-item step with
// __match_any_sync and carrying per-digit running counts, and the
// destination of sub-range s's items with digit d starts at the exclusive
// scan of the digit-major count table H[d][s].  No atomic whose order could
// vary decides a position, so the permutation is exactly the stable sort of
// the keys (numpy.argsort(kind="stable")).
//
// Traffic per pass: read key+index (8 B), write key+index (8 B) per particle,
// plus the count table; the gather reads the permutation once, reads the
// particle state in sorted order into scratch copies and copies them back.
#include "pdp3g_internal.cuh"

namespace pdp3g {

constexpr int SORT_WARPS = 8;                 // warps per CTA
constexpr int SORT_THREADS = SORT_WARPS * 32;
constexpr int SUB = 2048;                     // items per warp sub-range
constexpr int RADIX = 256;

// Each warp loads BATCH 32-item steps of its sub-range before it ranks them,
// so that BATCH loads per lane are in flight instead of one.
constexpr int BATCH = 8;
static_assert(SUB % (32 * BATCH) == 0, "a sub-range is whole batches");

// H[d * nsub + s] = number of items with digit d in sub-range s (shared
// memory atomics: the count does not depend on their order).
__global__ void __launch_bounds__(SORT_THREADS) k_digit_count(const unsigned *keys, long long n,
                                                              int shift, int nsub,
                                                              unsigned *H) {
  __shared__ unsigned cnt[SORT_WARPS][RADIX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int d = lane; d < RADIX; d += 32) cnt[warp][d] = 0;
  __syncwarp();
  const long long sub = (long long)blockIdx.x * SORT_WARPS + warp;
  if (sub < nsub) {
    const long long begin = sub * SUB;
    const long long end = begin + SUB < n ? begin + SUB : n;
    for (long long p0 = begin; p0 < end; p0 += 32 * BATCH) {
      unsigned d[BATCH];
#pragma unroll
      for (int j = 0; j < BATCH; j++) {
        const long long p = p0 + j * 32 + lane;
        d[j] = p < end ? (keys[p] >> shift) & (RADIX - 1) : RADIX;
      }
#pragma unroll
      for (int j = 0; j < BATCH; j++)
        if (d[j] < RADIX) atomicAdd(&cnt[warp][d[j]], 1u);
    }
    __syncwarp();
    for (int d = lane; d < RADIX; d += 32) H[(size_t)d * nsub + sub] = cnt[warp][d];
  }
}

// exclusive scan, three kernels: per-block sums, scan of the block sums, and
// the in-block scan plus the block's offset.
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;  // per thread
constexpr int SCAN_BLOCK = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ unsigned block_exclusive_scan(unsigned v, unsigned *total) {
  __shared__ unsigned warp_sums[SCAN_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    unsigned s = lane < SCAN_THREADS / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < SCAN_THREADS / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  const unsigned before = warp > 0 ? warp_sums[warp - 1] : 0;
  if (total) *total = warp_sums[SCAN_THREADS / 32 - 1];
  const unsigned excl = before + x - v;
  __syncthreads();
  return excl;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_sums(const unsigned *in, long long m,
                                                            unsigned *block_sums) {
  const long long base = (long long)blockIdx.x * SCAN_BLOCK + (long long)threadIdx.x * SCAN_ITEMS;
  unsigned v = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++)
    if (base + j < m) v += in[base + j];
  unsigned total = 0;
  block_exclusive_scan(v, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// one block: exclusive scan of nb block sums in place (nb <= SCAN_BLOCK * 64)
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_block_sums(unsigned *sums, int nb) {
  __shared__ unsigned carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += SCAN_BLOCK) {
    unsigned v[SCAN_ITEMS], s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; j++) {
      const int idx = base + threadIdx.x * SCAN_ITEMS + j;
      v[j] = idx < nb ? sums[idx] : 0;
      s += v[j];
    }
    unsigned total = 0;
    unsigned excl = block_exclusive_scan(s, &total) + carry;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; j++) {
      const int idx = base + threadIdx.x * SCAN_ITEMS + j;
      if (idx < nb) sums[idx] = excl;
      excl += v[j];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(unsigned *data, long long m,
                                                             const unsigned *block_offsets) {
  const long long base = (long long)blockIdx.x * SCAN_BLOCK + (long long)threadIdx.x * SCAN_ITEMS;
  unsigned v[SCAN_ITEMS], s = 0;
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    v[j] = base + j < m ? data[base + j] : 0;
    s += v[j];
  }
  unsigned excl = block_exclusive_scan(s, nullptr) + block_offsets[blockIdx.x];
#pragma unroll
  for (int j = 0; j < SCAN_ITEMS; j++) {
    if (base + j < m) data[base + j] = excl;
    excl += v[j];
  }
}

// stable scatter of (key, idx) by digit
__global__ void __launch_bounds__(SORT_THREADS) k_digit_scatter(
    const unsigned *keys_in, const unsigned *idx_in, long long n, int shift, int nsub,
    const unsigned *offsets, unsigned *keys_out, unsigned *idx_out) {
  __shared__ unsigned run[SORT_WARPS][RADIX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long sub = (long long)blockIdx.x * SORT_WARPS + warp;
  if (sub >= nsub) return;
  for (int d = lane; d < RADIX; d += 32) run[warp][d] = offsets[(size_t)d * nsub + sub];
  __syncwarp();
  const long long begin = sub * SUB;
  const long long end = begin + SUB < n ? begin + SUB : n;
  const unsigned below = (1u << lane) - 1u;
  for (long long p0 = begin; p0 < end; p0 += 32 * BATCH) {
    unsigned key[BATCH], id[BATCH];
#pragma unroll
    for (int j = 0; j < BATCH; j++) {
      const long long p = p0 + j * 32 + lane;
      key[j] = 0;
      id[j] = (unsigned)p;
      if (p < end) {
        key[j] = keys_in[p];
        if (idx_in) id[j] = idx_in[p];
      }
    }
    // the batch's steps in item order: ranks and runs as one step at a time
#pragma unroll
    for (int j = 0; j < BATCH; j++) {
      const bool valid = p0 + j * 32 + lane < end;
      const unsigned d = valid ? (key[j] >> shift) & (RADIX - 1) : RADIX;  // RADIX: no valid lane
      const unsigned peers = __match_any_sync(0xffffffffu, d);
      if (valid) {
        const unsigned pos = run[warp][d] + __popc(peers & below);
        keys_out[pos] = key[j];
        idx_out[pos] = id[j];
      }
      __syncwarp();
      // the highest lane of each digit group advances that digit's run
      if (valid && (peers >> lane) == 1u) run[warp][d] += __popc(peers);
      __syncwarp();
    }
  }
}

// cell key of every FP64 particle (CELL_NUMBER of r and z, clamped)
__global__ void k_keys_f64(SpeciesDev s, double dr, double dz, int nr, int nz, unsigned *keys) {
  const int ncz = nz - 1;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x) {
    int i = (int)ceil(s.r[p] / dr) - 1, k = (int)ceil(s.z[p] / dz) - 1;
    i = min(max(i, 0), nr - 2);
    k = min(max(k, 0), nz - 2);
    keys[p] = (unsigned)(i * ncz + k);
  }
}

__global__ void k_keys_f32(SpeciesF32 s, unsigned *keys) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < s.n;
       p += (long long)gridDim.x * blockDim.x)
    keys[p] = (unsigned)max(s.cell[p], 0);
}

template <typename T>
__global__ void k_gather(const T *src, const unsigned *perm, long long n, T *dst) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x)
    dst[p] = src[perm[p]];
}

// NA state arrays of one element type, gathered through one read of the
// permutation: dst.a[j][p] = src.a[j][perm[p]]
template <typename T, int NA>
struct ArraySet {
  T *a[NA];
};

template <typename T, int NA>
__global__ void __launch_bounds__(256) k_gather_set(ArraySet<T, NA> src,
                                                    const unsigned *__restrict__ perm,
                                                    long long n, ArraySet<T, NA> dst) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n;
       p += (long long)gridDim.x * blockDim.x) {
    const unsigned q = perm[p];
    T v[NA];
#pragma unroll
    for (int j = 0; j < NA; j++) v[j] = src.a[j][q];
#pragma unroll
    for (int j = 0; j < NA; j++) dst.a[j][p] = v[j];
  }
}

// ---------------------------------------------------------------- host side

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

SortLayout sort_layout(long long n, size_t state_bytes) {
  SortLayout L;
  const long long nsub = (n + SUB - 1) / SUB;
  L.nsub = nsub;
  L.m = nsub * RADIX;
  L.nb = (L.m + SCAN_BLOCK - 1) / SCAN_BLOCK;
  size_t off = 0;
  L.keys_a = off; off = align256(off + sizeof(unsigned) * (size_t)n);
  L.keys_b = off; off = align256(off + sizeof(unsigned) * (size_t)n);
  L.idx_a = off;  off = align256(off + sizeof(unsigned) * (size_t)n);
  L.idx_b = off;  off = align256(off + sizeof(unsigned) * (size_t)n);
  L.H = off;      off = align256(off + sizeof(unsigned) * (size_t)L.m);
  L.bs = off;     off = align256(off + sizeof(unsigned) * (size_t)L.nb);
  L.tmp = off;    off = align256(off + state_bytes * (size_t)n);
  L.total = off;
  return L;
}

static int grid_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

static int key_bits_for(long long ncells) {
  int b = 1;
  while (((long long)1 << b) < ncells) b++;
  return b;
}

// Stable sort of the keys at scratch + L.keys_a; returns the permutation
// (sorted position -> original index) inside scratch.  Launch count in *nl.
static const unsigned *radix_sort(char *scratch, const SortLayout &L, long long n, int key_bits,
                                  cudaStream_t st, int *nl) {
  unsigned *ka = (unsigned *)(scratch + L.keys_a), *kb = (unsigned *)(scratch + L.keys_b);
  unsigned *ia = (unsigned *)(scratch + L.idx_a), *ib = (unsigned *)(scratch + L.idx_b);
  unsigned *H = (unsigned *)(scratch + L.H), *bs = (unsigned *)(scratch + L.bs);
  unsigned *kin = ka, *kout = kb, *iin = nullptr, *iout = ia;
  const int sort_blocks = (int)((L.nsub + SORT_WARPS - 1) / SORT_WARPS);
  for (int shift = 0; shift < key_bits; shift += 8) {
    k_digit_count<<<sort_blocks, SORT_THREADS, 0, st>>>(kin, n, shift, (int)L.nsub, H);
    k_scan_sums<<<(int)L.nb, SCAN_THREADS, 0, st>>>(H, L.m, bs);
    k_scan_block_sums<<<1, SCAN_THREADS, 0, st>>>(bs, (int)L.nb);
    k_scan_apply<<<(int)L.nb, SCAN_THREADS, 0, st>>>(H, L.m, bs);
    k_digit_scatter<<<sort_blocks, SORT_THREADS, 0, st>>>(kin, iin, n, shift, (int)L.nsub, H,
                                                          kout, iout);
    *nl += 5;
    unsigned *t = kin;
    kin = kout;
    kout = t;
    iin = iout;
    iout = (iout == ia) ? ib : ia;
  }
  return iin;
}

// the sorted order of NA arrays: gathered into the scratch copies through
// one read of the permutation, then copied back in place
template <typename T, int NA>
static void permute_set(T *const (&arr)[NA], const unsigned *perm, long long n, char *tmp,
                        cudaStream_t st, int *nl) {
  ArraySet<T, NA> src, dst;
  for (int j = 0; j < NA; j++) {
    src.a[j] = arr[j];
    dst.a[j] = (T *)tmp + (size_t)j * n;
  }
  k_gather_set<T, NA><<<grid_for(n, 256), 256, 0, st>>>(src, perm, n, dst);
  *nl += 1;
  for (int j = 0; j < NA; j++)
    cudaMemcpyAsync(arr[j], dst.a[j], sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, st);
}

static void permute_alive(uint8_t *alive, const unsigned *perm, long long n, char *tmp,
                          cudaStream_t st, int *nl) {
  k_gather<uint8_t><<<grid_for(n, 256), 256, 0, st>>>(alive, perm, n, (uint8_t *)tmp);
  cudaMemcpyAsync(alive, tmp, (size_t)n, cudaMemcpyDeviceToDevice, st);
  *nl += 1;
}

int sort_species_f64(const GridDev &g, SpeciesDev &s, char *scratch, cudaStream_t st) {
  const long long n = s.n;
  if (n <= 1) return 0;
  const SortLayout L = sort_layout(n, SORT_STATE_F64);
  int nl = 1;
  k_keys_f64<<<grid_for(n, 256), 256, 0, st>>>(s, g.dr, g.dz, g.nr, g.nz,
                                                (unsigned *)(scratch + L.keys_a));
  const int bits = key_bits_for((long long)(g.nr - 1) * (g.nz - 1));
  const unsigned *perm = radix_sort(scratch, L, n, bits, st, &nl);
  double *const arrays[6] = {s.r, s.z, s.vr, s.vphi, s.vz, (double *)s.w};
  permute_set(arrays, perm, n, scratch + L.tmp, st, &nl);
  if (s.alive) permute_alive(s.alive, perm, n, scratch + L.tmp, st, &nl);
  return nl;
}

int sort_species_f32(const GridDev &g, SpeciesF32 &s, char *scratch, cudaStream_t st) {
  const long long n = s.n;
  if (n <= 1) return 0;
  const SortLayout L = sort_layout(n, SORT_STATE_F32);
  int nl = 1;
  k_keys_f32<<<grid_for(n, 256), 256, 0, st>>>(s, (unsigned *)(scratch + L.keys_a));
  const int bits = key_bits_for((long long)(g.nr - 1) * (g.nz - 1));
  const unsigned *perm = radix_sort(scratch, L, n, bits, st, &nl);
  // the cell index and the FP32 values move as 32-bit words
  unsigned *const arrays[7] = {(unsigned *)s.cell, (unsigned *)s.fr,   (unsigned *)s.fz,
                               (unsigned *)s.ur,   (unsigned *)s.uphi, (unsigned *)s.uz,
                               (unsigned *)s.w};
  permute_set(arrays, perm, n, scratch + L.tmp, st, &nl);
  if (s.alive) permute_alive(s.alive, perm, n, scratch + L.tmp, st, &nl);
  return nl;
}

}  // namespace pdp3g
