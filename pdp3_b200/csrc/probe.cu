// Probe reads on the device (ProbePlain, src/probePlain.cpp:80-224): a grid
// component's values over a probe region in the order the upstream writes
// them, and the particles of a species inside a cell region (mpframe) in
// slot order, so a host fetches only what a probe prints.
#include "pdp3g_internal.cuh"

namespace pdp3g {

// type 0 frame: rows r0..r1-1, each z0..z1-1; 1 col: r0..r1-1 at z0;
// 2 row: z0..z1-1 at r0; 3 dot: (r0, z0)
__global__ void k_probe_gather(const double *f, int nz, int type, int r0, int z0, int r1, int z1,
                               long long n, double *out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    long long i = r0, k = z0;
    if (type == 0) {
      const long long w = z1 - z0;
      i = r0 + t / w;
      k = z0 + t % w;
    } else if (type == 1) {
      i = r0 + t;
    } else if (type == 2) {
      k = z0 + t;
    }
    out[t] = f[i * nz + k];
  }
}

void launch_probe_gather(const double *f, int nz, int type, int r0, int z0, int r1, int z1,
                         long long n, double *out, cudaStream_t st) {
  long long b = (n + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  if (b < 1) b = 1;
  k_probe_gather<<<(int)b, 256, 0, st>>>(f, nz, type, r0, z0, r1, z1, n, out);
}

// mpframe selection (src/probePlain.cpp:196-221): r_i = ceil(r/dr) - 1 and
// z_k = ceil(z/dz) - 1 with start <= index <= end (inclusive, unsigned, so a
// negative index never matches); every slot, alive or not, as upstream.
__device__ __forceinline__ bool mp_inside(double r, double z, double dr, double dz, int r0, int z0,
                                          int r1, int z1) {
  const int ri = (int)ceil(r / dr) - 1, zk = (int)ceil(z / dz) - 1;
  return (unsigned)ri >= (unsigned)r0 && (unsigned)ri <= (unsigned)r1 &&
         (unsigned)zk >= (unsigned)z0 && (unsigned)zk <= (unsigned)z1;
}

constexpr int MP_THREADS = 256;
constexpr int MP_ITEMS = 8;  // consecutive slots per thread
constexpr long long MP_BLOCK = (long long)MP_THREADS * MP_ITEMS;

// pass 1: selected slots per block of MP_BLOCK consecutive slots
__global__ void k_mp_count(const double *r, const double *z, long long n, double dr, double dz,
                           int r0, int z0, int r1, int z1, unsigned *counts) {
  __shared__ unsigned total;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  const long long base = blockIdx.x * MP_BLOCK + (long long)threadIdx.x * MP_ITEMS;
  unsigned c = 0;
  for (int j = 0; j < MP_ITEMS; j++) {
    const long long p = base + j;
    if (p < n && mp_inside(r[p], z[p], dr, dz, r0, z0, r1, z1)) c++;
  }
  atomicAdd(&total, c);
  __syncthreads();
  if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// pass 2: each block writes its selected slots in slot order from its offset
// (a block-wide exclusive scan of the per-thread counts)
__global__ void k_mp_write(MpArrays arr, long long n, double dr, double dz, int r0, int z0, int r1,
                           int z1, const unsigned long long *offsets) {
  const double *r = arr.src[0], *z = arr.src[1];
  __shared__ unsigned scan[MP_THREADS];
  const long long base = blockIdx.x * MP_BLOCK + (long long)threadIdx.x * MP_ITEMS;
  unsigned mine = 0;
  for (int j = 0; j < MP_ITEMS; j++) {
    const long long p = base + j;
    if (p < n && mp_inside(r[p], z[p], dr, dz, r0, z0, r1, z1)) mine++;
  }
  scan[threadIdx.x] = mine;
  __syncthreads();
  for (int o = 1; o < MP_THREADS; o <<= 1) {  // inclusive Hillis-Steele scan
    const unsigned v = threadIdx.x >= (unsigned)o ? scan[threadIdx.x - o] : 0u;
    __syncthreads();
    scan[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned long long pos = offsets[blockIdx.x] + scan[threadIdx.x] - mine;
  for (int j = 0; j < MP_ITEMS; j++) {
    const long long p = base + j;
    if (p < n && mp_inside(r[p], z[p], dr, dz, r0, z0, r1, z1)) {
      for (int a = 0; a < 5; a++) arr.dst[a][pos] = arr.src[a][p];
      pos++;
    }
  }
}

long long mp_blocks(long long n) { return (n + MP_BLOCK - 1) / MP_BLOCK; }

void launch_mp_count(const double *r, const double *z, long long n, double dr, double dz, int r0,
                     int z0, int r1, int z1, unsigned *counts, cudaStream_t st) {
  const long long b = mp_blocks(n);
  if (b > 0) k_mp_count<<<(unsigned)b, MP_THREADS, 0, st>>>(r, z, n, dr, dz, r0, z0, r1, z1, counts);
}

void launch_mp_write(const MpArrays &arr, long long n, double dr, double dz, int r0, int z0,
                     int r1, int z1, const unsigned long long *offsets, cudaStream_t st) {
  const long long b = mp_blocks(n);
  if (b > 0)
    k_mp_write<<<(unsigned)b, MP_THREADS, 0, st>>>(arr, n, dr, dz, r0, z0, r1, z1, offsets);
}

}  // namespace pdp3g
