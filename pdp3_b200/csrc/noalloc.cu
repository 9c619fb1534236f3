// Allocation-free variant of the grid diagnostics (field energy, Gauss-law
// residual, total charge) for callers that cannot allocate device memory:
// code running while a CUDA graph is being captured, under a framework
// whose caching allocator owns every device byte, or in an embedding host
// that forbids cudaMalloc/cudaFree after start-up.  Such a caller passes
// device pointers it already holds; this entry point makes no allocation
// of its own, through the CUDA runtime or any library.
//
// Its scratch (one partial sum triple per chunk of the grid) lives in a
// file-scope __device__ array of fixed size, which every GPU that loads
// this library keeps until the process exits.  All calls share it.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/pdp3g.h"
#include "pdp3g_internal.cuh"

namespace pdp3g {
namespace {

constexpr int NA_THREADS = 256;
constexpr long long NA_CHUNK = 4096;      // grid nodes summed by one block
constexpr int NA_MAX_CHUNKS = 4096;       // scratch capacity, in chunks
constexpr int NA_MAX_DEVICES = 64;

// 4096 chunks x 3 partial sums x 8 B = 96 KiB per device.
static __device__ __align__(256) double g_noalloc_scratch[NA_MAX_CHUNKS * 3];

std::mutex g_setup_mutex;
// The array's address is looked up per device and per context: after a
// cudaDeviceReset, or with a non-primary context current, the module is
// loaded again and the array may sit elsewhere.
double *g_scratch_addr[NA_MAX_DEVICES] = {nullptr};
CUcontext g_scratch_ctx[NA_MAX_DEVICES] = {nullptr};
typedef CUresult (*ctx_get_current_fn)(CUcontext *);
ctx_get_current_fn g_ctx_get_current = nullptr;

// Block b sums nodes [b*NA_CHUNK, (b+1)*NA_CHUNK) and writes its three
// partial sums to scratch[3b .. 3b+2].  The per-node terms are those of
// pdp3g_diagnostics: 1/2 (eps0 E^2 + mu0 H^2) dV, the squared Gauss
// residual eps0 div E - (rho - rho0) on the interior nodes whose divergence
// stencil has sigma == 0 (node (i,k) and the nodes (i-1,k), (i,k-1)), and
// rho dV.
__global__ void __launch_bounds__(NA_THREADS)
    k_field_diag_chunks(const double *er, const double *ephi, const double *ez,
                        const double *hr, const double *hphi, const double *hz,
                        const double *rho, const double *rho0, const double *sigma, int nr,
                        int nz, double dr, double dz, double *scratch) {
  const long long total = (long long)nr * nz;
  const long long begin = (long long)blockIdx.x * NA_CHUNK;
  const long long end = begin + NA_CHUNK < total ? begin + NA_CHUNK : total;
  double v[3] = {0, 0, 0};
  for (long long t = begin + threadIdx.x; t < end; t += blockDim.x) {
    const int i = (int)(t / nz), k = (int)(t - (long long)i * nz);
    const double vol = i == 0 ? PI * dz * dr * dr / 4. : 2.0 * PI * dz * dr * dr * i;
    const double e2 = er[t] * er[t] + ephi[t] * ephi[t] + ez[t] * ez[t];
    const double h2 = hr[t] * hr[t] + hphi[t] * hphi[t] + hz[t] * hz[t];
    v[0] += 0.5 * (EPSILON0 * e2 + MAGN_CONST * h2) * vol;
    v[2] += rho[t] * vol;
    // nodes whose whole divergence stencil is updated without damping
    if (i >= 2 && i <= nr - 3 && k >= 2 && k <= nz - 3 && sigma[t] == 0.0 &&
        sigma[t - nz] == 0.0 && sigma[t - 1] == 0.0) {
      const double div = (er[t] * (i + 0.5) - er[t - nz] * (i - 0.5)) / (i * dr) +
                         (ez[t] - ez[t - 1]) / dz;
      const double res = EPSILON0 * div - (rho[t] - (rho0 ? rho0[t] : 0.0));
      v[1] += res * res;
    }
  }
  __shared__ double sh[3][NA_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    double x = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sh[j][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0;
    for (int w = 0; w < NA_THREADS / 32; w++) s += sh[threadIdx.x][w];
    scratch[(size_t)blockIdx.x * 3 + threadIdx.x] = s;
  }
}

// One block adds the chunk partials in chunk order; out = {field energy,
// sqrt(sum res^2), sum rho dV}.
__global__ void k_field_diag_finish(const double *scratch, int chunks, double *out) {
  __shared__ double sh[NA_THREADS];
  for (int j = 0; j < 3; j++) {
    double s = 0;
    for (int b = threadIdx.x; b < chunks; b += blockDim.x) s += scratch[(size_t)b * 3 + j];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[j] = j == 1 ? sqrt(sh[0]) : sh[0];
    __syncthreads();
  }
}

// Device address of the scratch array on the current device, looked up once
// per device and context (the array's name is only a host-side stand-in in
// host code).  The driver's cuCtxGetCurrent is reached through the runtime's
// entry-point query, so the library keeps no link-time dependency on libcuda.
cudaError_t scratch_address(int device, double **ptr) {
  if (device < 0 || device >= NA_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_ctx_get_current == nullptr) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || fn == nullptr) return cudaErrorSymbolNotFound;
    g_ctx_get_current = (ctx_get_current_fn)fn;
  }
  CUcontext cur = nullptr;
  if (g_ctx_get_current(&cur) != CUDA_SUCCESS) return cudaErrorContextIsDestroyed;
  if (g_scratch_addr[device] == nullptr || cur == nullptr || g_scratch_ctx[device] != cur) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    // the runtime makes the primary context current if none was
    if (cur == nullptr && g_ctx_get_current(&cur) != CUDA_SUCCESS) return cudaErrorContextIsDestroyed;
    g_scratch_addr[device] = (double *)p;
    g_scratch_ctx[device] = cur;
  }
  *ptr = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace
}  // namespace pdp3g

extern "C" pdp3g_status pdp3g_field_diagnostics_noalloc(
    const double *e_r, const double *e_phi, const double *e_z, const double *h_r,
    const double *h_phi, const double *h_z, const double *rho, const double *rho0,
    const double *sigma, int32_t n_grid_r, int32_t n_grid_z, double r_size, double z_size,
    double *out, void *stream) {
  using namespace pdp3g;
  if (!e_r || !e_phi || !e_z || !h_r || !h_phi || !h_z || !rho || !sigma || !out) {
    fprintf(stderr, "pdp3g_field_diagnostics_noalloc: null device pointer\n");
    return PDP3G_INVALID_ARG;
  }
  if (n_grid_r < 3 || n_grid_z < 3 || !(r_size > 0) || !(z_size > 0)) {
    fprintf(stderr, "pdp3g_field_diagnostics_noalloc: grid must be at least 3 x 3 nodes "
                    "with positive extents\n");
    return PDP3G_INVALID_ARG;
  }
  const long long nodes = (long long)n_grid_r * n_grid_z;
  const long long chunks = (nodes + NA_CHUNK - 1) / NA_CHUNK;
  if (chunks > NA_MAX_CHUNKS) {
    fprintf(stderr,
            "pdp3g_field_diagnostics_noalloc: %lld grid nodes exceed the maximum of %lld "
            "(%d chunks of %lld nodes of static scratch)\n",
            nodes, (long long)NA_MAX_CHUNKS * NA_CHUNK, NA_MAX_CHUNKS, NA_CHUNK);
    return PDP3G_INVALID_ARG;
  }
  // an error left pending by the caller's own earlier work is reported and
  // left in place for the caller's check; nothing is launched
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    fprintf(stderr, "pdp3g_field_diagnostics_noalloc: a CUDA error was pending before the "
                    "call (%s); nothing launched\n", cudaGetErrorString(pending));
    return PDP3G_CUDA_ERROR;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return PDP3G_CUDA_ERROR;
  double *scratch = nullptr;
  if (scratch_address(device, &scratch) != cudaSuccess) return PDP3G_CUDA_ERROR;
  const double dr = r_size / (n_grid_r - 1);  // src/geometry.cpp:45-53
  const double dz = z_size / (n_grid_z - 1);
  cudaStream_t st = (cudaStream_t)stream;
  k_field_diag_chunks<<<(int)chunks, NA_THREADS, 0, st>>>(e_r, e_phi, e_z, h_r, h_phi, h_z, rho,
                                                          rho0, sigma, n_grid_r, n_grid_z, dr,
                                                          dz, scratch);
  if (cudaGetLastError() != cudaSuccess) return PDP3G_CUDA_ERROR;
  k_field_diag_finish<<<1, NA_THREADS, 0, st>>>(scratch, (int)chunks, out);
  return cudaGetLastError() == cudaSuccess ? PDP3G_OK : PDP3G_CUDA_ERROR;
}
