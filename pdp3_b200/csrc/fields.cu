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
#include "fields_body.cuh"

namespace pdp3g {

// H update over i in [0, nr-1], k in [0, nz-2]
__global__ void __launch_bounds__(256) k_yee_h(GridDev g) {
  const int nz = g.nz;
  const long long total = (long long)g.nr * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1));
    yee_h_node(g, i, (int)(t - (long long)i * (nz - 1)));
  }
}

// E update over i in [0, nr-2], k in [0, nz-2]
__global__ void __launch_bounds__(256) k_yee_e(GridDev g) {
  const int nz = g.nz;
  const long long total = (long long)(g.nr - 1) * (nz - 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / (nz - 1));
    yee_e_node(g, i, (int)(t - (long long)i * (nz - 1)));
  }
}

__global__ void k_to_f32(const double *src, float *dst, size_t n) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x)
    dst[t] = (float)src[t];
}

// thread t = c * ncells + cell: the 2x2 nodes of the cell of component c
// (0-2 E_r, E_phi, E_z from e32; 3-5 the half-step H_r, H_phi, H_z from hh32)
__global__ void k_pack_quads(GridDev g, float4 *q) {
  const int nz = g.nz, ncz = nz - 1;
  const long long ng = (long long)g.nr * nz, ncells = (long long)(g.nr - 1) * ncz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * ncells;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / ncells);
    const long long cell = t - c * ncells;
    const int i = (int)(cell / ncz), k = (int)(cell - (long long)i * ncz);
    const float *f = (c < 3 ? g.e32 : g.hh32) + (c % 3) * ng + (long long)i * nz + k;
    q[t] = make_float4(__ldg(f), __ldg(f + nz), __ldg(f + 1), __ldg(f + nz + 1));
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

namespace pdp3g {
void launch_pack_quads(const GridDev &g, float4 *q, cudaStream_t st) {
  k_pack_quads<<<grid_blocks(6LL * (g.nr - 1) * (g.nz - 1)), 256, 0, st>>>(g, q);
}

void launch_to_f32(const double *src, float *dst, size_t n, cudaStream_t st) {
  long long b = ((long long)n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  k_to_f32<<<(int)b, 256, 0, st>>>(src, dst, n);
}
}  // namespace pdp3g
