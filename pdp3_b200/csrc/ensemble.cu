// Batched ensemble: many independent runs (different grids, species and
// bunches, FP32 cell-local form) advanced together by ONE persistent
// cooperative kernel per launch, replayed from a captured CUDA graph.
//
// Every step has three phases separated by grid-wide barriers:
//   A  bunch injection, H update and J clear of every run
//   B  push + deposition of every chunk of every species of every run
//   C  E update of every run, t += dt
// Work items are global index spaces (nodes of all runs, F32_CHUNK-particle
// chunks of all species) dealt to CTAs round-robin, so runs of very different sizes
// share the GPU without per-run launches.  Each run's step is the same as
// pdp3g_step on that run alone (same device functions, fields_body.cuh and
// particles_f32.cuh).
//
// Stop path: at the top of each step one thread reads a host-mapped cancel
// flag and compares clock64() with a cycle budget; the decision is published
// through device memory before the barrier, so every CTA leaves together and
// the kernel never spins on the host.
#include <cooperative_groups.h>

#include "fields_body.cuh"
#include "particles_f32.cuh"

namespace cg = cooperative_groups;

namespace pdp3g {

// Bunch::bunch_inject (src/bunch.cpp:87-124) for one bunch species, by one CTA
__device__ void ens_inject(const EnsembleDev &E, const EnsSpecies &sp) {
  const EnsRun &run = E.runs[sp.run];
  const double dt = run.g.dt, t = run.t;
  const double begin = sp.duration * sp.bunch_number + sp.hole_duration * sp.bunch_number;
  const double end = begin + sp.duration;
  const double dl = sp.velocity * dt;
  const int steps_amount = (int)ceil(sp.duration / dt);
  const unsigned number = (unsigned)sp.s.n;
  const unsigned particles_in_step = number / steps_amount;
  const int start_number = (t - begin) / dt * particles_in_step;
  if (!(t >= begin && t < end) || particles_in_step == 0) return;
  const long long start = (long long)(unsigned)start_number;
  const int ncz = run.g.nz - 1;
  const double dz = run.g.dz;
  for (long long j = threadIdx.x; j < particles_in_step; j += blockDim.x) {
    const long long idx = start + j;
    if (idx >= (long long)number) break;
    int int_vel = (int)floor((double)(unsigned)idx);
    double ost = 0, rr = 0;
    int order = 1;
    while (int_vel >= 1 && order < 40) {
      ost = int_vel % 11;
      rr = rr + ost * E.inv_pow11[order];
      int_vel = (int)((int_vel - ost) / 11);
      order = order + 1;
    }
    const double z = dl * rr + dz / 2.0;
    int k = (int)ceil(z / dz) - 1;
    k = max(0, min(k, ncz - 1));
    const int i = sp.s.cell[idx] / ncz;
    sp.s.cell[idx] = i * ncz + k;
    sp.s.fz[idx] = (float)(z / dz - k);
    sp.s.uz[idx] = sp.uz_beam;
    sp.s.alive[idx] = 1;
  }
}

// The step count is read from E.status[2] (written before each launch), so
// one captured graph serves every segment length.  PUSHER: the pusher of
// every run when they share one (compiled in, as in k_push_deposit_f32),
// -1 for runs with different pushers (chosen per species at run time).
template <int PUSHER>
__global__ void __launch_bounds__(F32_THREADS, F32_MIN_BLOCKS) k_ensemble(EnsembleDev E) {
  const int nsteps = *(volatile int *)&E.status[2];
  cg::grid_group grid = cg::this_grid();
  __shared__ F32Shared sm;
  __shared__ struct {
    GridDev g;
    SpeciesF32 s;
    int pusher;
  } desc;
  // thread 0 alone tests the cancel flag and the budget: its start clock
  // lives in shared memory, not in every thread's registers
  __shared__ long long t_start_sh;
  if (threadIdx.x == 0) t_start_sh = clock64();
  for (int step = 0; step < nsteps; step++) {
    const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long gstride = (long long)gridDim.x * blockDim.x;
    if (gtid == 0) {
      int stop = 0;
      const long long budget = *(volatile const long long *)E.budget_cycles;
      if (*E.cancel) stop = 1;
      else if (budget > 0 && clock64() - t_start_sh > budget) stop = 2;
      E.status[1] = stop;
      __threadfence();
    }
    grid.sync();
    if (*(volatile int *)&E.status[1] != 0) return;
    // ---- phase A: injection, H update, J clear
    for (int sp = blockIdx.x; sp < E.nspecies; sp += gridDim.x)
      if (E.species[sp].is_bunch) ens_inject(E, E.species[sp]);
    for (int r = 0; r < E.nruns; r++) {
      __syncthreads();
      if (threadIdx.x == 0) desc.g = E.runs[r].g;
      __syncthreads();
      const GridDev &g = desc.g;
      const long long nh = (long long)g.nr * (g.nz - 1);
      for (long long l = gtid; l < nh; l += gstride) {
        const int i = (int)(l / (g.nz - 1));
        yee_h_node(g, i, (int)(l - (long long)i * (g.nz - 1)));
      }
      const long long nj = (long long)g.nr * g.nz;
      for (long long l = gtid; l < nj; l += gstride) {
        g.jr[l] = 0.0;
        g.jphi[l] = 0.0;
        g.jz[l] = 0.0;
      }
    }
    grid.sync();
    // ---- phase B: particles.  Global chunk j goes to CTA j mod gridDim.x;
    // the CTA walks the species in order and keeps the current run's grid
    // and species descriptors in shared memory, where they cannot alias the
    // grids and particle arrays that the chunk loop writes.
    for (int sp = 0; sp < E.nspecies; sp++) {
      const int cb = (int)E.species[sp].chunk_begin;
      const int ce = (int)(sp + 1 < E.nspecies ? E.species[sp + 1].chunk_begin : E.total_chunks);
      const int G = (int)gridDim.x;
      int first = cb + (((int)blockIdx.x - cb) % G + G) % G;
      if (first >= ce) continue;
      __syncthreads();
      if (threadIdx.x == 0) {
        desc.g = E.runs[E.species[sp].run].g;
        desc.s = E.species[sp].s;
        desc.pusher = E.runs[E.species[sp].run].pusher;
      }
      __syncthreads();
      for (int c = first; c < ce; c += G)
        f32_chunk<false, PUSHER, false>(desc.g, desc.s, SpeciesOut{}, desc.pusher, c - cb, sm);
    }
    grid.sync();
    // ---- phase C: E update, t += dt
    for (int r = 0; r < E.nruns; r++) {
      __syncthreads();
      if (threadIdx.x == 0) desc.g = E.runs[r].g;
      __syncthreads();
      const GridDev &g = desc.g;
      const long long ne = (long long)(g.nr - 1) * (g.nz - 1);
      for (long long l = gtid; l < ne; l += gstride) {
        const int i = (int)(l / (g.nz - 1));
        yee_e_node(g, i, (int)(l - (long long)i * (g.nz - 1)));
      }
    }
    if (gtid < E.nruns) E.runs[gtid].t = E.runs[gtid].t + E.runs[gtid].g.dt;
    if (gtid == 0) E.status[0] = step + 1;
  }
}

// ---- graph mode: every run's own step kernels on parallel branches of one
// captured graph per ensemble step.  Two small kernels make that graph the
// same for every step: the injection reads each run's time from device
// memory (as the persistent kernel's phase A does), and the time advance
// runs on the device after the runs' branches join.

// Bunch::bunch_inject for every bunch species of every run: CTA j handles
// species j (grid = number of species)
__global__ void k_ens_inject_all(EnsembleDev E) {
  if (blockIdx.x < (unsigned)E.nspecies && E.species[blockIdx.x].is_bunch)
    ens_inject(E, E.species[blockIdx.x]);
}

// t += dt of every run (src/loadInitParam.cpp:586), the same FP64 accumulation
__global__ void k_ens_advance(EnsembleDev E) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < E.nruns) E.runs[r].t = E.runs[r].t + E.runs[r].g.dt;
  if (r == 0) E.status[0] = E.status[0] + 1;
}

cudaError_t ensemble_inject_all(const EnsembleDev &E, cudaStream_t st) {
  if (E.nspecies <= 0) return cudaSuccess;
  k_ens_inject_all<<<E.nspecies, F32_THREADS, 0, st>>>(E);
  return cudaGetLastError();
}

cudaError_t ensemble_advance(const EnsembleDev &E, cudaStream_t st) {
  k_ens_advance<<<(E.nruns + 127) / 128, 128, 0, st>>>(E);
  return cudaGetLastError();
}

static void (*ensemble_kernel(int pusher))(EnsembleDev) {
  switch (pusher) {
    case 0: return k_ensemble<0>;
    case 1: return k_ensemble<1>;
    case 2: return k_ensemble<2>;
    default: return k_ensemble<-1>;
  }
}

int ensemble_max_blocks_per_sm(int pusher) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, ensemble_kernel(pusher), F32_THREADS,
                                                    0) != cudaSuccess)
    return 0;
  return nb;
}

// One cooperative launch of E.status[2] steps (graph capture of this call is
// done by the caller); pusher: the runs' common pusher, or -1.
cudaError_t ensemble_launch(const EnsembleDev &E, int blocks, int pusher, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(F32_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, ensemble_kernel(pusher), E);
}

}  // namespace pdp3g
