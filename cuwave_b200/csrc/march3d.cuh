// The multi-step march of an L2-resident 3D grid: one cooperative launch runs `steps`
// steps of [step (sources and refill folded), records], a grid-wide barrier between a
// step and its records, where the per-step march launches a step and its transfers
// every step. It stands in for cuwave's 3D blocked_kernel (several steps per launch,
// excitation, refill and record folded in; cuwave/kernels/scalar.cu:1094-1370) on a grid
// whose fields stay in L2 between steps, as march2d_kernel does in 2D.
//
// Each step is the generic tile step of step.cuh (step_block: a BX x BY tile of the
// plane, a chunk of planes along axis 0, the axis-0 taps in a register queue, the plane
// staged in shared memory), so the node arithmetic, the pml terms, the folded sources and
// the folded refill are that kernel's (cuwave fd_kernel and pml_kernel, scalar.cu:347-532,
// excitation_kernel, common.cuh:456-464, the refill, scalar.cu:535-555) to the bit. The
// blocks, all resident, take the tiles in turn; the next step writes the level two back
// and reads this one, so a step needs no barrier before the next one's tiles.
#pragma once

#include <cooperative_groups.h>

#include "step.cuh"
#include "transfer.cuh"

namespace cwb {

constexpr int MARCH3_RECORDS = 4;

template <typename T>
struct March3Params {
  StepParams<T> s;                        // the step (its sources' lists by tile)
  TransferParams<T> rec[MARCH3_RECORDS];  // store, level and rows of each record
  int nrec;
  int t0, steps;
  int nbx, nby, nbz;  // the tile grid
};

template <typename T, int R, bool UNIF, int BX, int BY>
__global__ void __launch_bounds__(BX *BY) march3d_kernel(const __grid_constant__ March3Params<T> mp) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *tiles = reinterpret_cast<T *>(smem_raw);
  const int ntiles = mp.nbx * mp.nby * mp.nbz;
  const long long gtid = (long long)blockIdx.x * (BX * BY) + threadIdx.y * BX + threadIdx.x;
  const long long gsize = (long long)gridDim.x * (BX * BY);
  for (int s = 0; s < mp.steps; ++s) {
    const int t = mp.t0 + s;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      step_block<T, 3, R, UNIF, BX, BY>(mp.s, t, tile % mp.nbx, (tile / mp.nbx) % mp.nby,
                                        tile / (mp.nbx * mp.nby), mp.nbx, mp.nby, tiles);
      __syncthreads();  // the next tile stages its planes into the same shared memory
    }
    grid.sync();  // the step's nodes and ghosts are all written
    for (int r = 0; r < mp.nrec; ++r) {
      const TransferParams<T> &rp = mp.rec[r];
      const T *a = level<T>(rp.a, t);
      const long long row = (long long)rp.row_mul * t + rp.row_add;
      for (long long j = gtid; j < rp.num; j += gsize)
        record_write(rp, row * rp.num + j, a[rp.lin[j]]);
    }
  }
  if (gtid == 0) {
    mp.s.ctr[1] = 0;
    mp.s.ctr[0] = mp.t0 + mp.steps;
  }
}

}  // namespace cwb
