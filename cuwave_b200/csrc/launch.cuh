// Host-side launchers of the kernel families. The stencil kernels are instantiated
// one translation unit per (precision, dimension, radius), unit.cu compiled with
// CWB_REAL / CWB_NDIM / CWB_RADIUS, so the build runs in parallel.
#pragma once

#include "params.cuh"

namespace cwb {

// block shapes: BX fast-axis nodes by BY axis-1 nodes (3D), BX nodes (2D)
constexpr int STEP_BX3 = 32, STEP_BY3 = 8, STEP_BX2 = 128;
constexpr int ADJ_BX3 = 32, ADJ_BY3 = 8, ADJ_BX2 = 128;

inline void block_shape(const int ndim, int &bx, int &by) {
  bx = ndim == 3 ? STEP_BX3 : STEP_BX2;
  by = ndim == 3 ? STEP_BY3 : 1;
}

template <typename T, int NDIM, int R>
cudaError_t step_unit(const StepParams<T> &p, bool uniform, dim3 grid, cudaStream_t stream);
template <typename T>
struct StepTmaParams;

// the TMA step: BX x BY tile, each thread RY rows (3D); a BX-wide row (2D)
constexpr int TMA_BX3 = 32, TMA_BY3 = 16, TMA_RY3 = 2, TMA_BX2 = 128;

template <typename T, int NDIM, int R>
cudaError_t step_tma_unit(const StepTmaParams<T> &p, bool uniform, dim3 grid,
                          cudaStream_t stream);
template <typename T, int NDIM, int R>
int step_tma_halo();  // the x halo of the staged box, a multiple of 16 bytes

template <typename T>
struct Step3Params;

// the register-blocked 3D step of a uniform stiffness: 64 x 16 tiles, 256 threads
template <typename T, int R>
cudaError_t step3d_unit(const Step3Params<T> &p, bool uniform, dim3 grid, cudaStream_t stream);
template <typename T, int R>
int step3d_halo();  // the staged box's axis-2 halo, -1 where the kernel is not built

// the 2D quad step of a uniform stiffness (float), 128 threads a block
template <typename T, int R>
cudaError_t step2d_unit(const StepParams<T> &p, bool uniform, dim3 grid, cudaStream_t stream);
template <typename T, int R>
bool step2d_built();
// the pml terms of the 2D quad step when the update kernel leaves them out
struct Pml2Layout;
template <typename T, int R>
cudaError_t pml2d_unit(const StepParams<T> &p, const Pml2Layout &lay, const TransferParams<T> &src,
                       const TransferParams<T> &rec, cudaStream_t stream);

// the 2D quad adjoint of a uniform stiffness (float, radius <= 4), MODE_STEP or
// MODE_STEP_GRAD, 128 threads a block
template <typename T, int R>
cudaError_t adjoint2d_unit(const AdjointParams<T> &p, int mode, dim3 grid, cudaStream_t stream);
struct Adj2Reach;
// its pml transpose, a launch after it over the nodes within R of a slab
template <typename T, int R>
cudaError_t adjoint2d_pml_unit(const AdjointParams<T> &p, const Adj2Reach &reach, int mode,
                               const TransferParams<T> &ld, T *ld_mass, dim3 grid,
                               cudaStream_t stream);

template <typename T>
struct March3Params;
// all steps of an L2-resident 3D grid in one cooperative launch (the generic tile step)
template <typename T, int R>
cudaError_t march3d_unit(const March3Params<T> &p, bool uniform, int sms, cudaStream_t stream);

template <typename T>
struct March2Params;
// the multi-step 2D march, one cooperative launch of as many blocks as fit on `sms` SMs
template <typename T, int R>
cudaError_t march2d_unit(const March2Params<T> &p, int sms, cudaStream_t stream);

template <typename T>
struct TBlock2Params;
// the temporally blocked 2D forward (float, radius <= 4): TB_K steps per pass over HBM,
// a block of TB_TQ threads a tile
template <typename T, int R>
cudaError_t tblock2d_unit(const TBlock2Params<float> &p, dim3 grid, cudaStream_t stream);

template <typename T>
struct Pml3Params;

// the pml memory update of a 3D step along axis 1 or 2, over its slab nodes (after the
// blocked step)
template <typename T, int R>
cudaError_t pml3d_unit(const Pml3Params<T> &p, int axis, dim3 grid, cudaStream_t stream);

template <typename T, int NDIM, int R>
cudaError_t adjoint_unit(const AdjointParams<T> &p, bool uniform, int mode, dim3 grid,
                         cudaStream_t stream);
struct Adj3Reach;
// the 3D adjoint's pml transpose, a launch after the march over the nodes within R of a slab
template <typename T, int R>
cudaError_t adjoint3d_pml_unit(const AdjointParams<T> &p, const Adj3Reach &reach, bool uniform,
                               int mode, dim3 grid, cudaStream_t stream);

template <typename T>
cudaError_t launch_transfer(int kind, const TransferParams<T> &p, T *g_mass, int faces,
                            int threads_total, cudaStream_t stream);

// the 3D ghost refill, with the step's sources and the following record folded in where
// they touch no node the refill reads or writes (null: none)
template <typename T>
cudaError_t launch_refill3d(const TransferParams<T> &p, int faces, const TransferParams<T> *src,
                            const TransferParams<T> *rec, cudaStream_t stream);
template <typename T>
cudaError_t launch_pml_aux(const PmlAuxSet<T> &set, cudaStream_t stream);
template <typename T>
cudaError_t launch_frechet(const FrechetParams<T> &p, cudaStream_t stream);
cudaError_t launch_set_counter(int *ctr, int t0, cudaStream_t stream);

template <typename T>
struct Batch2Params;
template <typename T>
struct BatchRecordParams;
// one step of a batch's items of radius R (2D quad step)
template <typename T, int R>
cudaError_t batch2d_unit(const Batch2Params<T> &p, dim3 grid, cudaStream_t stream);
template <typename T>
cudaError_t launch_batch_record(const BatchRecordParams<T> &p, cudaStream_t stream);

enum : int { TR_EXCITE = 0, TR_LOAD = 1, TR_RECORD = 2, TR_REPLAY = 3, TR_REFILL = 4, TR_DFT = 5 };

}  // namespace cwb
