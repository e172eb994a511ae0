// One (precision, dimension, radius) of the step and adjoint kernels, selected by
// CWB_REAL, CWB_NDIM and CWB_RADIUS at compile time.
#include <algorithm>

#include "adjoint.cuh"
#include "launch.cuh"
#include "step.cuh"
#include "step_tma.cuh"
#include "pml.cuh"
#include "batch.cuh"
#include "adjoint2d.cuh"
#include "step2d.cuh"
#include "step3d.cuh"
#include "step3d_flow.cuh"
#include "tblock2d.cuh"
#include "march3d.cuh"

#if !defined(CWB_REAL) || !defined(CWB_NDIM) || !defined(CWB_RADIUS)
#error "unit.cu is compiled with CWB_REAL, CWB_NDIM and CWB_RADIUS"
#endif

namespace cwb {

namespace {

template <class Kernel>
cudaError_t allow_smem(Kernel k, const size_t bytes) {
  if (bytes <= 48 * 1024)
    return cudaSuccess;
  return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename T, int NDIM, int R, bool U>
cudaError_t step_one(const StepParams<T> &p, const dim3 grid, cudaStream_t s) {
  constexpr int BX = NDIM == 3 ? STEP_BX3 : STEP_BX2;
  constexpr int BY = NDIM == 3 ? STEP_BY3 : 1;
  const size_t smem = 2 * StepShape<NDIM, R, BX, BY>::PLANE * sizeof(T);
  const auto k = step_kernel<T, NDIM, R, U, BX, BY>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess)
    return e;
  k<<<grid, dim3(BX, BY), smem, s>>>(p);
  return cudaGetLastError();
}

template <typename T, int NDIM, int R, bool U, int MODE>
cudaError_t adjoint_one(const AdjointParams<T> &p, const dim3 grid, cudaStream_t s) {
  constexpr int BX = NDIM == 3 ? ADJ_BX3 : ADJ_BX2;
  constexpr int BY = NDIM == 3 ? ADJ_BY3 : 1;
  const size_t smem =
      2 * AdjFields<MODE, U>::COUNT * AdjShape<NDIM, R, BX, BY>::PLANE * sizeof(T);
  const auto k = (p.flags & K_PML) ? adjoint_kernel<T, NDIM, R, U, MODE, BX, BY, true>
                                  : adjoint_kernel<T, NDIM, R, U, MODE, BX, BY, false>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess)
    return e;
  k<<<grid, dim3(BX, BY), smem, s>>>(p);
  return cudaGetLastError();
}

}  // namespace

template <typename T, int NDIM, int R, bool U>
cudaError_t step_tma_one(const StepTmaParams<T> &p, const dim3 grid, cudaStream_t s) {
  constexpr int BX = NDIM == 3 ? TMA_BX3 : TMA_BX2;
  constexpr int BY = NDIM == 3 ? TMA_BY3 : 1;
  constexpr int RY = NDIM == 3 ? TMA_RY3 : 1;
  const size_t smem = TmaShape<T, NDIM, R, BX, BY>::SMEM;
  const auto k = step_tma_kernel<T, NDIM, R, U, BX, BY, RY>;
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess)
    return e;
  k<<<grid, dim3(BX, BY / RY), smem, s>>>(p);
  return cudaGetLastError();
}

template <typename T, int NDIM, int R>
cudaError_t step_tma_unit(const StepTmaParams<T> &p, const bool uniform, const dim3 grid,
                          cudaStream_t stream) {
  return uniform ? step_tma_one<T, NDIM, R, true>(p, grid, stream)
                 : step_tma_one<T, NDIM, R, false>(p, grid, stream);
}

template <typename T, int NDIM, int R>
int step_tma_halo() {
  return TmaShape<T, NDIM, R, 32, 1>::H;
}

#if CWB_NDIM == 3
template <typename T, int R, bool U>
cudaError_t step3d_one(const Step3Params<T> &p, const dim3 grid, cudaStream_t s) {
  if constexpr (!Step3Shape<T, R>::SUPPORTED || !U) {
    return cudaErrorInvalidValue;
  } else {
    // p.flow: 0 the per-plane barrier march, else the barrier-free one (step3d_flow.cuh),
    // built per (Dirichlet face, derived inertia, damping)
    const size_t smem = Step3Shape<T, R>::SMEM;
    const bool hold = p.s.g.dir, derive = p.s.flags & K_DERIVE, damp = p.s.flags & K_DAMP;
    using K = void (*)(const Step3Params<T>);
    K k;
    if (!p.flow)
      k = hold ? step3d_kernel<T, R, U, true> : step3d_kernel<T, R, U, false>;
    else if (hold)
      k = derive ? (damp ? step3d_flow_kernel<T, R, true, true, true> : step3d_flow_kernel<T, R, true, true, false>)
                 : (damp ? step3d_flow_kernel<T, R, true, false, true> : step3d_flow_kernel<T, R, true, false, false>);
    else
      k = derive ? (damp ? step3d_flow_kernel<T, R, false, true, true> : step3d_flow_kernel<T, R, false, true, false>)
                 : (damp ? step3d_flow_kernel<T, R, false, false, true> : step3d_flow_kernel<T, R, false, false, false>);
    cudaError_t e = allow_smem(k, smem);
    if (e != cudaSuccess)
      return e;
    k<<<grid, S3_THREADS, smem, s>>>(p);
    return cudaGetLastError();
  }
}

template <typename T, int R>
cudaError_t step3d_unit(const Step3Params<T> &p, const bool uniform, const dim3 grid,
                        cudaStream_t stream) {
  return uniform ? step3d_one<T, R, true>(p, grid, stream) : step3d_one<T, R, false>(p, grid, stream);
}

template <typename T, int R>
int step3d_halo() {
  return Step3Shape<T, R>::SUPPORTED && Step3Shape<T, R>::SMEM <= 227 * 1024 ? Step3Shape<T, R>::H
                                                                            : -1;
}
#endif

#if CWB_NDIM == 2
template <typename T, int R>
cudaError_t step2d_unit(const StepParams<T> &p, const bool uniform, const dim3 grid,
                        cudaStream_t s) {
  if constexpr (!Step2Shape<T, R>::SUPPORTED) {
    return cudaErrorInvalidValue;
  } else {
    if (!uniform)
      return cudaErrorInvalidValue;
    // the pml inside the update kernel where its flag is on; without it (no pml, or
    // pml2d_kernel applying it after) the instance without the slab code
    const bool pml = p.flags & K_PML;
    if (p.g.dir)
      (pml ? step2d_kernel<T, R, true, true, true> : step2d_kernel<T, R, true, true, false>)
          <<<grid, S2_THREADS, 0, s>>>(p);
    else
      (pml ? step2d_kernel<T, R, true, false, true> : step2d_kernel<T, R, true, false, false>)
          <<<grid, S2_THREADS, 0, s>>>(p);
    return cudaGetLastError();
  }
}

template <typename T, int R>
cudaError_t pml2d_unit(const StepParams<T> &p, const Pml2Layout &lay, const TransferParams<T> &src,
                       const TransferParams<T> &rec, cudaStream_t s) {
  if constexpr (!Step2Shape<T, R>::SUPPORTED) {
    return cudaErrorInvalidValue;
  } else {
    const dim3 grid((unsigned)((lay.total + src.num + rec.num + S2_THREADS - 1) / S2_THREADS));
    if (p.g.dir)
      pml2d_kernel<T, R, true><<<grid, S2_THREADS, 0, s>>>(p, lay, src, rec);
    else
      pml2d_kernel<T, R, false><<<grid, S2_THREADS, 0, s>>>(p, lay, src, rec);
    return cudaGetLastError();
  }
}

template <typename T, int R>
bool step2d_built() {
  return Step2Shape<T, R>::SUPPORTED;
}

template <typename T, int R>
cudaError_t batch2d_unit(const Batch2Params<T> &p, const dim3 grid, cudaStream_t s) {
  if constexpr (!Step2Shape<T, R>::SUPPORTED) {
    return cudaErrorInvalidValue;
  } else {
    if (p.hold)
      (p.pml ? batch2d_kernel<T, R, true, true> : batch2d_kernel<T, R, true, false>)
          <<<grid, S2_THREADS, 0, s>>>(p);
    else
      (p.pml ? batch2d_kernel<T, R, false, true> : batch2d_kernel<T, R, false, false>)
          <<<grid, S2_THREADS, 0, s>>>(p);
    return cudaGetLastError();
  }
}

template <typename T, int R>
cudaError_t march2d_unit(const March2Params<T> &mp, const int sms, cudaStream_t s) {
  if constexpr (!Step2Shape<T, R>::SUPPORTED) {
    return cudaErrorInvalidValue;
  } else {
    const bool pml = mp.s.flags & K_PML;
    const auto k = mp.s.g.dir ? (pml ? march2d_kernel<T, R, true, true> : march2d_kernel<T, R, true, false>)
                              : (pml ? march2d_kernel<T, R, false, true> : march2d_kernel<T, R, false, false>);
    int per = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, S2_THREADS, 0);
    if (e != cudaSuccess)
      return e;
    if (per < 1)
      return cudaErrorInvalidConfiguration;
    const long long want = (mp.units + S2_THREADS - 1) / S2_THREADS;
    const unsigned blocks = (unsigned)std::min<long long>(want, (long long)per * sms);
    void *args[] = {const_cast<March2Params<T> *>(&mp)};
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(k), dim3(blocks),
                                    dim3(S2_THREADS), args, 0, s);
    return e;
  }
}

template <typename T, int R>
cudaError_t tblock2d_unit(const TBlock2Params<float> &p, const dim3 grid, cudaStream_t s) {
  if constexpr (sizeof(T) != 4 || R > 4) {
    return cudaErrorInvalidValue;
  } else {
    const bool pml = p.s.flags & K_PML;
    const auto k = p.s.g.dir ? (pml ? tblock2d_kernel<R, TB_K, true, true> : tblock2d_kernel<R, TB_K, true, false>)
                             : (pml ? tblock2d_kernel<R, TB_K, false, true> : tblock2d_kernel<R, TB_K, false, false>);
    const size_t smem = tblock_smem<R, TB_K>();
    cudaError_t e = allow_smem(k, smem);
    if (e != cudaSuccess)
      return e;
    k<<<grid, TB_TQ * TB_K, smem, s>>>(p);
    return cudaGetLastError();
  }
}

template <typename T, int R>
cudaError_t adjoint2d_unit(const AdjointParams<T> &p, const int mode, const dim3 grid,
                           cudaStream_t s) {
  if constexpr (!Adj2Shape<T, R>::SUPPORTED) {
    return cudaErrorInvalidValue;
  } else {
    const bool hold = p.g.dir != 0, damp = p.flags & K_DAMP;
    using K = void (*)(const AdjointParams<T>);
    K k;
    if (mode == MODE_STEP_GRAD)
      k = hold ? (damp ? adjoint2d_kernel<T, R, MODE_STEP_GRAD, true, true>
                       : adjoint2d_kernel<T, R, MODE_STEP_GRAD, true, false>)
               : (damp ? adjoint2d_kernel<T, R, MODE_STEP_GRAD, false, true>
                       : adjoint2d_kernel<T, R, MODE_STEP_GRAD, false, false>);
    else if (mode == MODE_STEP)
      k = hold ? (damp ? adjoint2d_kernel<T, R, MODE_STEP, true, true>
                       : adjoint2d_kernel<T, R, MODE_STEP, true, false>)
               : (damp ? adjoint2d_kernel<T, R, MODE_STEP, false, true>
                       : adjoint2d_kernel<T, R, MODE_STEP, false, false>);
    else
      return cudaErrorInvalidValue;
    k<<<grid, A2_THREADS, 0, s>>>(p);
    return cudaGetLastError();
  }
}

template <typename T, int R>
cudaError_t adjoint2d_pml_unit(const AdjointParams<T> &p, const Adj2Reach &reach, const int mode,
                               const TransferParams<T> &ld, T *ld_mass, const dim3 grid,
                               cudaStream_t s) {
  if constexpr (!Adj2Shape<T, R>::SUPPORTED) {
    return cudaErrorInvalidValue;
  } else {
    if (mode == MODE_STEP_GRAD)
      adjoint2d_pml_kernel<T, R, MODE_STEP_GRAD><<<grid, A2P_THREADS, 0, s>>>(p, reach, ld, ld_mass);
    else if (mode == MODE_STEP)
      adjoint2d_pml_kernel<T, R, MODE_STEP><<<grid, A2P_THREADS, 0, s>>>(p, reach, ld, ld_mass);
    else
      return cudaErrorInvalidValue;
    return cudaGetLastError();
  }
}
#endif

#if CWB_NDIM == 3
template <typename T, int R>
cudaError_t pml3d_unit(const Pml3Params<T> &p, const int axis, const dim3 grid, cudaStream_t s) {
  if (axis == 1)
    pml_axis1_kernel<T, R><<<grid, PML1_THREADS, 0, s>>>(p);
  else if (axis == 2)
    pml_axis2_kernel<T, R><<<grid, PML2_THREADS, 0, s>>>(p);
  else
    return cudaErrorInvalidValue;
  return cudaGetLastError();
}
#endif

template <typename T, int NDIM, int R>
cudaError_t step_unit(const StepParams<T> &p, const bool uniform, const dim3 grid,
                      cudaStream_t stream) {
  return uniform ? step_one<T, NDIM, R, true>(p, grid, stream)
                 : step_one<T, NDIM, R, false>(p, grid, stream);
}

template <typename T, int NDIM, int R>
cudaError_t adjoint_unit(const AdjointParams<T> &p, const bool u, const int mode,
                         const dim3 grid, cudaStream_t s) {
  if (mode == MODE_STEP)
    return u ? adjoint_one<T, NDIM, R, true, MODE_STEP>(p, grid, s)
             : adjoint_one<T, NDIM, R, false, MODE_STEP>(p, grid, s);
  if (mode == MODE_STEP_GRAD)
    return u ? adjoint_one<T, NDIM, R, true, MODE_STEP_GRAD>(p, grid, s)
             : adjoint_one<T, NDIM, R, false, MODE_STEP_GRAD>(p, grid, s);
  return u ? adjoint_one<T, NDIM, R, true, MODE_GRAD>(p, grid, s)
           : adjoint_one<T, NDIM, R, false, MODE_GRAD>(p, grid, s);
}

#if CWB_NDIM == 3
template <typename T, int R>
cudaError_t march3d_unit(const March3Params<T> &mp, const bool uniform, const int sms,
                         cudaStream_t s) {
  constexpr int BX = STEP_BX3, BY = STEP_BY3;
  const auto k = uniform ? march3d_kernel<T, R, true, BX, BY> : march3d_kernel<T, R, false, BX, BY>;
  const size_t smem = 2 * StepShape<3, R, BX, BY>::PLANE * sizeof(T);
  cudaError_t e = allow_smem(k, smem);
  if (e != cudaSuccess)
    return e;
  int per = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, BX * BY, smem);
  if (e != cudaSuccess)
    return e;
  if (per < 1)
    return cudaErrorInvalidConfiguration;
  const long long ntiles = (long long)mp.nbx * mp.nby * mp.nbz;
  const unsigned blocks = (unsigned)std::min<long long>(ntiles, (long long)per * sms);
  void *args[] = {const_cast<March3Params<T> *>(&mp)};
  return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(k), dim3(blocks), dim3(BX, BY),
                                     args, smem, s);
}
template cudaError_t march3d_unit<CWB_REAL, CWB_RADIUS>(const March3Params<CWB_REAL> &, bool, int,
                                                        cudaStream_t);

template <typename T, int R>
cudaError_t adjoint3d_pml_unit(const AdjointParams<T> &p, const Adj3Reach &reach, const bool u,
                               const int mode, const dim3 grid, cudaStream_t s) {
  if (mode == MODE_STEP_GRAD)
    u ? adjoint3d_pml_kernel<T, R, true, MODE_STEP_GRAD><<<grid, A3P_THREADS, 0, s>>>(p, reach)
      : adjoint3d_pml_kernel<T, R, false, MODE_STEP_GRAD><<<grid, A3P_THREADS, 0, s>>>(p, reach);
  else
    u ? adjoint3d_pml_kernel<T, R, true, MODE_STEP><<<grid, A3P_THREADS, 0, s>>>(p, reach)
      : adjoint3d_pml_kernel<T, R, false, MODE_STEP><<<grid, A3P_THREADS, 0, s>>>(p, reach);
  return cudaGetLastError();
}
template cudaError_t adjoint3d_pml_unit<CWB_REAL, CWB_RADIUS>(const AdjointParams<CWB_REAL> &,
                                                               const Adj3Reach &, bool, int, dim3,
                                                               cudaStream_t);
#endif

template cudaError_t step_unit<CWB_REAL, CWB_NDIM, CWB_RADIUS>(const StepParams<CWB_REAL> &,
                                                               bool, dim3, cudaStream_t);
template cudaError_t step_tma_unit<CWB_REAL, CWB_NDIM, CWB_RADIUS>(
    const StepTmaParams<CWB_REAL> &, bool, dim3, cudaStream_t);
template int step_tma_halo<CWB_REAL, CWB_NDIM, CWB_RADIUS>();
#if CWB_NDIM == 2
template cudaError_t step2d_unit<CWB_REAL, CWB_RADIUS>(const StepParams<CWB_REAL> &, bool, dim3,
                                                       cudaStream_t);
template bool step2d_built<CWB_REAL, CWB_RADIUS>();
template cudaError_t pml2d_unit<CWB_REAL, CWB_RADIUS>(const StepParams<CWB_REAL> &, const Pml2Layout &,
                                                      const TransferParams<CWB_REAL> &,
                                                      const TransferParams<CWB_REAL> &, cudaStream_t);
template cudaError_t batch2d_unit<CWB_REAL, CWB_RADIUS>(const Batch2Params<CWB_REAL> &, dim3,
                                                        cudaStream_t);
template cudaError_t march2d_unit<CWB_REAL, CWB_RADIUS>(const March2Params<CWB_REAL> &, int,
                                                         cudaStream_t);
template cudaError_t tblock2d_unit<CWB_REAL, CWB_RADIUS>(const TBlock2Params<float> &, dim3,
                                                          cudaStream_t);
template cudaError_t adjoint2d_unit<CWB_REAL, CWB_RADIUS>(const AdjointParams<CWB_REAL> &, int,
                                                          dim3, cudaStream_t);
template cudaError_t adjoint2d_pml_unit<CWB_REAL, CWB_RADIUS>(const AdjointParams<CWB_REAL> &,
                                                              const Adj2Reach &, int,
                                                              const TransferParams<CWB_REAL> &,
                                                              CWB_REAL *, dim3, cudaStream_t);
#endif
#if CWB_NDIM == 3
template cudaError_t step3d_unit<CWB_REAL, CWB_RADIUS>(const Step3Params<CWB_REAL> &, bool, dim3,
                                                       cudaStream_t);
template int step3d_halo<CWB_REAL, CWB_RADIUS>();
template cudaError_t pml3d_unit<CWB_REAL, CWB_RADIUS>(const Pml3Params<CWB_REAL> &, int, dim3,
                                                      cudaStream_t);
#endif
template cudaError_t adjoint_unit<CWB_REAL, CWB_NDIM, CWB_RADIUS>(
    const AdjointParams<CWB_REAL> &, bool, int, dim3, cudaStream_t);

}  // namespace cwb
