// The transfer, refill and adjoint pml memory kernels of both precisions.
#include "launch.cuh"
#include "transfer.cuh"
#include "batch.cuh"

namespace cwb {

template <typename T>
cudaError_t launch_transfer(const int kind, const TransferParams<T> &p, T *g_mass,
                            const int faces, const int threads_total, cudaStream_t stream) {
  const int blocks = (threads_total + TRANSFER_THREADS - 1) / TRANSFER_THREADS;
  if (blocks <= 0)
    return cudaErrorInvalidValue;
  switch (kind) {
  case TR_EXCITE: excite_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p); break;
  case TR_LOAD: load_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p, g_mass); break;
  case TR_RECORD: record_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p); break;
  case TR_REPLAY: replay_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p); break;
  case TR_REFILL: refill_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p, faces); break;
  case TR_DFT: dft_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p, g_mass); break;
  default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_pml_aux(const PmlAuxParams<T> &p, cudaStream_t stream) {
  const int blocks = (p.memrow + TRANSFER_THREADS - 1) / TRANSFER_THREADS;
  if (blocks <= 0)
    return cudaErrorInvalidValue;
  pml_aux_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_frechet(const FrechetParams<T> &p, cudaStream_t stream) {
  const long long total = (long long)p.g.n[0] * p.g.s[0];
  const long long blocks = (total + TRANSFER_THREADS - 1) / TRANSFER_THREADS;
  if (blocks <= 0 || blocks > 0x7fffffffLL)
    return cudaErrorInvalidValue;
  frechet_kernel<T><<<(unsigned)blocks, TRANSFER_THREADS, 0, stream>>>(p);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_batch_record(const BatchRecordParams<T> &p, cudaStream_t stream) {
  const int blocks = (p.total + TRANSFER_THREADS - 1) / TRANSFER_THREADS;
  if (blocks <= 0)
    return cudaErrorInvalidValue;
  batch_record_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p);
  return cudaGetLastError();
}

__global__ void set_counter_kernel(int *ctr, const int t0) {
  ctr[0] = t0;
  ctr[1] = 0;
}

cudaError_t launch_set_counter(int *ctr, const int t0, cudaStream_t stream) {
  set_counter_kernel<<<1, 1, 0, stream>>>(ctr, t0);
  return cudaGetLastError();
}

template cudaError_t launch_transfer<float>(int, const TransferParams<float> &, float *, int,
                                            int, cudaStream_t);
template cudaError_t launch_transfer<double>(int, const TransferParams<double> &, double *,
                                             int, int, cudaStream_t);
template cudaError_t launch_frechet<float>(const FrechetParams<float> &, cudaStream_t);
template cudaError_t launch_frechet<double>(const FrechetParams<double> &, cudaStream_t);
template cudaError_t launch_batch_record<float>(const BatchRecordParams<float> &, cudaStream_t);
template cudaError_t launch_batch_record<double>(const BatchRecordParams<double> &, cudaStream_t);
template cudaError_t launch_pml_aux<float>(const PmlAuxParams<float> &, cudaStream_t);
template cudaError_t launch_pml_aux<double>(const PmlAuxParams<double> &, cudaStream_t);

}  // namespace cwb
