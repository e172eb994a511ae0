// The transfer, refill and adjoint pml memory kernels of both precisions.
#include <cstring>

#include "launch.cuh"
#include "transfer.cuh"
#include "batch.cuh"

namespace cwb {

template <typename T>
cudaError_t launch_refill3d(const TransferParams<T> &p, int faces, const TransferParams<T> *src,
                            const TransferParams<T> *rec, cudaStream_t stream);

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
  case TR_REFILL:
    if (p.g.ndim == 3)
      return launch_refill3d<T>(p, faces, nullptr, nullptr, stream);
    refill_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p, faces);
    break;
  case TR_DFT: dft_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(p, g_mass); break;
  default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_refill3d(const TransferParams<T> &p, const int faces, const TransferParams<T> *src,
                            const TransferParams<T> *rec, cudaStream_t stream) {
  const Geometry &g = p.g;
  Refill3Layout lay;
  lay.faces = faces;
  lay.nq = (g.n[2] - 2) / 4 + 1;
  lay.n0 = (faces & 3) ? 2LL * (g.n[1] - 2) * lay.nq : 0;
  lay.n1 = (faces & 12) ? 2LL * (g.n[0] - 2) * lay.nq : 0;
  const long long n2 = (faces & 48) ? (long long)(g.n[0] - 2) * (g.n[1] - 2) : 0;
  lay.total = lay.n0 + lay.n1 + n2;
  TransferParams<T> none;
  std::memset(&none, 0, sizeof none);
  const TransferParams<T> &sp = src ? *src : none, &rp = rec ? *rec : none;
  const long long threads = lay.total + sp.num + rp.num;
  if (threads <= 0)
    return cudaSuccess;
  const long long blocks = (threads + TRANSFER_THREADS - 1) / TRANSFER_THREADS;
  refill3d_kernel<T><<<(unsigned)blocks, TRANSFER_THREADS, 0, stream>>>(p, lay, sp, rp);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_pml_aux(const PmlAuxSet<T> &set, cudaStream_t stream) {
  const int blocks = set.first[set.nax];
  if (set.nax <= 0 || blocks <= 0)
    return cudaErrorInvalidValue;
  pml_aux_kernel<T><<<blocks, TRANSFER_THREADS, 0, stream>>>(set);
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
template cudaError_t launch_refill3d<float>(const TransferParams<float> &, int,
                                            const TransferParams<float> *,
                                            const TransferParams<float> *, cudaStream_t);
template cudaError_t launch_refill3d<double>(const TransferParams<double> &, int,
                                             const TransferParams<double> *,
                                             const TransferParams<double> *, cudaStream_t);
template cudaError_t launch_frechet<float>(const FrechetParams<float> &, cudaStream_t);
template cudaError_t launch_frechet<double>(const FrechetParams<double> &, cudaStream_t);
template cudaError_t launch_batch_record<float>(const BatchRecordParams<float> &, cudaStream_t);
template cudaError_t launch_batch_record<double>(const BatchRecordParams<double> &, cudaStream_t);
template cudaError_t launch_pml_aux<float>(const PmlAuxSet<float> &, cudaStream_t);
template cudaError_t launch_pml_aux<double>(const PmlAuxSet<double> &, cudaStream_t);

}  // namespace cwb
