// TMA tile loads and mbarriers for sm_100a, as inline PTX.
//
// Every wait on an mbarrier is bounded: after WAIT_CYCLES clock cycles (about a second)
// it gives up, the kernel raises its error flag, drains what it issued and finishes, so
// a lost copy can never hang the GPU. The host reads the flag after the march.
#pragma once

#include <cstdint>
#include <cuda.h>

namespace cwb {

constexpr long long WAIT_CYCLES = 2000000000LL;  // ~1 s at 1.9 GHz

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// `base` advanced to the next 128-byte boundary by pointer arithmetic on the shared array
// itself, so the compiler keeps every access through it in the shared window (a round
// trip through an integer would leave it a generic pointer, with 64-bit address math)
__device__ __forceinline__ unsigned char *align_smem128(unsigned char *base) {
  return base + ((128u - (smem_addr(base) & 127u)) & 127u);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, const unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// arrive once and announce `bytes` of transaction the copies will complete
__device__ __forceinline__ void mbar_expect(uint64_t *bar, const unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// wait for phase `parity` of the barrier to complete; false if the bound ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, const unsigned parity) {
  const unsigned addr = smem_addr(bar);
  const long long start = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done)
      return true;
    if (clock64() - start > WAIT_CYCLES)
      return false;
  }
}

// one test of phase `parity`, without the waiting loop: true if it has completed
__device__ __forceinline__ bool mbar_try(uint64_t *bar, const unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return done;
}

// a 4D tile (x fastest) of `map` at coordinates (x, y, z, w) into shared memory, its
// bytes completing on `bar`; x * element size must be a multiple of 16 bytes
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            const int x, const int y, const int z,
                                            const int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            const int x, const int y, const int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

__device__ __forceinline__ void prefetch_map(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace cwb
