// Device helpers shared by the step, adjoint and transfer kernels.
//
// Arithmetic is written in the reference's own expression order and the library is
// built with --fmad=false, so nothing is contracted that the reference's host build
// (g++ -ffp-contract=off, cuwave/cpu.py) does not contract either; the explicit fused
// operations of cuwave/kernels/common.cuh:11-19 (MUL_RN, FMA_RN) are kept as such.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cwb {

// op flags as the kernels read them
enum : int {
  K_PML = 1,      // step / adjoint: the lined axes carry memory terms
  K_DAMP = 2,     // a damping field divides the update
  K_DERIVE = 4,   // 1 / m = 1 / k
  K_SRC = 8,      // step: sources folded in
  K_REFILL = 16,  // step: face ghosts written from their mirrors
  K_ADV = 32,     // this launch ends the step: the last block advances the counter
  K_GRAD = 64,    // adjoint: accumulate g_mass, g_stiff
  K_MASS = 128,   // load: the adjoint load's inertia share
  K_SUPER = 256,  // step: add the superposition densities of the triplet (acc_mass, acc_stiff)
  K_CELLS = 512,  // step: a masked domain, per-node cell radii in `cells`
};

// cell codes of a masked domain
constexpr int CELL_DEEP = 1 << 30;  // every cell of the node at the full radius
constexpr int CELL_HELD = 7;        // a cell open onto a node held at zero

struct DLevel {
  char *base;
  long long stride;  // bytes between levels
  int mul, add, period;
};

// level index mul * t + add (mod period): 32-bit integer arithmetic, a 64-bit modulo
// being a long emulated sequence on the GPU (step counts and level counts are far below
// 2^31)
template <typename T>
__device__ __forceinline__ T *level(const DLevel &L, const int t) {
  int k = L.mul * t + L.add;
  if (L.period > 0) {
    k %= L.period;
    if (k < 0)
      k += L.period;
  }
  return reinterpret_cast<T *>(L.base + (long long)k * L.stride);
}

__device__ __forceinline__ int step_index(const int *ctr) {
  return *reinterpret_cast<const volatile int *>(ctr);
}

// The launch that ends a time step advances the step counter once every block is
// done: each block reads the counter when it starts, so the last to finish is past
// every read. All threads of the block must reach this call.
__device__ __forceinline__ void finish_step(int *ctr, const bool advance) {
  if (!advance)
    return;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    __threadfence();
    const unsigned total = gridDim.x * gridDim.y * gridDim.z;
    const unsigned prev = atomicAdd(reinterpret_cast<unsigned *>(ctr + 1), 1u);
    if (prev == total - 1) {
      ctr[1] = 0;
      ctr[0] = ctr[0] + 1;
      __threadfence();
    }
  }
}

// a += v as one IEEE addition, atomically: a compare-and-swap loop, since the hardware's
// float atomic add flushes subnormal results to zero and the reference's host adds do not
__device__ __forceinline__ void atomic_add_exact(float *a, const float v) {
  unsigned *w = reinterpret_cast<unsigned *>(a);
  unsigned old = *reinterpret_cast<volatile unsigned *>(w), seen;
  do {
    seen = old;
    old = atomicCAS(w, seen, __float_as_uint(__uint_as_float(seen) + v));
  } while (old != seen);
}
__device__ __forceinline__ void atomic_add_exact(double *a, const double v) {
  unsigned long long *w = reinterpret_cast<unsigned long long *>(a);
  unsigned long long old = *reinterpret_cast<volatile unsigned long long *>(w), seen;
  do {
    seen = old;
    old = atomicCAS(w, seen,
                    (unsigned long long)__double_as_longlong(__longlong_as_double((long long)seen) + v));
  } while (old != seen);
}

// products and fused products the compiler keeps as written
__device__ __forceinline__ float mul_rn(const float a, const float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(const double a, const double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float fma_rn(const float a, const float b, const float c) {
  return __fmaf_rn(a, b, c);
}
__device__ __forceinline__ double fma_rn(const double a, const double b, const double c) {
  return __fma_rn(a, b, c);
}

// node b of an axis of N nodes as the forward step reads it: past the stored ghost
// its mirror about the wall node, negated past a face of `odd` (cuwave common.cuh:50-54)
__device__ __forceinline__ int mirror_node(const int b, const int N, const int odd, int &sign) {
  sign = ((b < 0 && (odd & 1)) || (b > N - 1 && (odd & 2))) ? -1 : 1;
  return b < 0 ? 2 - b : (b > N - 1 ? 2 * (N - 2) - b : b);
}

// node b past the wall node its image, as the adjoint reads a field no refill keeps:
// the ghost itself is mirrored too (cuwave common.cuh:73-77)
__device__ __forceinline__ int node_image(const int b, const int N, const int odd, int &sign) {
  sign = ((b < 1 && (odd & 1)) || (b > N - 2 && (odd & 2))) ? -1 : 1;
  return b < 1 ? 2 - b : (b > N - 2 ? 2 * (N - 2) - b : b);
}

// whether node a is the wall node of a Dirichlet face of `odd` (cuwave common.cuh:43-46)
__device__ __forceinline__ bool held_wall(const int a, const int N, const int odd) {
  return ((odd & 1) && a == 1) || ((odd & 2) && a == N - 2);
}

// A run of nodes along the fast axis past its walls takes the mirrored values (cuwave common.cuh:50-54).
// Low wall: node -1 - m sits at run index H - 1 - m, its mirror 3 + m at H + 3 + m. High
// wall: with E the run index of node NF, node NF + m sits at E + m and its mirror
// NF - 4 - m at E - 4 - m. E is a compile-time case of the run's place.
template <typename T, int XR, int H>
__device__ __forceinline__ void mirror_run_lo(T *xr, const T s) {
#pragma unroll
  for (int m = 0; m < H; ++m)
    xr[H - 1 - m] = s * xr[H + 3 + m];
}

// mirror_run_lo for a run whose first `lead` values lie past the low wall: a run of halo
// H that starts at node -lead (lead = H - x0 of its quad, a multiple of four up to H)
template <typename T, int XR, int H>
__device__ __forceinline__ void mirror_run_lo_at(T *xr, const T s, const int lead) {
  if (lead == H)
    mirror_run_lo<T, XR, H>(xr, s);
  else if constexpr (H > 4)
    mirror_run_lo_at<T, XR, H - 4>(xr, s, lead);
}

template <typename T, int XR, int E>
__device__ __forceinline__ void mirror_run_hi(T *xr, const T s) {
#pragma unroll
  for (int m = 0; E + m < XR; ++m)
    xr[E + m] = E - 4 - m >= 0 ? s * xr[E - 4 - m] : (T)0;
}

// mirror_run_hi for the run's place e = E0, E0 + 1, .. < XR, chosen at run time
template <typename T, int XR, int E>
__device__ __forceinline__ void mirror_run_hi_at(T *xr, const T s, const int e) {
  if (e == E)
    mirror_run_hi<T, XR, E>(xr, s);
  else if constexpr (E + 1 < XR)
    mirror_run_hi_at<T, XR, E + 1>(xr, s, e);
}

// four consecutive values from 16-byte aligned memory, and back
template <typename T>
__device__ __forceinline__ void load4(T *dst, const T *src) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4 *>(src);
    dst[0] = v.x, dst[1] = v.y, dst[2] = v.z, dst[3] = v.w;
  } else {
    const double2 a = reinterpret_cast<const double2 *>(src)[0];
    const double2 b = reinterpret_cast<const double2 *>(src)[1];
    dst[0] = a.x, dst[1] = a.y, dst[2] = b.x, dst[3] = b.y;
  }
}
template <typename T>
__device__ __forceinline__ void store4(T *dst, const T *v) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4 *>(dst) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    reinterpret_cast<double2 *>(dst)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(dst)[1] = make_double2(v[2], v[3]);
  }
}

template <typename T>
__device__ __forceinline__ T signed_value(const T v, const int sign) {
  return sign > 0 ? v : (sign < 0 ? -v : (T)0);
}

// d(D+)/d(u at row q off the node) and d(D-)/d(u ...) at the full radius, the weights
// the pml transpose scatters with (cuwave scalar_sensitivity.cu:221-234)
template <typename T, int R>
__device__ __forceinline__ T plus_tap(const T *w, const int q) {
  if (q >= 1)
    return q <= R ? w[q - 1] : (T)0;
  return 1 - q <= R ? -w[-q] : (T)0;
}
template <typename T, int R>
__device__ __forceinline__ T minus_tap(const T *w, const int q) {
  if (q >= 0)
    return q + 1 <= R ? w[q] : (T)0;
  return -q <= R ? -w[-q - 1] : (T)0;
}

// ------------------------------------------------------------------ pml slabs
// A lined axis d keeps its memory over the slab of its layer rows: row r < lo is node
// 1 + r, row lo + k is node N - 1 - hi + k. The memory is laid out as the padded grid
// with axis d replaced by those lo + hi rows, so a slab row along the march stays
// contiguous in the fast axis.
__device__ __forceinline__ int slab_row(const int a, const int N, const int lo, const int hi) {
  if (lo && a >= 1 && a <= lo)
    return a - 1;
  if (hi && a >= N - 1 - hi && a <= N - 2)
    return lo + a - (N - 1 - hi);
  return -1;
}

struct Geometry {
  int ndim;
  int n[3];      // logical extents
  int ext[3];    // padded extents (only the last differs)
  int s[3];      // strides in elements
  int lo[3], hi[3];
  int dir;       // Dirichlet faces
};

// flat slab index of node A (its axis-d coordinate replaced by slab row r)
__device__ __forceinline__ int slab_index(const Geometry &g, const int d, const int r,
                                          const int *A) {
  int idx = 0;
  for (int e = 0; e < g.ndim; ++e) {
    const int extent = e == d ? g.lo[d] + g.hi[d] : g.ext[e];
    idx = idx * extent + (e == d ? r : A[e]);
  }
  return idx;
}

// the cell weight W of an interior node: 1/2 per axis on whose wall it sits
template <typename T>
__device__ __forceinline__ T cell_weight(const Geometry &g, const int *A) {
  T w = (T)1;
  for (int e = 0; e < g.ndim; ++e)
    if (A[e] == 1 || A[e] == g.n[e] - 2)
      w *= (T)0.5;
  return w;
}

}  // namespace cwb
