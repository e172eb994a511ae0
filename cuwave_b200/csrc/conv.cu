// 5x5 convolutions of the learned dispersion corrector on the tensor cores.
//
// The corrector is a small network of 5x5 convolutions (stride 1, zero padding 2) over
// channels-last BF16 activations (B, H, W, C). Each convolution is an implicit GEMM run
// with the warp-level BF16 MMA (m16n8k16, FP32 accumulation):
//
//   forward         y[m][n]  = sum_k A[m][k] w[n][k] (+ bias, ReLU)   M pixels, N out channels
//   data gradient   the forward over dy with the weights flipped and transposed (the
//                   host lays them out), gated by the layer input's ReLU mask
//   weight gradient dw[n][k] = sum_m dy[m][n] A[m][k]                 split over pixel chunks
//
// with A the im2col of the input: A[m][k] = x[pixel m shifted by tap k / C][channel
// k % C], zero past the image, k running over the 25 taps x C channels (tap-major) and
// zero-padded to a multiple of 16. C is even, so a pair of consecutive k is one 32-bit
// load of two channels. The weights of a layer ((N, K) BF16, at most 32 x 800) sit in
// shared memory for the forward launches. Every access is bounds-checked against the
// sizes passed in.
#include <cuda_bf16.h>

#include <cstdint>

#include "conv.cuh"

namespace cwb {

constexpr int CONV_WARPS = 4;
constexpr int CONV_THREADS = CONV_WARPS * 32;

__device__ __forceinline__ void mma_bf16(float *c, const unsigned *a, const unsigned *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// two channels (k, k + 1) of im2col row m: one 32-bit load, zero off the image
__device__ __forceinline__ unsigned im2col_pair(const __nv_bfloat16 *x, const ConvShape &s,
                                                const long long m, const int k) {
  if (m >= s.pixels() || k >= 25 * s.cin)
    return 0u;
  const int tap = k / s.cin, ci = k - tap * s.cin;
  const int ky = tap / 5, kx = tap - ky * 5;
  const long long plane = (long long)s.h * s.w;
  const int b = (int)(m / plane);
  const int rest = (int)(m - (long long)b * plane);
  const int y = rest / s.w + ky - 2, xx = rest % s.w + kx - 2;
  if (y < 0 || y >= s.h || xx < 0 || xx >= s.w)
    return 0u;
  const long long at = (((long long)b * s.h + y) * s.w + xx) * s.cin + ci;
  return *reinterpret_cast<const unsigned *>(x + at);
}

// forward (and data gradient): a warp computes 16 pixels x all output channels
__global__ void __launch_bounds__(CONV_THREADS) conv_fwd_kernel(
    const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
    const float *__restrict__ bias, const __nv_bfloat16 *__restrict__ mask,
    __nv_bfloat16 *__restrict__ y16, float *__restrict__ y32, const ConvShape s,
    const int relu) {
  extern __shared__ __align__(16) unsigned char conv_smem[];
  __nv_bfloat16 *ws = reinterpret_cast<__nv_bfloat16 *>(conv_smem);
  const int ntiles = (s.cout + 7) / 8;
  const int wn = ntiles * 8;
  // the weights, (wn, kpad), rows past cout zero
  for (int i = threadIdx.x; i < wn * s.kpad; i += CONV_THREADS) {
    const int n = i / s.kpad;
    ws[i] = n < s.cout ? w[(long long)n * s.kpad + (i - n * s.kpad)] : __float2bfloat16(0.f);
  }
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = lane / 4, q = lane % 4;
  const long long m0 = ((long long)blockIdx.x * CONV_WARPS + warp) * 16;
  float acc[CONV_MAX_N / 8][4];
#pragma unroll
  for (int t = 0; t < CONV_MAX_N / 8; ++t)
    acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.f;
  for (int k0 = 0; k0 < s.kpad; k0 += 16) {
    unsigned a[4];
    a[0] = im2col_pair(x, s, m0 + g, k0 + 2 * q);
    a[1] = im2col_pair(x, s, m0 + g + 8, k0 + 2 * q);
    a[2] = im2col_pair(x, s, m0 + g, k0 + 2 * q + 8);
    a[3] = im2col_pair(x, s, m0 + g + 8, k0 + 2 * q + 8);
#pragma unroll
    for (int t = 0; t < CONV_MAX_N / 8; ++t) {
      if (t < ntiles) {
        const __nv_bfloat16 *row = ws + (t * 8 + g) * s.kpad + k0 + 2 * q;
        unsigned b[2];
        b[0] = *reinterpret_cast<const unsigned *>(row);
        b[1] = *reinterpret_cast<const unsigned *>(row + 8);
        mma_bf16(acc[t], a, b);
      }
    }
  }
#pragma unroll
  for (int t = 0; t < CONV_MAX_N / 8; ++t) {
    if (t >= ntiles)
      continue;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const long long m = m0 + g + (e >= 2 ? 8 : 0);
      const int n = t * 8 + 2 * q + (e & 1);
      if (m >= s.pixels() || n >= s.cout)
        continue;
      float v = acc[t][e];
      if (bias)
        v += bias[n];
      if (relu && v < 0.f)
        v = 0.f;
      const long long at = m * s.cout + n;
      if (mask && !(__bfloat162float(mask[at]) > 0.f))
        v = 0.f;
      if (y16)
        y16[at] = __float2bfloat16(v);
      if (y32)
        y32[at] = v;
    }
  }
}

// weight gradient: a warp owns 4 column tiles (32 k) of dw for every row tile of cout,
// summed over the block's pixel chunk, then added into dw
constexpr int WGRAD_CHUNK = 1024;

__device__ __forceinline__ unsigned pack_bf16(const __nv_bfloat16 lo, const __nv_bfloat16 hi) {
  return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ __nv_bfloat16 im2col_one(const __nv_bfloat16 *x, const ConvShape &s,
                                                    const long long m, const int k) {
  if (m >= s.pixels() || k >= 25 * s.cin)
    return __float2bfloat16(0.f);
  const int tap = k / s.cin, ci = k - tap * s.cin;
  const int ky = tap / 5, kx = tap - ky * 5;
  const long long plane = (long long)s.h * s.w;
  const int b = (int)(m / plane);
  const int rest = (int)(m - (long long)b * plane);
  const int y = rest / s.w + ky - 2, xx = rest % s.w + kx - 2;
  if (y < 0 || y >= s.h || xx < 0 || xx >= s.w)
    return __float2bfloat16(0.f);
  return x[(((long long)b * s.h + y) * s.w + xx) * s.cin + ci];
}

__global__ void __launch_bounds__(CONV_THREADS) conv_wgrad_kernel(
    const __nv_bfloat16 *__restrict__ dy, const __nv_bfloat16 *__restrict__ x,
    float *__restrict__ dw, const ConvShape s) {
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int g = lane / 4, q = lane % 4;
  const int kbase = (blockIdx.y * CONV_WARPS + warp) * 32;  // the warp's 32 columns of dw
  const long long p_begin = (long long)blockIdx.x * WGRAD_CHUNK;
  const long long p_end = min(p_begin + WGRAD_CHUNK, s.pixels());
  const int mtiles = (s.cout + 15) / 16;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int t = 0; t < 4; ++t)
      acc[i][t][0] = acc[i][t][1] = acc[i][t][2] = acc[i][t][3] = 0.f;
  if (kbase < s.kpad) {
    const auto dyv = [&](const long long p, const int n) -> __nv_bfloat16 {
      return (p < p_end && n < s.cout) ? dy[p * s.cout + n] : __float2bfloat16(0.f);
    };
    for (long long p0 = p_begin; p0 < p_end; p0 += 16) {
      // B: rows are pixels p0 + 2q (+1) (+8), columns the warp's k
      unsigned b[4][2];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int k = kbase + t * 8 + g;
        const long long pa = p0 + 2 * q, pb = p0 + 2 * q + 8;
        b[t][0] = pack_bf16(pa < p_end ? im2col_one(x, s, pa, k) : __float2bfloat16(0.f),
                            pa + 1 < p_end ? im2col_one(x, s, pa + 1, k) : __float2bfloat16(0.f));
        b[t][1] = pack_bf16(pb < p_end ? im2col_one(x, s, pb, k) : __float2bfloat16(0.f),
                            pb + 1 < p_end ? im2col_one(x, s, pb + 1, k) : __float2bfloat16(0.f));
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        if (i >= mtiles)
          continue;
        // A: rows are output channels i * 16 + g (+8), columns the pixels
        const int n0 = i * 16 + g, n1 = n0 + 8;
        const long long pa = p0 + 2 * q, pb = p0 + 2 * q + 8;
        unsigned a[4];
        a[0] = pack_bf16(dyv(pa, n0), dyv(pa + 1, n0));
        a[1] = pack_bf16(dyv(pa, n1), dyv(pa + 1, n1));
        a[2] = pack_bf16(dyv(pb, n0), dyv(pb + 1, n0));
        a[3] = pack_bf16(dyv(pb, n1), dyv(pb + 1, n1));
#pragma unroll
        for (int t = 0; t < 4; ++t)
          mma_bf16(acc[i][t], a, b[t]);
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      if (i >= mtiles)
        continue;
#pragma unroll
      for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int n = i * 16 + g + (e >= 2 ? 8 : 0);
          const int k = kbase + t * 8 + 2 * q + (e & 1);
          if (n < s.cout && k < s.kpad)
            atomicAdd(&dw[(long long)n * s.kpad + k], acc[i][t][e]);
        }
    }
  }
}

// the bias gradient: sums of dy over the pixels, per output channel
__global__ void conv_bgrad_kernel(const __nv_bfloat16 *__restrict__ dy, float *__restrict__ db,
                                  const ConvShape s) {
  const int n = threadIdx.x % 32;
  float sum = 0.f;
  if (n < s.cout) {
    const long long stride = (long long)gridDim.x * (blockDim.x / 32);
    for (long long p = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; p < s.pixels();
         p += stride)
      sum += __bfloat162float(dy[p * s.cout + n]);
    atomicAdd(&db[n], sum);
  }
}

cudaError_t conv_forward(const void *x, const void *w, const float *bias, const void *mask,
                         void *y16, float *y32, const ConvShape &s, const int relu,
                         cudaStream_t stream) {
  const long long blocks = (s.pixels() + CONV_WARPS * 16 - 1) / (CONV_WARPS * 16);
  const size_t smem = (size_t)((s.cout + 7) / 8 * 8) * s.kpad * sizeof(__nv_bfloat16);
  if (blocks <= 0 || blocks > 0x7fffffffLL || s.cout > CONV_MAX_N || smem > 200 * 1024)
    return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(conv_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess)
    return e;
  conv_fwd_kernel<<<(unsigned)blocks, CONV_THREADS, smem, stream>>>(
      static_cast<const __nv_bfloat16 *>(x), static_cast<const __nv_bfloat16 *>(w), bias,
      static_cast<const __nv_bfloat16 *>(mask), static_cast<__nv_bfloat16 *>(y16), y32, s, relu);
  return cudaGetLastError();
}

cudaError_t conv_weight_grad(const void *dy, const void *x, float *dw, float *db,
                             const ConvShape &s, cudaStream_t stream) {
  if (s.cout > CONV_MAX_N)
    return cudaErrorInvalidValue;
  const long long chunks = (s.pixels() + WGRAD_CHUNK - 1) / WGRAD_CHUNK;
  const int kgroups = (s.kpad + CONV_WARPS * 32 - 1) / (CONV_WARPS * 32);
  if (chunks <= 0 || chunks > 0x7fffffffLL)
    return cudaErrorInvalidValue;
  conv_wgrad_kernel<<<dim3((unsigned)chunks, kgroups), CONV_THREADS, 0, stream>>>(
      static_cast<const __nv_bfloat16 *>(dy), static_cast<const __nv_bfloat16 *>(x), dw, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !db)
    return e;
  conv_bgrad_kernel<<<296, 256, 0, stream>>>(static_cast<const __nv_bfloat16 *>(dy), db, s);
  return cudaGetLastError();
}

}  // namespace cwb
