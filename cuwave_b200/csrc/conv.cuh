// The corrector's 5x5 convolutions (conv.cu): shapes and host launchers.
#pragma once

#include <cuda_runtime.h>

namespace cwb {

constexpr int CONV_MAX_N = 32;  // output channels of a launch, at most

struct ConvShape {
  int batch, h, w;
  int cin, cout;
  int kpad;  // 25 * cin rounded up to 16
  __host__ __device__ long long pixels() const { return (long long)batch * h * w; }
};

// y = conv(x, w) (+ bias, ReLU), gated by mask > 0 where given; y16 / y32 optional
cudaError_t conv_forward(const void *x, const void *w, const float *bias, const void *mask,
                         void *y16, float *y32, const ConvShape &s, int relu, cudaStream_t stream);
// dw += conv weight gradient of dy against x; db += the bias gradient (optional)
cudaError_t conv_weight_grad(const void *dy, const void *x, float *dw, float *db,
                             const ConvShape &s, cudaStream_t stream);

}  // namespace cwb
