// nn.cuh -- kernels of the learned pressure warm start (no reference counterpart).
//
// A small convolutional network predicts the rigid-lid pressure from the barotropic
// divergence and the two previous pressure fields. Activations are NHWC bf16 with the
// channel count a multiple of 16; weights are [Cout][3][3][Cin] bf16 (an FP32 master copy
// is kept for training). The 3x3 convolutions are implicit GEMMs on the 5th-generation
// tensor cores (tcgen05.mma, kind::f16, BF16 operands, FP32 accumulators in tensor
// memory): M = pixels (128 per CTA), N = output channels, K = 9 * input channels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pawsim {
namespace nn {

using bf16 = __nv_bfloat16;

// out[b,y,x,co] = act(bias[co] + sum_{ky,kx,ci} in[b,y+ky-1,x+kx-1,ci] * w[co,ky,kx,ci]),
// zero padding. Cin in {16, 32, 48, 64}, Cout a multiple of 16 up to 64. `relu` applies
// max(0, .). Writes bf16 to out_bf (nullable) and FP32 to out_f32 (nullable). `err` is a
// device int that a kernel sets when one of its bounded waits gives up.
int conv3x3(const bf16* in, int B, int H, int W, int Cin, const bf16* w, const float* bias, int Cout,
            bool relu, bf16* out_bf, float* out_f32, int* err, cudaStream_t s);

// weight gradient: dw[co,ky,kx,ci] += sum_{b,y,x} dout[b,y,x,co] * in[b,y+ky-1,x+kx-1,ci]
// and db[co] += sum dout[b,y,x,co] (FP32, accumulated with atomics)
int conv3x3_wgrad(const bf16* in, const bf16* dout, int B, int H, int W, int Cin, int Cout, float* dw,
                  float* db, int* err, cudaStream_t s);

// w_t[ci,ky,kx,co] = w[co,2-ky,2-kx,ci]: the weights of the transposed convolution, so
// that conv3x3(dout, w_t) is the gradient with respect to the input
int flip_weights(const bf16* w, int Cout, int Cin, bf16* w_t, cudaStream_t s);

}  // namespace nn
}  // namespace pawsim
