// Pointwise eddy-viscosity MLP 9 -> 64 -> 64 -> 1: the model layout and the
// tcgen05 operand helpers shared by the inference and training kernels
// (sns_mlp.cu) and the fused x pass of the closure step (sns_les.cu).
//
// No reference counterpart (the reference has no subgrid model).  BF16
// weights, inputs and hidden activations; FP32 accumulation and biases;
// ReLU hidden layers; nu_t = s_out * softplus(z).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "sns_tc.cuh"

namespace sns {

constexpr int kMlpHidden = 64;
constexpr int kMlpIn = 9;
constexpr int kMlpK1 = 16;  // inputs padded to one k-tile
// FP32 master parameters: W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3
constexpr int kMlpOffW1 = 0, kMlpOffB1 = 1024, kMlpOffW2 = 1088, kMlpOffB2 = 5184,
              kMlpOffW3 = 5248, kMlpOffB3 = 5312;
constexpr int kMlpParams = 5313;

// Packed inference model (device bytes): bf16 W1[64][16], W2[64][64], w3[64];
// f32 b1[64], b2[64], b3, s_in, s_out.
struct MlpPacked {
  __nv_bfloat16 W1[kMlpHidden * kMlpK1];
  __nv_bfloat16 W2[kMlpHidden * kMlpHidden];
  __nv_bfloat16 w3[kMlpHidden];
  float b1[kMlpHidden];
  float b2[kMlpHidden];
  float b3, s_in, s_out, pad_;
};
static_assert(sizeof(MlpPacked) % 16 == 0, "packed model is copied in 16-byte words");

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float softplus_f(float z) {
  return z > 20.f ? z : log1pf(expf(z));
}

// ---------------------------------------------------------------------------
// The model as tcgen05 operands (sns_tc.cuh layouts): W1 (64 x 16, b1 split
// into two BF16 terms in its padding columns 9, 10), W2 (64 x 64), the
// layer-2 bias slice B2 (64 x 16: b2 hi, lo) and w3 in FP32.  Cooperative
// (nthr threads); the caller synchronises afterwards.
__device__ __forceinline__ uint32_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return (uint32_t)*reinterpret_cast<unsigned short*>(&h);
}

__device__ __forceinline__ void mlp_tc_load_weights(const MlpPacked* __restrict__ P,
                                                    unsigned char* W1, unsigned char* W2,
                                                    unsigned char* B2, float* w3, int tid,
                                                    int nthr) {
  for (int i = tid; i < kMlpHidden * kMlpK1 / 8; i += nthr) {
    const int n = i / (kMlpK1 / 8), c = i % (kMlpK1 / 8);
    uint4 v = reinterpret_cast<const uint4*>(P->W1)[i];
    if (c == 1) {
      const float b = P->b1[n];
      const float hi = __bfloat162float(__float2bfloat16_rn(b));
      v.x = (v.x & 0xFFFFu) | (bf16_bits(hi) << 16);
      v.y = (v.y & 0xFFFF0000u) | bf16_bits(b - hi);
    }
    *reinterpret_cast<uint4*>(W1 + tc::kmajor_off(n, 8 * c, kMlpK1)) = v;
  }
  for (int i = tid; i < kMlpHidden * kMlpHidden / 8; i += nthr) {
    const int n = i / (kMlpHidden / 8), c = i % (kMlpHidden / 8);
    *reinterpret_cast<uint4*>(W2 + tc::kmajor_off(n, 8 * c, kMlpHidden)) =
        reinterpret_cast<const uint4*>(P->W2)[i];
  }
  for (int n = tid; n < kMlpHidden; n += nthr) {
    const float b = P->b2[n];
    const float hi = __bfloat162float(__float2bfloat16_rn(b));
    *reinterpret_cast<uint4*>(B2 + tc::kmajor_off(n, 0, 16)) =
        make_uint4(bf16_bits(hi) | (bf16_bits(b - hi) << 16), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(B2 + tc::kmajor_off(n, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
    w3[n] = __bfloat162float(P->w3[n]);
  }
}

// Rows of the constant A slice (1, 1, 0, ...) that multiplies B2 (rows < nrows)
__device__ __forceinline__ void mlp_tc_fill_ones(unsigned char* ONES, int nrows, int tid,
                                                 int nthr) {
  const uint32_t one = bf16_bits(1.f);
  for (int r = tid; r < nrows; r += nthr) {
    *reinterpret_cast<uint4*>(ONES + tc::kmajor_off(r, 0, 16)) =
        make_uint4(one | (one << 16), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(ONES + tc::kmajor_off(r, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
  }
}

}  // namespace sns
