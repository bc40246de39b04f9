// Pointwise eddy-viscosity MLP 9 -> 64 -> 64 -> 1 on the tensor cores.
//
// No reference counterpart (the reference has no subgrid model).  BF16
// weights, inputs and hidden activations; FP32 accumulation and biases;
// ReLU hidden layers; nu_t = s_out * softplus(z).  The model layout and the
// warp-level forward used inside the fused x pass of the closure step
// (k_xles); the standalone inference and training kernels run on tcgen05
// (sns_mlp.cu, sns_tc.cuh).  The warp-level forward evaluates 16 points
// at a time with mma.sync m16n8k16 (bf16 in, f32 accumulate): the layer-1
// accumulators are rounded to bf16 and reused in registers as the layer-2 A
// operand (the m16n8 accumulator layout of two adjacent n-tiles is the
// m16k16 A layout), and the 64-wide output layer is a dot product reduced
// over the four lanes that share a row.
//
// Fragment layouts (PTX ISA, mma.m16n8k16 .bf16): lane = 4*g + t;
//   A (16x16, row): a0 = A[g][2t..2t+1], a1 = A[g+8][2t..], a2 = A[g][2t+8..],
//                   a3 = A[g+8][2t+8..]   (two bf16 per 32-bit register)
//   B (16x8, col):  b0 = B[2t..2t+1][g], b1 = B[2t+8..2t+9][g]
//   C (16x8, f32):  c0,c1 = C[g][2t..2t+1], c2,c3 = C[g+8][2t..2t+1]
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

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

// Shared-memory copy of the model with padded rows: a row stride of 12 / 36
// 32-bit words puts the eight g-rows of a B fragment on distinct banks.
constexpr int kW1Stride = kMlpK1 + 8;      // bf16 per W1 row (48 bytes)
constexpr int kW2Stride = kMlpHidden + 8;  // bf16 per W2 row (144 bytes)
// 16-byte aligned: ldmatrix reads its rows
struct __align__(16) MlpSmem {
  __nv_bfloat16 W1[kMlpHidden * kW1Stride];
  __nv_bfloat16 W2[kMlpHidden * kW2Stride];
  float w3[kMlpHidden];
  float b1[kMlpHidden];
  float b2[kMlpHidden];
  float b3, s_in, s_out, pad_;
};

// Cooperative copy of the packed model into shared memory (all threads of
// the CTA; the caller synchronises afterwards).
__device__ __forceinline__ void mlp_load_smem(const MlpPacked* __restrict__ p, MlpSmem& s,
                                              int tid, int nthr) {
  for (int i = tid; i < kMlpHidden * kMlpK1 / 2; i += nthr) {
    const int r = (2 * i) / kMlpK1, c = (2 * i) % kMlpK1;
    *reinterpret_cast<uint32_t*>(&s.W1[r * kW1Stride + c]) =
        reinterpret_cast<const uint32_t*>(p->W1)[i];
  }
  for (int i = tid; i < kMlpHidden * kMlpHidden / 2; i += nthr) {
    const int r = (2 * i) / kMlpHidden, c = (2 * i) % kMlpHidden;
    *reinterpret_cast<uint32_t*>(&s.W2[r * kW2Stride + c]) =
        reinterpret_cast<const uint32_t*>(p->W2)[i];
  }
  for (int i = tid; i < kMlpHidden; i += nthr) {
    s.w3[i] = __bfloat162float(p->w3[i]);
    s.b1[i] = p->b1[i];
    s.b2[i] = p->b2[i];
  }
  if (tid == 0) {
    s.b3 = p->b3;
    s.s_in = p->s_in;
    s.s_out = p->s_out;
  }
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                               uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ldmatrix: lanes 8m..8m+7 give the row addresses of 8x8 bf16 matrix m; lane
// l receives row l/4, columns 2(l%4), 2(l%4)+1 of each matrix.  Rows must
// start on 16-byte boundaries.
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low half), .y = hi
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ float softplus_f(float z) {
  return z > 20.f ? z : log1pf(expf(z));
}

// Layer activations of one 16-row tile, in fragment layout.
struct MlpTile {
  uint32_t h1[4][4];  // layer-1 output (bf16) as the A operand of layer 2, per k-tile
  float z[2];         // output pre-activation of rows g and g + 8
};

// Forward of one 16-row tile whose A operand (inputs) is xa.
__device__ __forceinline__ void mlp_tile_forward(const MlpSmem& s, const uint32_t (&xa)[4],
                                                 MlpTile& T) {
  const int lane = threadIdx.x & 31, t = lane & 3;
  const int lm = lane >> 3, lr = lane & 7;  // ldmatrix: matrix and row of this lane's address
  // layer 1: [16 x 16] x [16 x 64]; B[k][n] = W1[n][k], two n-tiles per ldmatrix
  uint32_t b1f[4];
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    if ((nt & 1) == 0)
      ldsm_x4(b1f, &s.W1[((nt + (lm >> 1)) * 8 + lr) * kW1Stride + (lm & 1) * 8]);
    mma_bf16_16816(c, xa, b1f[(nt & 1) * 2], b1f[(nt & 1) * 2 + 1]);
    const float bl = s.b1[nt * 8 + 2 * t], bh = s.b1[nt * 8 + 2 * t + 1];
    c[0] += bl;
    c[1] += bh;
    c[2] += bl;
    c[3] += bh;
    const uint32_t lo = pack_bf16(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f));
    const uint32_t hi = pack_bf16(fmaxf(c[2], 0.f), fmaxf(c[3], 0.f));
    // n-tile nt holds columns 8nt..8nt+7 = k-tile nt/2, half nt%2
    T.h1[nt >> 1][(nt & 1) ? 2 : 0] = lo;
    T.h1[nt >> 1][(nt & 1) ? 3 : 1] = hi;
  }
  // layer 2: [16 x 64] x [64 x 64]
  float zl = 0.f, zh = 0.f;
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kp = 0; kp < 2; kp++) {
      // B[k][n] = W2[n][k]: k-tiles 2kp and 2kp+1 of n-tile nt in one ldmatrix
      uint32_t b[4];
      ldsm_x4(b, &s.W2[(nt * 8 + lr) * kW2Stride + (2 * kp + (lm >> 1)) * 16 + (lm & 1) * 8]);
      mma_bf16_16816(c, T.h1[2 * kp], b[0], b[1]);
      mma_bf16_16816(c, T.h1[2 * kp + 1], b[2], b[3]);
    }
    const int col = nt * 8 + 2 * t;
    const float bl = s.b2[col], bh = s.b2[col + 1];
    c[0] += bl;
    c[1] += bh;
    c[2] += bl;
    c[3] += bh;
    // layer 3: dot product with w3 over this lane's columns
    const float wl = s.w3[col], wh = s.w3[col + 1];
    zl += fmaxf(c[0], 0.f) * wl + fmaxf(c[1], 0.f) * wh;
    zh += fmaxf(c[2], 0.f) * wl + fmaxf(c[3], 0.f) * wh;
  }
  zl += __shfl_xor_sync(0xffffffffu, zl, 1);
  zl += __shfl_xor_sync(0xffffffffu, zl, 2);
  zh += __shfl_xor_sync(0xffffffffu, zh, 1);
  zh += __shfl_xor_sync(0xffffffffu, zh, 2);
  T.z[0] = zl + s.b3;
  T.z[1] = zh + s.b3;
}

}  // namespace sns
