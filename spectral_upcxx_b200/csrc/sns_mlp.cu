// Training and inference of the eddy-viscosity MLP (sns_mlp.cuh) on the
// tensor cores.  No reference counterpart.
//
// One training step over a batch of B samples is three launches:
//   k_mlp_grad    CTAs of 128 samples (4 warps x 2 tiles of 16 rows): forward,
//                 loss, backward through the three layers with mma.sync
//                 (dH1 = dPre2 W2), then the weight gradients as GEMMs over the
//                 CTA's samples (dW2 = dPre2^T H1, dW1 = dPre1^T X) from
//                 transposed bf16 copies in shared memory; per-CTA partial
//                 gradients go to a work array
//   k_mlp_reduce  sums the partials in a fixed order (deterministic)
//   k_mlp_adam    Adam on the FP32 masters, then the bf16 inference copy
// Rounding points: inputs, W1, W2, w3, the layer-1 activations and the
// backward operands dPre2, dPre1 are bf16; everything else is FP32.
#include <cuda_bf16.h>
#include <math.h>

#include <string>
#include <vector>

#include "../../include/spectral_b200.h"
#include "sns_common.cuh"
#include "sns_ens.cuh"
#include "sns_mlp.cuh"
#include "sns_tc.cuh"

namespace sns {

constexpr int kTrainWarps = 4;
constexpr int kTrainRows = kTrainWarps * 32;  // samples per CTA
constexpr int kTS = kTrainRows + 8;           // bf16 stride of the transposed tiles
constexpr int kPart = kMlpParams + 1;         // gradients + loss sum

struct TrainSmem {
  MlpSmem m;
  __nv_bfloat16 XT[kMlpK1 * kTS];             // inputs, [feature][sample]
  __nv_bfloat16 H1T[kMlpHidden * kTS];        // layer-1 activations, [unit][sample]
  __nv_bfloat16 P2T[kMlpHidden * kTS];        // dPre2, [unit][sample]
  __nv_bfloat16 P1T[kMlpHidden * kTS];        // dPre1, [unit][sample]
  float vec[kTrainWarps][3][kMlpHidden];      // per-warp db1, db2, dw3
  float scal[kTrainWarps][2];                 // per-warp db3, loss sum
};

__global__ void __launch_bounds__(kTrainRows)
    k_mlp_grad(const MlpPacked* __restrict__ P, const __nv_bfloat16* __restrict__ X,
               const float* __restrict__ target, const float* __restrict__ weight,
               const int* __restrict__ idx, int64_t B, float inv_batch,
               float* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  mlp_load_smem(P, S.m, tid, blockDim.x);
  __syncthreads();
  const int lm = lane >> 3, lr = lane & 7;

  float db1[8][2], db2[8][2], dw3[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; nt++)
#pragma unroll
    for (int q = 0; q < 2; q++) db1[nt][q] = db2[nt][q] = dw3[nt][q] = 0.f;
  float db3 = 0.f, loss = 0.f;

  for (int tile = 0; tile < 2; tile++) {
    const int s0 = warp * 32 + tile * 16;  // first sample (CTA-local) of the tile
    const int64_t b0 = (int64_t)blockIdx.x * kTrainRows + s0;
    // rows g and g + 8 of this tile
    const int64_t ra = b0 + g, rb = b0 + g + 8;
    const bool va = ra < B, vb = rb < B;
    const int64_t xa_row = va ? (idx ? idx[ra] : ra) : 0;
    const int64_t xb_row = vb ? (idx ? idx[rb] : rb) : 0;
    uint32_t xa[4];
    {
      const uint32_t* pa = reinterpret_cast<const uint32_t*>(X + xa_row * kMlpK1);
      const uint32_t* pb = reinterpret_cast<const uint32_t*>(X + xb_row * kMlpK1);
      xa[0] = va ? pa[t] : 0u;
      xa[1] = vb ? pb[t] : 0u;
      xa[2] = va ? pa[t + 4] : 0u;
      xa[3] = vb ? pb[t + 4] : 0u;
      // transposed copy for dW1
      S.XT[(2 * t) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(xa[0] & 0xffff));
      S.XT[(2 * t + 1) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(xa[0] >> 16));
      S.XT[(2 * t) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(xa[1] & 0xffff));
      S.XT[(2 * t + 1) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(xa[1] >> 16));
      S.XT[(2 * t + 8) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(xa[2] & 0xffff));
      S.XT[(2 * t + 9) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(xa[2] >> 16));
      S.XT[(2 * t + 8) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(xa[3] & 0xffff));
      S.XT[(2 * t + 9) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(xa[3] >> 16));
    }
    MlpTile T;
    mlp_tile_forward<true>(S.m, xa, T);
    // loss and dL/dz for rows g and g + 8 (the four lanes of a row agree)
    float dz[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const bool v = h ? vb : va;
      const int64_t r = h ? xb_row : xa_row;
      const float z = T.z[h];
      const float y = softplus_f(z);
      const float d = v ? y - target[r] : 0.f;
      const float wt = (v && weight) ? weight[r] : 1.f;
      if (t == 0) loss += wt * d * d;
      dz[h] = 2.f * inv_batch * wt * d / (1.f + expf(-z));
      if (t == 0) db3 += dz[h];
    }
    // layer 3 and layer-2 activation gradients; dPre2 as bf16 A fragments
    uint32_t p2a[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int col = nt * 8 + 2 * t;
      const float wl = S.m.w3[col], wh = S.m.w3[col + 1];
      float h2[4], dp[4];
#pragma unroll
      for (int q = 0; q < 4; q++) h2[q] = fmaxf(T.pre2[nt][q], 0.f);
      dw3[nt][0] += dz[0] * h2[0] + dz[1] * h2[2];
      dw3[nt][1] += dz[0] * h2[1] + dz[1] * h2[3];
      dp[0] = T.pre2[nt][0] > 0.f ? dz[0] * wl : 0.f;
      dp[1] = T.pre2[nt][1] > 0.f ? dz[0] * wh : 0.f;
      dp[2] = T.pre2[nt][2] > 0.f ? dz[1] * wl : 0.f;
      dp[3] = T.pre2[nt][3] > 0.f ? dz[1] * wh : 0.f;
      db2[nt][0] += dp[0] + dp[2];
      db2[nt][1] += dp[1] + dp[3];
      const uint32_t lo = pack_bf16(dp[0], dp[1]), hi = pack_bf16(dp[2], dp[3]);
      p2a[nt >> 1][(nt & 1) ? 2 : 0] = lo;
      p2a[nt >> 1][(nt & 1) ? 3 : 1] = hi;
      // transposed copies for the weight gradients
      S.P2T[col * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(lo & 0xffff));
      S.P2T[(col + 1) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(lo >> 16));
      S.P2T[col * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(hi & 0xffff));
      S.P2T[(col + 1) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(hi >> 16));
      const uint32_t h1lo = T.h1[nt >> 1][(nt & 1) ? 2 : 0];
      const uint32_t h1hi = T.h1[nt >> 1][(nt & 1) ? 3 : 1];
      S.H1T[col * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(h1lo & 0xffff));
      S.H1T[(col + 1) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(h1lo >> 16));
      S.H1T[col * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(h1hi & 0xffff));
      S.H1T[(col + 1) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(h1hi >> 16));
    }
    // dH1 = dPre2 W2 ([16 x 64] x [64 x 64]); dPre1 = dH1 * (pre1 > 0)
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int kp = 0; kp < 2; kp++) {
        // B[k = n2][n = n1] = W2[n2][n1]: transposed 8x8 matrices of W2's rows
        // 16 kt + 0..15, columns 8 nt..8 nt+7, for k-tiles 2kp and 2kp+1
        uint32_t b[4];
        ldsm_x4_trans(b, &S.m.W2[((2 * kp + (lm >> 1)) * 16 + (lm & 1) * 8 + lr) * kW2Stride +
                                 nt * 8]);
        mma_bf16_16816(c, p2a[2 * kp], b[0], b[1]);
        mma_bf16_16816(c, p2a[2 * kp + 1], b[2], b[3]);
      }
      const int col = nt * 8 + 2 * t;
      float dp[4];
#pragma unroll
      for (int q = 0; q < 4; q++) dp[q] = T.pre1[nt][q] > 0.f ? c[q] : 0.f;
      db1[nt][0] += dp[0] + dp[2];
      db1[nt][1] += dp[1] + dp[3];
      const uint32_t lo = pack_bf16(dp[0], dp[1]), hi = pack_bf16(dp[2], dp[3]);
      S.P1T[col * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(lo & 0xffff));
      S.P1T[(col + 1) * kTS + s0 + g] = __ushort_as_bfloat16((unsigned short)(lo >> 16));
      S.P1T[col * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(hi & 0xffff));
      S.P1T[(col + 1) * kTS + s0 + g + 8] = __ushort_as_bfloat16((unsigned short)(hi >> 16));
    }
  }
  // per-warp vectors: reduce over the eight row groups g (lanes with equal t)
#pragma unroll
  for (int nt = 0; nt < 8; nt++)
#pragma unroll
    for (int q = 0; q < 2; q++) {
#pragma unroll
      for (int o = 4; o < 32; o <<= 1) {
        db1[nt][q] += __shfl_xor_sync(0xffffffffu, db1[nt][q], o);
        db2[nt][q] += __shfl_xor_sync(0xffffffffu, db2[nt][q], o);
        dw3[nt][q] += __shfl_xor_sync(0xffffffffu, dw3[nt][q], o);
      }
    }
#pragma unroll
  for (int o = 4; o < 32; o <<= 1) {
    db3 += __shfl_xor_sync(0xffffffffu, db3, o);
    loss += __shfl_xor_sync(0xffffffffu, loss, o);
  }
  if (g == 0) {
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int col = nt * 8 + 2 * t + q;
        S.vec[warp][0][col] = db1[nt][q];
        S.vec[warp][1][col] = db2[nt][q];
        S.vec[warp][2][col] = dw3[nt][q];
      }
  }
  if (lane == 0) {
    S.scal[warp][0] = db3;
    S.scal[warp][1] = loss;
  }
  __syncthreads();

  float* out = part + (int64_t)blockIdx.x * kPart;
  // dW2[n2][n1] = sum_s dPre2[s][n2] H1[s][n1]: warp w owns rows n2 in [16w, 16w + 16)
  {
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[nt][q] = 0.f;
#pragma unroll
    for (int ks = 0; ks < kTrainRows / 16; ks++) {
      uint32_t a[4];
      load_a_tile(&S.P2T[(16 * warp) * kTS + 16 * ks], kTS, a);
#pragma unroll
      for (int nt = 0; nt < 8; nt += 2) {
        uint32_t b[4];
        load_b_pair(&S.H1T[(nt * 8) * kTS + 16 * ks], kTS, b);
        mma_bf16_16816(acc[nt], a, b[0], b[1]);
        mma_bf16_16816(acc[nt + 1], a, b[2], b[3]);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int r0 = 16 * warp + g, c0 = nt * 8 + 2 * t;
      out[kMlpOffW2 + r0 * kMlpHidden + c0] = acc[nt][0];
      out[kMlpOffW2 + r0 * kMlpHidden + c0 + 1] = acc[nt][1];
      out[kMlpOffW2 + (r0 + 8) * kMlpHidden + c0] = acc[nt][2];
      out[kMlpOffW2 + (r0 + 8) * kMlpHidden + c0 + 1] = acc[nt][3];
    }
  }
  // dW1[n1][f] = sum_s dPre1[s][n1] X[s][f]: warp w owns rows n1 in [16w, 16w + 16)
  {
    float acc[2][4];
#pragma unroll
    for (int nt = 0; nt < 2; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[nt][q] = 0.f;
#pragma unroll
    for (int ks = 0; ks < kTrainRows / 16; ks++) {
      uint32_t a[4];
      load_a_tile(&S.P1T[(16 * warp) * kTS + 16 * ks], kTS, a);
      {
        uint32_t b[4];
        load_b_pair(&S.XT[16 * ks], kTS, b);
        mma_bf16_16816(acc[0], a, b[0], b[1]);
        mma_bf16_16816(acc[1], a, b[2], b[3]);
      }
    }
#pragma unroll
    for (int nt = 0; nt < 2; nt++) {
      const int r0 = 16 * warp + g, c0 = nt * 8 + 2 * t;
      out[kMlpOffW1 + r0 * kMlpK1 + c0] = acc[nt][0];
      out[kMlpOffW1 + r0 * kMlpK1 + c0 + 1] = acc[nt][1];
      out[kMlpOffW1 + (r0 + 8) * kMlpK1 + c0] = acc[nt][2];
      out[kMlpOffW1 + (r0 + 8) * kMlpK1 + c0 + 1] = acc[nt][3];
    }
  }
  // vectors and scalars, summed over the warps in a fixed order
  for (int i = tid; i < kMlpHidden; i += blockDim.x) {
    float a = 0.f, b = 0.f, c = 0.f;
    for (int w = 0; w < kTrainWarps; w++) {
      a += S.vec[w][0][i];
      b += S.vec[w][1][i];
      c += S.vec[w][2][i];
    }
    out[kMlpOffB1 + i] = a;
    out[kMlpOffB2 + i] = b;
    out[kMlpOffW3 + i] = c;
  }
  if (tid == 0) {
    float a = 0.f, l = 0.f;
    for (int w = 0; w < kTrainWarps; w++) {
      a += S.scal[w][0];
      l += S.scal[w][1];
    }
    out[kMlpOffB3] = a;
    out[kMlpParams] = l;
  }
}

// grad[p] = sum over CTAs of part[cta][p] (fixed order); the loss entry is
// turned into the batch mean.
__global__ void k_mlp_reduce(const float* __restrict__ part, int nblocks, float inv_batch,
                             float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kPart) return;
  float s = 0.f;
  for (int b = 0; b < nblocks; b++) s += part[(int64_t)b * kPart + p];
  grad[p] = p == kMlpParams ? s * inv_batch : s;
}

// Adam (bias-corrected) on the FP32 masters; writes the bf16 inference copy.
__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ grad, float lr, float b1, float b2,
                           float eps, float c1, float c2, MlpPacked* __restrict__ P) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const float gr = grad[p];
  const float mi = b1 * m[p] + (1.f - b1) * gr;
  const float vi = b2 * v[p] + (1.f - b2) * gr * gr;
  m[p] = mi;
  v[p] = vi;
  float x = w[p] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  // the padding columns of W1 stay zero
  if (p < kMlpOffB1 && (p % kMlpK1) >= kMlpIn) x = 0.f;
  w[p] = x;
  if (p < kMlpOffB1)
    P->W1[p] = __float2bfloat16_rn(x);
  else if (p < kMlpOffW2)
    P->b1[p - kMlpOffB1] = x;
  else if (p < kMlpOffB2)
    P->W2[p - kMlpOffW2] = __float2bfloat16_rn(x);
  else if (p < kMlpOffW3)
    P->b2[p - kMlpOffB2] = x;
  else if (p < kMlpOffB3)
    P->w3[p - kMlpOffW3] = __float2bfloat16_rn(x);
  else
    P->b3 = x;
}

__global__ void k_mlp_pack(const float* __restrict__ w, float s_in, float s_out,
                           MlpPacked* __restrict__ P) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) {
    P->s_in = s_in;
    P->s_out = s_out;
    P->pad_ = 0.f;
  }
  if (p >= kMlpParams) return;
  const float x = w[p];
  if (p < kMlpOffB1)
    P->W1[p] = __float2bfloat16_rn(x);
  else if (p < kMlpOffW2)
    P->b1[p - kMlpOffB1] = x;
  else if (p < kMlpOffB2)
    P->W2[p - kMlpOffW2] = __float2bfloat16_rn(x);
  else if (p < kMlpOffW3)
    P->b2[p - kMlpOffB2] = x;
  else if (p < kMlpOffB3)
    P->w3[p - kMlpOffW3] = __float2bfloat16_rn(x);
  else
    P->b3 = x;
}

// nu_t = s_out softplus(z) for M rows of bf16 features (warps of 16 rows).
__global__ void __launch_bounds__(256)
    k_mlp_infer(const MlpPacked* __restrict__ P, const __nv_bfloat16* __restrict__ X, int64_t M,
                float* __restrict__ nut) {
  __shared__ MlpSmem S;
  mlp_load_smem(P, S, threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 16; r0 < M;
       r0 += warps * 16) {
    const int64_t ra = r0 + g, rb = r0 + g + 8;
    const uint32_t* pa = reinterpret_cast<const uint32_t*>(X + (ra < M ? ra : 0) * kMlpK1);
    const uint32_t* pb = reinterpret_cast<const uint32_t*>(X + (rb < M ? rb : 0) * kMlpK1);
    uint32_t xa[4] = {ra < M ? pa[t] : 0u, rb < M ? pb[t] : 0u, ra < M ? pa[t + 4] : 0u,
                      rb < M ? pb[t + 4] : 0u};
    MlpTile T;
    mlp_tile_forward<false>(S, xa, T);
    if (t == 0) {
      if (ra < M) nut[ra] = S.s_out * softplus_f(T.z[0]);
      if (rb < M) nut[rb] = S.s_out * softplus_f(T.z[1]);
    }
  }
}

// ---------------------------------------------------------------------------
// Inference on the fifth-generation tensor cores: a CTA of 128 threads takes
// tiles of 128 points; thread m owns point m of the tile (its input row, its
// accumulator lane in tensor memory and its output).  The biases ride in the
// MMAs: input columns 9 and 10 (padding) are set to 1 in the A tile and the
// matching columns of W1 hold b1 split into two BF16 terms (hi + lo = b1 to
// 16 bits); layer 2 gets a fifth K-slice whose A rows are (1, 1, 0, ...) and
// whose B rows are (b2 hi, b2 lo, 0, ...).  Per tile: layer 1 is one
// tcgen05.mma (M 128, N 64, K 16) into 64 tensor-memory columns, the epilogue
// reads them back (ReLU, BF16) into the layer-2 A tile, layer 2 is five MMAs
// into the same columns, and the output epilogue forms
// s_out softplus(relu(.) . w3 + b3) per lane.  Rounding points as in the
// mma.sync path: hidden layer 1 rounded to BF16, layer 2 kept in FP32.
constexpr int kTcRows = 128;
constexpr int kTcCols = 64;  // tensor-memory columns: the accumulator of either layer

struct __align__(128) TcSmem {
  unsigned char W1[kMlpHidden * kMlpK1 * 2];       // B of layer 1 (b1 in columns 9, 10)
  unsigned char W2[kMlpHidden * kMlpHidden * 2];   // B of layer 2, K-slices 0..3
  unsigned char B2[kMlpHidden * 16 * 2];           // B of layer 2, bias slice
  unsigned char X[kTcRows * kMlpK1 * 2];           // A of layer 1
  unsigned char H[kTcRows * kMlpHidden * 2];       // A of layer 2, K-slices 0..3
  unsigned char ONES[kTcRows * 16 * 2];            // A of layer 2, bias slice
  float w3[kMlpHidden];
  float b3, s_out;
  uint64_t mbar;
  uint32_t tmem;
  int abort;
};

__device__ int g_mlp_tc_status;  // nonzero: a tensor-core wait ran out

__device__ __forceinline__ uint32_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return (uint32_t)*reinterpret_cast<unsigned short*>(&h);
}

__global__ void __launch_bounds__(kTcRows)
    k_mlp_infer_tc(const MlpPacked* __restrict__ P, const __nv_bfloat16* __restrict__ X,
                   int64_t M, float* __restrict__ nut) {
  extern __shared__ __align__(128) unsigned char tc_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  // weights into the K-major operand layouts, 16 bytes (8 bf16 along k) at a time
  for (int i = tid; i < kMlpHidden * kMlpK1 / 8; i += kTcRows) {
    const int n = i / (kMlpK1 / 8), c = i % (kMlpK1 / 8);
    uint4 v = reinterpret_cast<const uint4*>(P->W1)[i];
    if (c == 1) {
      // W1 columns 9, 10 (zero in the model) carry b1 = hi + lo
      const float b = P->b1[n];
      const float hi = __bfloat162float(__float2bfloat16_rn(b));
      v.x = (v.x & 0xFFFFu) | (bf16_bits(hi) << 16);
      v.y = (v.y & 0xFFFF0000u) | bf16_bits(b - hi);
    }
    *reinterpret_cast<uint4*>(S.W1 + tc::kmajor_off(n, 8 * c, kMlpK1)) = v;
  }
  for (int i = tid; i < kMlpHidden * kMlpHidden / 8; i += kTcRows) {
    const int n = i / (kMlpHidden / 8), c = i % (kMlpHidden / 8);
    *reinterpret_cast<uint4*>(S.W2 + tc::kmajor_off(n, 8 * c, kMlpHidden)) =
        reinterpret_cast<const uint4*>(P->W2)[i];
  }
  for (int n = tid; n < kMlpHidden; n += kTcRows) {
    const float b = P->b2[n];
    const float hi = __bfloat162float(__float2bfloat16_rn(b));
    *reinterpret_cast<uint4*>(S.B2 + tc::kmajor_off(n, 0, 16)) =
        make_uint4(bf16_bits(hi) | (bf16_bits(b - hi) << 16), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(S.B2 + tc::kmajor_off(n, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
    S.w3[n] = __bfloat162float(P->w3[n]);
  }
  {
    const uint32_t one = bf16_bits(1.f);
    *reinterpret_cast<uint4*>(S.ONES + tc::kmajor_off(tid, 0, 16)) =
        make_uint4(one | (one << 16), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(S.ONES + tc::kmajor_off(tid, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) {
    S.b3 = P->b3;
    S.s_out = P->s_out;
    S.abort = 0;
    tc::mbar_init(&S.mbar, 1);
  }
  if (warp == 0) {
    tc::tmem_alloc(&S.tmem, kTcCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;  // this warp's accumulator lanes
  const uint32_t sX = tc::smem_u32(S.X), sH = tc::smem_u32(S.H), sO = tc::smem_u32(S.ONES);
  const uint32_t sW1 = tc::smem_u32(S.W1), sW2 = tc::smem_u32(S.W2), sB2 = tc::smem_u32(S.B2);
  constexpr uint32_t id = tc::idesc_bf16(kTcRows, kMlpHidden);
  const uint32_t one2 = bf16_bits(1.f) * 0x10001u;
  uint32_t phase = 0;
  const int64_t tiles = (M + kTcRows - 1) / kTcRows;
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row = tile * kTcRows + tid;
    {
      uint4 x0 = make_uint4(0, 0, 0, 0), x1 = x0;
      if (row < M) {
        const uint4* src = reinterpret_cast<const uint4*>(X + row * kMlpK1);
        x0 = src[0];
        x1 = src[1];
      }
      // columns 9, 10: the constant 1 of the b1 terms
      x1.x = (x1.x & 0xFFFFu) | (one2 & 0xFFFF0000u);
      x1.y = (x1.y & 0xFFFF0000u) | (one2 & 0xFFFFu);
      *reinterpret_cast<uint4*>(S.X + tc::kmajor_off(tid, 0, kMlpK1)) = x0;
      *reinterpret_cast<uint4*>(S.X + tc::kmajor_off(tid, 8, kMlpK1)) = x1;
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      tc::mma_bf16(tmem, tc::sdesc(sX, 128, 16 * kMlpK1), tc::sdesc(sW1, 128, 16 * kMlpK1), id, 0);
      tc::commit(&S.mbar);
    }
    if (!tc::mbar_wait(&S.mbar, phase, tc::kWaitCycles)) S.abort = 1;
    phase ^= 1;
    tc::fence_after_sync();
    __syncthreads();
    if (S.abort) break;
    // layer-1 epilogue: h1 = bf16(relu(acc)) into the layer-2 A tile
#pragma unroll
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + lane_base + c0, r);
      uint32_t h[8];
#pragma unroll
      for (int j = 0; j < 8; j++)
        h[j] = pack_bf16(fmaxf(__uint_as_float(r[2 * j]), 0.f),
                         fmaxf(__uint_as_float(r[2 * j + 1]), 0.f));
      *reinterpret_cast<uint4*>(S.H + tc::kmajor_off(tid, c0, kMlpHidden)) =
          make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(S.H + tc::kmajor_off(tid, c0 + 8, kMlpHidden)) =
          make_uint4(h[4], h[5], h[6], h[7]);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < kMlpHidden / 16; s++)
        tc::mma_bf16(tmem, tc::sdesc(sH + 256 * s, 128, 16 * kMlpHidden),
                     tc::sdesc(sW2 + 256 * s, 128, 16 * kMlpHidden), id, s > 0);
      tc::mma_bf16(tmem, tc::sdesc(sO, 128, 256), tc::sdesc(sB2, 128, 256), id, 1);
      tc::commit(&S.mbar);
    }
    if (!tc::mbar_wait(&S.mbar, phase, tc::kWaitCycles)) S.abort = 1;
    phase ^= 1;
    tc::fence_after_sync();
    __syncthreads();
    if (S.abort) break;
    // output epilogue
    float z = 0.f;
#pragma unroll
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + lane_base + c0, r);
#pragma unroll
      for (int j = 0; j < 16; j++) z += fmaxf(__uint_as_float(r[j]), 0.f) * S.w3[c0 + j];
    }
    if (row < M) nut[row] = S.s_out * softplus_f(z + S.b3);
    tc::fence_before_sync();
  }
  __syncthreads();
  if (S.abort) {
    // the MMA whose wait ran out may still be in flight: one more bounded wait
    tc::mbar_wait(&S.mbar, phase ^ 1, tc::kWaitCycles);
    if (tid == 0) atomicExch(&g_mlp_tc_status, 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTcCols);
  }
}

namespace {

int grad_launch(const void* packed, const void* X, const float* t, const float* w,
                const int* idx, int64_t B, float* grad, cudaStream_t s) {
  const int64_t nb = (B + kTrainRows - 1) / kTrainRows;
  if (nb > (1 << 24)) {
    set_error("sns_mlp_grad: batch too large");
    return ERR_UNSUPPORTED;
  }
  void* part = nullptr;
  int rc = pool_malloc(&part, sizeof(float) * kPart * nb);
  if (rc) return rc;
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    rc = cuda_status(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(TrainSmem)),
                     "cudaFuncSetAttribute(k_mlp_grad)");
    if (rc) {
      pool_free(part);
      return rc;
    }
    attr[dev & 63] = true;
  }
  const float inv = (float)(1.0 / (double)B);
  k_mlp_grad<<<(unsigned)nb, kTrainRows, sizeof(TrainSmem), s>>>(
      reinterpret_cast<const MlpPacked*>(packed), reinterpret_cast<const __nv_bfloat16*>(X), t, w,
      idx, B, inv, reinterpret_cast<float*>(part));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_mlp_reduce<<<(kPart + 255) / 256, 256, 0, s>>>(reinterpret_cast<float*>(part), (int)nb, inv,
                                                    grad);
    e = cudaGetLastError();
  }
  // the pool may hand the block to any later caller: wait for the kernels
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  pool_free(part);
  return cuda_status(e, "k_mlp_grad");
}

}  // namespace
}  // namespace sns

using namespace sns;

extern "C" {

int sns_mlp_sizes(int64_t* nparams, int64_t* packed_bytes) {
  if (nparams) *nparams = kMlpParams;
  if (packed_bytes) *packed_bytes = (int64_t)sizeof(MlpPacked);
  return OK;
}

int sns_mlp_pack(const float* master, double s_in, double s_out, void* packed, void* stream) {
  if (!master || !packed) {
    set_error("sns_mlp_pack: null pointer");
    return ERR_ARG;
  }
  k_mlp_pack<<<(kMlpParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      master, (float)s_in, (float)s_out, reinterpret_cast<MlpPacked*>(packed));
  SNS_CHECK_LAUNCH("k_mlp_pack");
  return OK;
}

int sns_mlp_infer(const void* packed, const void* X, int64_t M, float* nut, void* stream) {
  if (!packed || (M > 0 && (!X || !nut)) || M < 0) {
    set_error("sns_mlp_infer: bad arguments");
    return ERR_ARG;
  }
  if (M == 0) return OK;
  if (reinterpret_cast<uintptr_t>(X) % 16 || reinterpret_cast<uintptr_t>(packed) % 16) {
    set_error("sns_mlp_infer: X and the packed model must be 16-byte aligned");
    return ERR_ARG;
  }
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    int rc = cuda_status(cudaFuncSetAttribute(k_mlp_infer_tc,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)sizeof(TcSmem)),
                         "cudaFuncSetAttribute(k_mlp_infer_tc)");
    if (rc) return rc;
    attr[dev & 63] = true;
  }
  // one persistent wave: the resident CTAs per SM (at most eight share an SM's
  // 512 tensor-memory columns)
  // (shared memory sets it: registers and threads allow more)
  static int per_sm[64] = {0};
  if (!per_sm[dev & 63]) {
    int smem_sm = 0, resv = 0;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&resv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    const int occ = smem_sm / (int)(sizeof(TcSmem) + resv);
    per_sm[dev & 63] = std::max(1, std::min(occ, 512 / kTcCols));
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t tiles = (M + kTcRows - 1) / kTcRows;
  const int blocks = (int)std::min<int64_t>(tiles, (int64_t)per_sm[dev & 63] * sms);
  k_mlp_infer_tc<<<blocks, kTcRows, sizeof(TcSmem), reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const MlpPacked*>(packed), reinterpret_cast<const __nv_bfloat16*>(X), M,
      nut);
  SNS_CHECK_LAUNCH("k_mlp_infer_tc");
  return OK;
}

int sns_mlp_status(void) {
  int v = 0;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpyFromSymbol(&v, g_mlp_tc_status, sizeof(int));
  if (e == cudaSuccess && v) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_mlp_tc_status, &zero, sizeof(int));
  }
  if (e != cudaSuccess) return cuda_status(e, "sns_mlp_status");
  if (v) {
    set_error("a tensor-core MLP kernel gave up waiting for its MMAs");
    return ERR_TIMEOUT;
  }
  return OK;
}

int sns_mlp_grad(const void* packed, const void* X, const float* target, const float* weight,
                 const int* idx, int64_t B, float* grad, void* stream) {
  if (!packed || !X || !target || !grad || B < 1) {
    set_error("sns_mlp_grad: bad arguments");
    return ERR_ARG;
  }
  return grad_launch(packed, X, target, weight, idx, B, grad,
                     reinterpret_cast<cudaStream_t>(stream));
}

int sns_mlp_adam(float* master, float* m, float* v, const float* grad, int step, double lr,
                 double beta1, double beta2, double eps, void* packed, void* stream) {
  if (!master || !m || !v || !grad || !packed || step < 1) {
    set_error("sns_mlp_adam: bad arguments");
    return ERR_ARG;
  }
  const double c1 = 1.0 - pow(beta1, step), c2 = 1.0 - pow(beta2, step);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      master, m, v, grad, (float)lr, (float)beta1, (float)beta2, (float)eps, (float)c1, (float)c2,
      reinterpret_cast<MlpPacked*>(packed));
  SNS_CHECK_LAUNCH("k_mlp_adam");
  return OK;
}

}  // extern "C"
