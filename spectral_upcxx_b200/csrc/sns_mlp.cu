// Training and inference of the eddy-viscosity MLP (sns_mlp.cuh) on the
// fifth-generation tensor cores (tcgen05, sns_tc.cuh).  No reference
// counterpart.
//
//   k_mlp_infer_tc  nu_t of M points, tiles of 128 points per CTA
// One training step over a batch of B samples is three launches:
//   k_mlp_grad_tc   persistent CTAs walking tiles of 128 samples: forward,
//                   loss, backward, the weight gradients accumulated in
//                   tensor memory; one partial gradient per CTA
//   k_mlp_reduce    sums the partials in a fixed order (deterministic)
//   k_mlp_adam      Adam on the FP32 masters, then the bf16 inference copy
// Rounding points: inputs, W1, W2, w3, the layer-1 activations and the
// backward operands dPre2, dPre1 are bf16; everything else is FP32.
#include <cuda_bf16.h>
#include <math.h>

#include <string>
#include <vector>

#include "../../include/spectral_b200.h"
#include "sns_common.cuh"
#include "sns_ens.cuh"
#include "sns_les.cuh"
#include "sns_mlp.cuh"
#include "sns_tc.cuh"

namespace sns {

constexpr int kPart = kMlpParams + 1;  // gradients + loss sum

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
// oracle: hidden layer 1 rounded to BF16, layer 2 kept in FP32.
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
  uint64_t never;  // a barrier nothing arrives at (the stall test's wait)
  uint32_t tmem;
  int abort;
};

__device__ int g_mlp_tc_status;  // nonzero: a tensor-core wait ran out


// stall_cycles > 0 (a test of the timeout path, SNS_TC_STALL_TEST): after the
// first layer-1 MMA of its first tile each CTA also waits, for that many
// cycles, on a barrier that nothing arrives at; the wait runs out, the CTA
// records the timeout and stops after waiting (with the full budget) for the
// MMA it issued, so tensor memory is freed only once the MMA is complete.
__global__ void __launch_bounds__(kTcRows)
    k_mlp_infer_tc(const MlpPacked* __restrict__ P, const __nv_bfloat16* __restrict__ X,
                   int64_t M, float* __restrict__ nut, long long stall_cycles) {
  extern __shared__ __align__(128) unsigned char tc_raw[];
  TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
  const int tid = threadIdx.x, warp = tid >> 5;
  mlp_tc_load_weights(P, S.W1, S.W2, S.B2, S.w3, tid, kTcRows);
  mlp_tc_fill_ones(S.ONES, kTcRows, tid, kTcRows);
  if (tid == 0) {
    S.b3 = P->b3;
    S.s_out = P->s_out;
    S.abort = 0;
    tc::mbar_init(&S.mbar, 1);
    tc::mbar_init(&S.never, 1);
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
  // this thread's input row of a tile (zeros past the end)
  auto load_row = [&](int64_t tile, uint4& x0, uint4& x1) {
    const int64_t r = tile * kTcRows + tid;
    x0 = make_uint4(0, 0, 0, 0);
    x1 = x0;
    if (tile < tiles && r < M) {
      const uint4* src = reinterpret_cast<const uint4*>(X + r * kMlpK1);
      x0 = src[0];
      x1 = src[1];
    }
  };
  // the next tile's row is loaded while this tile's MMAs and epilogues run
  uint4 nx0, nx1;
  load_row(blockIdx.x, nx0, nx1);
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t row = tile * kTcRows + tid;
    {
      uint4 x0 = nx0, x1 = nx1;
      load_row(tile + gridDim.x, nx0, nx1);
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
    if (stall_cycles > 0 && tile == blockIdx.x && !tc::mbar_wait(&S.never, 0, stall_cycles))
      S.abort = 1;
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

// ---------------------------------------------------------------------------
// Training (loss and gradients) on tcgen05: a persistent CTA of 128 threads
// walks tiles of 128 samples (thread m owns sample m: its input row, its
// accumulator lanes and its scalar terms).  Per tile, five MMA groups:
//   M1  pre1 = X W1^T (+ b1 via the bias columns)       D cols   0..63
//   M2  pre2 = H1 W2^T + b2 (bias slice)                D cols  64..127
//   M3  dH1 = dPre2 W2 (W2 read MN-major)               D cols   0..63
//   M4  dW2 += dPre2^T H1 (M 64, both operands MN-major, K = the samples)
//                                                       D cols 128..191
//   M5  dW1 += dPre1^T X (M 64, N 16)                   D cols 192..207
// dW1 and dW2 accumulate in tensor memory over all the CTA's tiles (M = 64
// accumulators: row r in lane 32 (r / 16) + r % 16).  The vector gradients
// (db1, db2, dw3) are FP32 sums over samples, reduced across each warp by a
// shuffle reduce-scatter (lane l keeps columns 2l, 2l + 1) and across warps
// in a fixed order at the end; the scalars (db3, loss) likewise.  Rounding
// points as in the oracle: dPre2 and dPre1 enter the MMAs in BF16, the
// vector sums use their FP32 values.  The CTA writes one partial (kPart
// floats) for the deterministic reduce.
constexpr int kGtRows = 128;
constexpr int kGtCols = 256;  // tensor-memory columns

struct __align__(128) GradTcSmem {
  unsigned char W1[kMlpHidden * kMlpK1 * 2];
  unsigned char W2[kMlpHidden * kMlpHidden * 2];
  unsigned char B2[kMlpHidden * 16 * 2];
  unsigned char ONES[kGtRows * 16 * 2];
  unsigned char X[kGtRows * kMlpK1 * 2];
  unsigned char H1[kGtRows * kMlpHidden * 2];
  unsigned char P2[kGtRows * kMlpHidden * 2];  // dPre2 (bf16)
  unsigned char P1[kGtRows * kMlpHidden * 2];  // dPre1 (bf16)
  float w3[kMlpHidden];
  float vec[4][3][kMlpHidden];  // per warp: db1, db2, dw3
  float scal[4][2];             // per warp: db3, loss
  float b3;
  uint64_t mbar;
  uint32_t tmem;
  int abort;
};
// at most two CTAs per SM (2 x 256 tensor-memory columns): reserve enough
// shared memory that a third never shares the SM
constexpr int kGtSmemBytes = 80 * 1024;
static_assert(sizeof(GradTcSmem) <= kGtSmemBytes, "training tile fits the reservation");

// Sum of v[c] over the 32 lanes of the warp for c = 0..63; lane l returns the
// sums of columns 2l and 2l + 1.
__device__ __forceinline__ void warp_colsum64(float (&v)[64], float& c0, float& c1) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 16, n = 32; o >= 1; o >>= 1, n >>= 1) {
    const bool up = lane & o;
#pragma unroll
    for (int i = 0; i < 32; i++) {
      if (i < n) {
        const float send = up ? v[i] : v[n + i];
        const float keep = up ? v[n + i] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
      }
    }
  }
  c0 = v[0];
  c1 = v[1];
}

__device__ __forceinline__ bool tc_step(uint64_t* mbar, uint32_t& phase, int& abort_flag) {
  const bool ok = tc::mbar_wait(mbar, phase, tc::kWaitCycles);
  phase ^= 1;
  if (!ok) abort_flag = 1;
  tc::fence_after_sync();
  __syncthreads();
  return !abort_flag;
}

__global__ void __launch_bounds__(kGtRows)
    k_mlp_grad_tc(const MlpPacked* __restrict__ P, const __nv_bfloat16* __restrict__ X,
                  const float* __restrict__ target, const float* __restrict__ weight,
                  const int* __restrict__ idx, int64_t B, float inv_batch,
                  float* __restrict__ part) {
  extern __shared__ __align__(128) unsigned char gt_raw[];
  GradTcSmem& S = *reinterpret_cast<GradTcSmem*>(gt_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kMlpHidden * kMlpK1 / 8; i += kGtRows) {
    const int n = i / (kMlpK1 / 8), c = i % (kMlpK1 / 8);
    uint4 v = reinterpret_cast<const uint4*>(P->W1)[i];
    if (c == 1) {
      const float b = P->b1[n];
      const float hi = __bfloat162float(__float2bfloat16_rn(b));
      v.x = (v.x & 0xFFFFu) | (bf16_bits(hi) << 16);
      v.y = (v.y & 0xFFFF0000u) | bf16_bits(b - hi);
    }
    *reinterpret_cast<uint4*>(S.W1 + tc::kmajor_off(n, 8 * c, kMlpK1)) = v;
  }
  for (int i = tid; i < kMlpHidden * kMlpHidden / 8; i += kGtRows) {
    const int n = i / (kMlpHidden / 8), c = i % (kMlpHidden / 8);
    *reinterpret_cast<uint4*>(S.W2 + tc::kmajor_off(n, 8 * c, kMlpHidden)) =
        reinterpret_cast<const uint4*>(P->W2)[i];
  }
  for (int n = tid; n < kMlpHidden; n += kGtRows) {
    const float b = P->b2[n];
    const float hi = __bfloat162float(__float2bfloat16_rn(b));
    *reinterpret_cast<uint4*>(S.B2 + tc::kmajor_off(n, 0, 16)) =
        make_uint4(bf16_bits(hi) | (bf16_bits(b - hi) << 16), 0u, 0u, 0u);
    *reinterpret_cast<uint4*>(S.B2 + tc::kmajor_off(n, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
    S.w3[n] = __bfloat162float(P->w3[n]);
  }
  const uint32_t one = bf16_bits(1.f), one2 = one * 0x10001u;
  *reinterpret_cast<uint4*>(S.ONES + tc::kmajor_off(tid, 0, 16)) = make_uint4(one2 & 0xFFFFFFFFu, 0u, 0u, 0u);
  *reinterpret_cast<uint4*>(S.ONES + tc::kmajor_off(tid, 8, 16)) = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    S.b3 = P->b3;
    S.abort = 0;
    tc::mbar_init(&S.mbar, 1);
  }
  if (warp == 0) {
    tc::tmem_alloc(&S.tmem, kGtCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tmem;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
  const uint32_t sX = tc::smem_u32(S.X), sH = tc::smem_u32(S.H1), sP2 = tc::smem_u32(S.P2),
                 sP1 = tc::smem_u32(S.P1), sO = tc::smem_u32(S.ONES);
  const uint32_t sW1 = tc::smem_u32(S.W1), sW2 = tc::smem_u32(S.W2), sB2 = tc::smem_u32(S.B2);
  constexpr uint32_t id_fwd = tc::idesc_bf16(kGtRows, kMlpHidden);          // M1, M2
  constexpr uint32_t id_dh = tc::idesc_bf16(kGtRows, kMlpHidden, false, true);  // M3
  constexpr uint32_t id_dw2 = tc::idesc_bf16(64, kMlpHidden, true, true);   // M4
  constexpr uint32_t id_dw1 = tc::idesc_bf16(64, kMlpK1, true, true);       // M5
  uint32_t phase = 0;
  float acc_db1[2] = {0.f, 0.f}, acc_db2[2] = {0.f, 0.f}, acc_dw3[2] = {0.f, 0.f};
  float acc_db3 = 0.f, acc_loss = 0.f;
  bool first = true;
  const int64_t tiles = (B + kGtRows - 1) / kGtRows;
  // this thread's sample of a tile: input row, target and weight (zeros past
  // the end); the next tile's is loaded while this tile's MMAs run
  auto load_sample = [&](int64_t tile, uint4& x0, uint4& x1, float& tgt, float& wt) {
    const int64_t b = tile * kGtRows + tid;
    x0 = make_uint4(0, 0, 0, 0);
    x1 = x0;
    tgt = 0.f;
    wt = 0.f;
    if (tile < tiles && b < B) {
      const int64_t row = idx ? (int64_t)idx[b] : b;
      const uint4* src = reinterpret_cast<const uint4*>(X + row * kMlpK1);
      x0 = src[0];
      x1 = src[1];
      tgt = target[row];
      wt = weight ? weight[row] : 1.f;
    }
  };
  uint4 nx0, nx1;
  float ntgt, nwt;
  load_sample(blockIdx.x, nx0, nx1, ntgt, nwt);
  for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int64_t b = tile * kGtRows + tid;
    const bool valid = b < B;
    float tgt = ntgt, wt = nwt;
    {
      uint4 x0 = nx0, x1 = nx1;
      load_sample(tile + gridDim.x, nx0, nx1, ntgt, nwt);
      x1.x = (x1.x & 0xFFFFu) | (one2 & 0xFFFF0000u);
      x1.y = (x1.y & 0xFFFF0000u) | (one2 & 0xFFFFu);
      *reinterpret_cast<uint4*>(S.X + tc::kmajor_off(tid, 0, kMlpK1)) = x0;
      *reinterpret_cast<uint4*>(S.X + tc::kmajor_off(tid, 8, kMlpK1)) = x1;
    }
    // M1
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      tc::mma_bf16(tmem, tc::sdesc(sX, 128, 16 * kMlpK1), tc::sdesc(sW1, 128, 16 * kMlpK1), id_fwd,
                   0);
      tc::commit(&S.mbar);
    }
    if (!tc_step(&S.mbar, phase, S.abort)) break;
    // pre1 -> mask, H1
    uint32_t mask1[2] = {0u, 0u};
#pragma unroll
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + lane_base + c0, r);
      uint32_t h[8];
#pragma unroll
      for (int j = 0; j < 16; j++)
        if (__uint_as_float(r[j]) > 0.f) mask1[(c0 + j) >> 5] |= 1u << ((c0 + j) & 31);
#pragma unroll
      for (int j = 0; j < 8; j++)
        h[j] = pack_bf16(fmaxf(__uint_as_float(r[2 * j]), 0.f),
                         fmaxf(__uint_as_float(r[2 * j + 1]), 0.f));
      *reinterpret_cast<uint4*>(S.H1 + tc::kmajor_off(tid, c0, kMlpHidden)) =
          make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(S.H1 + tc::kmajor_off(tid, c0 + 8, kMlpHidden)) =
          make_uint4(h[4], h[5], h[6], h[7]);
    }
    // M2
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < kMlpHidden / 16; s++)
        tc::mma_bf16(tmem + 64, tc::sdesc(sH + 256 * s, 128, 16 * kMlpHidden),
                     tc::sdesc(sW2 + 256 * s, 128, 16 * kMlpHidden), id_fwd, s > 0);
      tc::mma_bf16(tmem + 64, tc::sdesc(sO, 128, 256), tc::sdesc(sB2, 128, 256), id_fwd, 1);
      tc::commit(&S.mbar);
    }
    if (!tc_step(&S.mbar, phase, S.abort)) break;
    // output, loss, dz; then dw3, dPre2 (-> P2), db2
    float dz;
    {
      float z = S.b3;
#pragma unroll
      for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
        uint32_t r[16];
        tc::tmem_ld16(tmem + lane_base + 64 + c0, r);
#pragma unroll
        for (int j = 0; j < 16; j++) z += fmaxf(__uint_as_float(r[j]), 0.f) * S.w3[c0 + j];
      }
      const float y = softplus_f(z);
      const float d = valid ? y - tgt : 0.f;
      acc_loss += wt * d * d;
      dz = 2.f * inv_batch * wt * d / (1.f + expf(-z));
    }
    float vw3[64], vb2[64];
#pragma unroll
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + lane_base + 64 + c0, r);
      uint32_t h[8];
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const float p2 = __uint_as_float(r[j]);
        vw3[c0 + j] = dz * fmaxf(p2, 0.f);
        vb2[c0 + j] = p2 > 0.f ? dz * S.w3[c0 + j] : 0.f;
      }
#pragma unroll
      for (int j = 0; j < 8; j++) h[j] = pack_bf16(vb2[c0 + 2 * j], vb2[c0 + 2 * j + 1]);
      *reinterpret_cast<uint4*>(S.P2 + tc::kmajor_off(tid, c0, kMlpHidden)) =
          make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(S.P2 + tc::kmajor_off(tid, c0 + 8, kMlpHidden)) =
          make_uint4(h[4], h[5], h[6], h[7]);
    }
    {
      float a0, a1;
      warp_colsum64(vw3, a0, a1);
      acc_dw3[0] += a0;
      acc_dw3[1] += a1;
      warp_colsum64(vb2, a0, a1);
      acc_db2[0] += a0;
      acc_db2[1] += a1;
    }
    {
      float d3 = dz;
#pragma unroll
      for (int o = 16; o >= 1; o >>= 1) d3 += __shfl_xor_sync(0xffffffffu, d3, o);
      acc_db3 += d3;
    }
    // M3 (dH1) and M4 (dW2 += dPre2^T H1)
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < kMlpHidden / 16; s++)
        tc::mma_bf16(tmem, tc::sdesc(sP2 + 256 * s, 128, 16 * kMlpHidden),
                     tc::sdesc(sW2 + 2048 * s, 16 * kMlpHidden, 128), id_dh, s > 0);
#pragma unroll
      for (int s = 0; s < kGtRows / 16; s++)
        tc::mma_bf16(tmem + 128, tc::sdesc(sP2 + 2048 * s, 16 * kMlpHidden, 128),
                     tc::sdesc(sH + 2048 * s, 16 * kMlpHidden, 128), id_dw2, (!first) || s > 0);
      tc::commit(&S.mbar);
    }
    if (!tc_step(&S.mbar, phase, S.abort)) break;
    // dPre1 = dH1 * (pre1 > 0) -> P1, db1
    {
      float vb1[64];
#pragma unroll
      for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
        uint32_t r[16];
        tc::tmem_ld16(tmem + lane_base + c0, r);
        uint32_t h[8];
#pragma unroll
        for (int j = 0; j < 16; j++)
          vb1[c0 + j] = ((mask1[(c0 + j) >> 5] >> ((c0 + j) & 31)) & 1u) ? __uint_as_float(r[j])
                                                                          : 0.f;
#pragma unroll
        for (int j = 0; j < 8; j++) h[j] = pack_bf16(vb1[c0 + 2 * j], vb1[c0 + 2 * j + 1]);
        *reinterpret_cast<uint4*>(S.P1 + tc::kmajor_off(tid, c0, kMlpHidden)) =
            make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(S.P1 + tc::kmajor_off(tid, c0 + 8, kMlpHidden)) =
            make_uint4(h[4], h[5], h[6], h[7]);
      }
      float a0, a1;
      warp_colsum64(vb1, a0, a1);
      acc_db1[0] += a0;
      acc_db1[1] += a1;
    }
    // M5 (dW1 += dPre1^T X)
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int s = 0; s < kGtRows / 16; s++)
        tc::mma_bf16(tmem + 192, tc::sdesc(sP1 + 2048 * s, 16 * kMlpHidden, 128),
                     tc::sdesc(sX + 512 * s, 16 * kMlpK1, 128), id_dw1, (!first) || s > 0);
      tc::commit(&S.mbar);
    }
    if (!tc_step(&S.mbar, phase, S.abort)) break;
    first = false;
    tc::fence_before_sync();
  }
  __syncthreads();
  float* out = part + (int64_t)blockIdx.x * kPart;
  if (S.abort) {
    tc::mbar_wait(&S.mbar, phase ^ 1, tc::kWaitCycles);
    if (tid == 0) atomicExch(&g_mlp_tc_status, 1);
  } else {
    // dW2 and dW1 from the M = 64 accumulators: lanes 32 w .. 32 w + 15 hold
    // rows 16 w .. 16 w + 15 (a CTA without tiles writes zeros)
    const int n = 16 * warp + lane;
#pragma unroll
    for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
      uint32_t r[16];
      tc::tmem_ld16(tmem + lane_base + 128 + c0, r);
      if (lane < 16)
#pragma unroll
        for (int j = 0; j < 16; j++)
          out[kMlpOffW2 + n * kMlpHidden + c0 + j] = first ? 0.f : __uint_as_float(r[j]);
    }
    {
      uint32_t r[16];
      tc::tmem_ld16(tmem + lane_base + 192, r);
      if (lane < 16)
#pragma unroll
        for (int j = 0; j < 16; j++)
          out[kMlpOffW1 + n * kMlpK1 + j] = (first || j >= kMlpIn) ? 0.f : __uint_as_float(r[j]);
    }
    S.vec[warp][0][2 * lane] = acc_db1[0];
    S.vec[warp][0][2 * lane + 1] = acc_db1[1];
    S.vec[warp][1][2 * lane] = acc_db2[0];
    S.vec[warp][1][2 * lane + 1] = acc_db2[1];
    S.vec[warp][2][2 * lane] = acc_dw3[0];
    S.vec[warp][2][2 * lane + 1] = acc_dw3[1];
    float l = acc_loss;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if (lane == 0) {
      S.scal[warp][0] = acc_db3;
      S.scal[warp][1] = l;
    }
  }
  __syncthreads();
  if (!S.abort) {
    for (int i = tid; i < kMlpHidden; i += kGtRows) {
      float a = 0.f, b2 = 0.f, c = 0.f;
      for (int w = 0; w < 4; w++) {
        a += S.vec[w][0][i];
        b2 += S.vec[w][1][i];
        c += S.vec[w][2][i];
      }
      out[kMlpOffB1 + i] = a;
      out[kMlpOffB2 + i] = b2;
      out[kMlpOffW3 + i] = c;
    }
    if (tid == 0) {
      float a = 0.f, l = 0.f;
      for (int w = 0; w < 4; w++) {
        a += S.scal[w][0];
        l += S.scal[w][1];
      }
      out[kMlpOffB3] = a;
      out[kMlpParams] = l;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kGtCols);
  }
}

namespace {

int grad_launch(const void* packed, const void* X, const float* t, const float* w,
                const int* idx, int64_t B, float* grad, cudaStream_t s) {
  if (reinterpret_cast<uintptr_t>(X) % 16 || reinterpret_cast<uintptr_t>(packed) % 16) {
    set_error("sns_mlp_grad: X and the packed model must be 16-byte aligned");
    return ERR_ARG;
  }
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    int rc = cuda_status(cudaFuncSetAttribute(k_mlp_grad_tc,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              kGtSmemBytes),
                         "cudaFuncSetAttribute(k_mlp_grad_tc)");
    if (rc) return rc;
    attr[dev & 63] = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t tiles = (B + kGtRows - 1) / kGtRows;
  const int nb = (int)std::min<int64_t>(tiles, 2 * (int64_t)sms);
  void* part = nullptr;
  int rc = pool_malloc(&part, sizeof(float) * kPart * nb);
  if (rc) return rc;
  const float inv = (float)(1.0 / (double)B);
  k_mlp_grad_tc<<<(unsigned)nb, kGtRows, kGtSmemBytes, s>>>(
      reinterpret_cast<const MlpPacked*>(packed), reinterpret_cast<const __nv_bfloat16*>(X), t, w,
      idx, B, inv, reinterpret_cast<float*>(part));
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_mlp_reduce<<<(kPart + 255) / 256, 256, 0, s>>>(reinterpret_cast<float*>(part), nb, inv,
                                                    grad);
    e = cudaGetLastError();
  }
  // the pool may hand the block to any later caller: wait for the kernels
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  pool_free(part);
  return cuda_status(e, "k_mlp_grad_tc");
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
  // SNS_TC_STALL_TEST=<cycles>: exercise the timeout path (see k_mlp_infer_tc)
  long long stall = 0;
  if (const char* e = getenv("SNS_TC_STALL_TEST")) stall = atoll(e);
  if (stall < 0 || stall > tc::kWaitCycles) stall = 0;
  k_mlp_infer_tc<<<blocks, kTcRows, sizeof(TcSmem), reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const MlpPacked*>(packed), reinterpret_cast<const __nv_bfloat16*>(X), M,
      nut, stall);
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
  int w = 0;
  int rc = les_tc_status_take(&w);
  if (rc) return rc;
  v |= w;
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
