// Batched ensemble of independent Navier-Stokes boxes of uneven size.
//
// Every box runs the fused step of exec/ns.cpp:167-217 (the five passes of
// sns_ns.cu), but one step of the whole ensemble is five launches, one per
// stage, each over a work list of (box, tile) items that spans every box.
// The tile shape of each box size is derived from one thread count per stage,
// so every item of a stage is one CTA's worth of equal work (each thread owns
// 16 elements of a line whatever the line length): items balance without a
// scheduler, and a persistent grid may stride over them.  The five launches
// are captured once in a CUDA graph and replayed per step.  A tuner times the
// candidate thread counts, line-run widths and grid modes of each stage on the
// ensemble itself and keeps the fastest.
//
// The tile bodies are the ones the single-box kernels run (sns_tiles.cuh), so
// a box advanced in the ensemble follows the single-box stepper's arithmetic;
// the two agree to rounding (the compiler may contract multiply-adds
// differently once the bodies are inlined into other kernels).
#include <math.h>
#include <stdlib.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "../../include/spectral_b200.h"
#include "sns_ens.cuh"
#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_ns.cuh"
#include "sns_ops.cuh"
#include "sns_tiles.cuh"

namespace sns {

constexpr int kEnsStages = 5;
constexpr int kEnsMaxClasses = 8;
constexpr int kEnsMinLine = 16, kEnsMaxLine = 256;

// Device-resident description of one box (the table is ordered by class).
struct EnsBox {
  void* V[3];
  void* C0[3];
  void* U[6];
  double* stats;  // per-tile diagnostics of the update stage
  double hK, nuhK;
};

// Device-resident description of one box size within one stage.
struct EnsClass {
  LineGeo geo;  // line stages: the pass geometry; all stages: nx, ny, nz
  int L;        // line length of the stage
  int W, G, wshift, lx;
  int64_t tiles;  // items per box
  int box0;       // first box of the class in the box table
  int nf;         // fields of a line stage
  double scale2;  // 1/N^2 of the cross product
  const void* tw;
  int pf_self;    // update stage: ask L2 for a tile's V and C0 once its cross
                  // product's loads are in flight
};

// Kernel parameter of one stage launch.
struct EnsStage {
  const EnsClass* cls;
  const EnsBox* boxes;
  int nclass;
  int64_t total;                  // items
  int64_t first[kEnsMaxClasses];  // first item of each class
};

struct BoxCurlFields {  // K1: V in, U out
  const EnsBox* __restrict__ b;
  __device__ __forceinline__ const void* in(int i) const { return i < 3 ? b->V[i] : nullptr; }
  __device__ __forceinline__ void* out(int i) const { return b->U[i]; }
};
struct BoxWorkFields {  // K2, K3, K4: in place on U
  const EnsBox* __restrict__ b;
  __device__ __forceinline__ const void* in(int i) const { return b->U[i]; }
  __device__ __forceinline__ void* out(int i) const { return b->U[i]; }
};

template <typename T, int L, int STAGE>
__device__ __forceinline__ void ens_item(const EnsClass* __restrict__ k,
                                         const EnsBox* __restrict__ box, int64_t blk,
                                         cx_t<T>* sm, double (*red)[32]) {
  using C = cx_t<T>;
  const C* tw = reinterpret_cast<const C*>(k->tw);
  if constexpr (STAGE == 0) {  // K1: z-inverse of (V, i k x V)
    const LineGeo geo = k->geo;
    line_pass_tile<T, L, PRO_CURL6>(geo, BoxCurlFields{box}, 6, tw, (T)1, (T)1, 0, k->wshift,
                                    blk, sm);
  } else if constexpr (STAGE == 1) {  // K2: y-inverse of the six fields
    const LineGeo geo = k->geo;
    line_pass_tile<T, L, PRO_LOAD>(geo, BoxWorkFields{box}, 6, tw, (T)1, (T)1, 0, k->wshift, blk,
                                   sm);
  } else if constexpr (STAGE == 2) {  // K3: x-inverse, cross product, x-forward
    xcross_tile<T, L>(BoxWorkFields{box}, tw, k->G, (T)k->scale2, blk, (int)blockDim.x, sm);
  } else if constexpr (STAGE == 3) {  // K4: y-forward of the product
    const LineGeo geo = k->geo;
    line_pass_tile<T, L, PRO_LOAD>(geo, BoxWorkFields{box}, 3, tw, (T)-1, (T)1, 0, k->wshift,
                                   blk, sm);
  } else {  // K5: z-forward + update
    // the arguments live in shared memory, read where used, which keeps the
    // nine field pointers out of the registers of the update loop
    __shared__ UpdateArgs a;
    if (threadIdx.x == 0) {
      for (int d = 0; d < 3; d++) {
        a.U[d] = box->U[d];
        a.V[d] = box->V[d];
        a.C0[d] = box->C0[d];
      }
      a.nx = k->geo.nx;
      a.ny = k->geo.ny;
      a.nz = k->geo.nz;
      a.lx = k->lx;
      a.W = k->W;
      a.hK = box->hK;
      a.nuhK = box->nuhK;
      a.stats = box->stats;
      a.kc2 = 1e300;
      a.kx_half = 0;
      a.pf = 0;
      a.pf_self = k->pf_self;
      for (int i = 0; i < 6; i++) a.Uo[i] = nullptr;
    }
    __syncthreads();
    zfwd_update_tile<T, L>(a, tw, blk, (int)blockDim.x, sm, red);
  }
}

// One stage over every box.  Item i of the work list is tile i - first[c] of
// class c's boxes (box-major); the grid either has one CTA per item or
// strides over them.
template <typename T, int STAGE>
__global__ void __launch_bounds__(MaxThreads<T>::value) k_ens_stage(const EnsStage st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4][32];
  cx_t<T>* sm = reinterpret_cast<cx_t<T>*>(smem_raw);
  for (int64_t item = blockIdx.x; item < st.total; item += gridDim.x) {
    if (item != (int64_t)blockIdx.x) __syncthreads();  // the previous item's shared memory
    // class lookup with constant indices, so the table stays in parameter space
    int c = 0;
    int64_t first = 0;
#pragma unroll
    for (int i = 1; i < kEnsMaxClasses; i++)
      if (i < st.nclass && item >= st.first[i]) {
        c = i;
        first = st.first[i];
      }
    const EnsClass* __restrict__ k = st.cls + c;
    const int64_t local = item - first;
    const int64_t tiles = k->tiles;
    const int64_t b = local / tiles;
    const EnsBox* __restrict__ box = st.boxes + k->box0 + b;
    const int64_t blk = local - b * tiles;
    switch (k->L) {
      case 16: ens_item<T, 16, STAGE>(k, box, blk, sm, red); break;
      case 32: ens_item<T, 32, STAGE>(k, box, blk, sm, red); break;
      case 64: ens_item<T, 64, STAGE>(k, box, blk, sm, red); break;
      case 128: ens_item<T, 128, STAGE>(k, box, blk, sm, red); break;
      default: ens_item<T, 256, STAGE>(k, box, blk, sm, red); break;
    }
  }
}

// Per-box diagnostics: one CTA per box reduces its tiles' partials.
__global__ void k_ens_stats(const EnsBox* __restrict__ boxes, const int64_t* __restrict__ parts,
                            double* __restrict__ out) {
  __shared__ double sm[4][256];
  const double* p = boxes[blockIdx.x].stats;
  const int64_t n = parts[blockIdx.x];
  double a = 0, b = 0, c = 0, m = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    a += p[4 * i];
    b += p[4 * i + 1];
    c += p[4 * i + 2];
    m = fmax(m, p[4 * i + 3]);
  }
  sm[0][threadIdx.x] = a;
  sm[1][threadIdx.x] = b;
  sm[2][threadIdx.x] = c;
  sm[3][threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sm[0][threadIdx.x] += sm[0][threadIdx.x + o];
      sm[1][threadIdx.x] += sm[1][threadIdx.x + o];
      sm[2][threadIdx.x] += sm[2][threadIdx.x + o];
      sm[3][threadIdx.x] = fmax(sm[3][threadIdx.x], sm[3][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; q++) out[4 * blockIdx.x + q] = sm[q][0];
}

// ---------------------------------------------------------------------------
// host side

namespace {

int log2i(int64_t n) {
  int l = 0;
  while (((int64_t)1 << l) < n) l++;
  return l;
}
int tpl_of(int L) { return L / (L >= 16 ? 16 : L); }
size_t esize_of(int prec) { return prec == PREC_C128 ? 16 : 8; }

// Tuning choice of one stage.
struct StageCfg {
  int threads;     // CTA size
  int wcap;        // line stages: cap on adjacent lines per tile
  int persistent;  // 1: grid of resident CTAs striding over the items
};

struct BoxHost {
  int64_t nx, ny, nz;
  double nu;
  int cls;  // class index
  void* V[3];
  void* C0[3];
  void* U[6];
  double* stats;
};

struct ClassHost {
  int64_t nx, ny, nz;
  int nboxes, box0;
  NSPlan seq;  // the single-box plan of the sequential mode
};

template <typename T, int S>
cudaError_t set_attr() {
  return allow_max_dynamic_smem(k_ens_stage<T, S>);
}

template <typename T>
const void* stage_kernel(int s) {
  switch (s) {
    case 0: return (const void*)k_ens_stage<T, 0>;
    case 1: return (const void*)k_ens_stage<T, 1>;
    case 2: return (const void*)k_ens_stage<T, 2>;
    case 3: return (const void*)k_ens_stage<T, 3>;
    default: return (const void*)k_ens_stage<T, 4>;
  }
}

}  // namespace

}  // namespace sns

using namespace sns;

struct sns_ens {
  int prec = 0;
  double dt = 0;
  cudaStream_t s = nullptr;        // the caller's stream
  cudaStream_t cap = nullptr;      // private stream for graph capture
  std::vector<BoxHost> boxes;      // table order (grouped by class)
  std::vector<int> user_to_table;  // box index of the caller -> table index
  std::vector<ClassHost> classes;
  EnsBox* d_boxes = nullptr;
  EnsClass* d_cls = nullptr;  // kEnsStages x nclass
  int64_t* d_parts_ens = nullptr;
  int64_t* d_parts_seq = nullptr;
  double* d_stats = nullptr;  // 4 per box
  StageCfg cfg[kEnsStages];
  EnsStage st[kEnsStages];
  int grid[kEnsStages];
  size_t smem[kEnsStages];
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int last_mode = -1;  // mode of the last step (selects the partial counts)
  bool stepped = false;
};

namespace sns {
namespace {

int nclass(const sns_ens* e) { return (int)e->classes.size(); }

// Tile of class c in stage s under cfg; false if the configuration cannot
// tile the class.
bool make_class(const sns_ens* e, int s, int c, const StageCfg& cfg, EnsClass& k, size_t& smem) {
  const ClassHost& ch = e->classes[c];
  const int nx = (int)ch.nx, ny = (int)ch.ny, nz = (int)ch.nz;
  const size_t esz = esize_of(e->prec);
  const int T = cfg.threads;
  k = EnsClass{};
  k.geo.nx = nx;
  k.geo.ny = ny;
  k.geo.nz = nz;
  k.box0 = ch.box0;
  k.lx = log2i(nx);
  const double N = (double)nx * ny * nz;
  k.scale2 = 1.0 / (N * N);
  if (s == 0 || s == 1 || s == 3) {
    const int axis = s == 0 ? 2 : 1;
    const int L = axis == 2 ? nz : ny;
    const int tpl = tpl_of(L);
    if (T % tpl) return false;
    const int lines = T / tpl;
    int W = std::min(std::min(cfg.wcap, nx), lines);
    const int G = lines / W;
    const int groups = axis == 2 ? ny : nz;
    if (W * G != lines || G > groups || groups % G) return false;
    LineGeo& g = k.geo;
    g.L = L;
    g.W = W;
    g.G = G;
    g.axis = axis;
    const int64_t nxy = (int64_t)nx * ny;
    if (axis == 2) {
      g.ps = nxy;
      g.gs = nx;
      g.TA = nx / W;
      g.TB = ny / G;
      g.sa = W;
      g.sb = (int64_t)G * nx;
    } else {
      g.ps = nx;
      g.gs = nxy;
      g.TA = nx / W;
      g.TB = nz / G;
      g.sa = W;
      g.sb = (int64_t)G * nxy;
    }
    k.L = L;
    k.W = W;
    k.G = G;
    k.wshift = log2i(W);
    k.nf = s == 3 ? 3 : 6;
    k.tiles = g.TA * g.TB * k.nf;
    smem = (size_t)lines * tile_stride(L, W, (int)esz) * esz;
  } else if (s == 2) {
    const int tpl = tpl_of(nx);
    if (T % (6 * tpl)) return false;
    const int G = T / (6 * tpl);
    const int64_t rows = (int64_t)ny * nz;
    if (G > rows || rows % G) return false;
    k.L = nx;
    k.G = G;
    k.tiles = rows / G;
    smem = (size_t)6 * G * xrow_stride(nx, (int)esz) * esz;
  } else {
    const int tpl = tpl_of(nz);
    if (T % (3 * tpl)) return false;
    const int W = T / (3 * tpl);
    const int64_t cols = (int64_t)nx * ny;
    if ((W & (W - 1)) || W > cols || cols % W) return false;
    k.L = nz;
    k.W = W;
    k.tiles = cols / W;
    // the update stage's L2 prefetch of V and C0 (SNS_ENS_PFSELF=0: off).
    // Measured on B200 for 32 x 32^3 + 24 x 64^3 + 8 x 128^3 boxes: update
    // stage 0.646 against 0.675 ms
    const char* pe = getenv("SNS_ENS_PFSELF");
    k.pf_self = pe ? (pe[0] == '1') : 1;
    smem = (size_t)3 * W * tile_stride(nz, W, (int)esz) * esz;
  }
  k.tw = twiddles(k.L, e->prec);
  return k.tw != nullptr && smem <= 200 * 1024;
}

// Fill stage s from cfg (host descriptors copied to d_cls).  ERR_UNSUPPORTED
// when cfg cannot tile every class.
int build_stage(sns_ens* e, int s, const StageCfg& cfg) {
  const int nc = nclass(e);
  std::vector<EnsClass> ks(nc);
  EnsStage st{};
  st.cls = e->d_cls + (size_t)s * nc;
  st.boxes = e->d_boxes;
  st.nclass = nc;
  size_t smem = 0;
  int64_t total = 0;
  for (int c = 0; c < nc; c++) {
    size_t sc = 0;
    if (!make_class(e, s, c, cfg, ks[c], sc)) return ERR_UNSUPPORTED;
    smem = std::max(smem, sc);
    st.first[c] = total;
    total += ks[c].tiles * e->classes[c].nboxes;
  }
  for (int c = nc; c < kEnsMaxClasses; c++) st.first[c] = total;
  st.total = total;
  if (total > 0x7fffffff) {
    set_error("sns_ens: work list too long");
    return ERR_UNSUPPORTED;
  }
  int rc = cuda_status(cudaMemcpyAsync(e->d_cls + (size_t)s * nc, ks.data(),
                                       sizeof(EnsClass) * nc, cudaMemcpyHostToDevice, e->s),
                       "sns_ens(stage table)");
  if (rc) return rc;
  // keep the host vector alive until the copy has read it
  if ((rc = cuda_status(cudaStreamSynchronize(e->s), "sns_ens(stage table)"))) return rc;
  int grid = (int)total;
  if (cfg.persistent) {
    const void* kern = e->prec == PREC_C128 ? stage_kernel<double>(s) : stage_kernel<float>(s);
    int per_sm = 0;
    if ((rc = cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern,
                                                                        cfg.threads, smem),
                          "sns_ens(occupancy)")))
      return rc;
    if (per_sm < 1) return ERR_UNSUPPORTED;
    grid = (int)std::min<int64_t>(total, (int64_t)per_sm * sm_count());
  }
  e->cfg[s] = cfg;
  e->st[s] = st;
  e->grid[s] = grid;
  e->smem[s] = smem;
  return OK;
}

int launch_stage(const sns_ens* e, int s, cudaStream_t stream) {
  const EnsStage& st = e->st[s];
  const dim3 grid(e->grid[s]), block(e->cfg[s].threads);
  const size_t smem = e->smem[s];
  if (e->prec == PREC_C128) {
    switch (s) {
      case 0: k_ens_stage<double, 0><<<grid, block, smem, stream>>>(st); break;
      case 1: k_ens_stage<double, 1><<<grid, block, smem, stream>>>(st); break;
      case 2: k_ens_stage<double, 2><<<grid, block, smem, stream>>>(st); break;
      case 3: k_ens_stage<double, 3><<<grid, block, smem, stream>>>(st); break;
      default: k_ens_stage<double, 4><<<grid, block, smem, stream>>>(st); break;
    }
  } else {
    switch (s) {
      case 0: k_ens_stage<float, 0><<<grid, block, smem, stream>>>(st); break;
      case 1: k_ens_stage<float, 1><<<grid, block, smem, stream>>>(st); break;
      case 2: k_ens_stage<float, 2><<<grid, block, smem, stream>>>(st); break;
      case 3: k_ens_stage<float, 3><<<grid, block, smem, stream>>>(st); break;
      default: k_ens_stage<float, 4><<<grid, block, smem, stream>>>(st); break;
    }
  }
  SNS_CHECK_LAUNCH("k_ens_stage");
  return OK;
}

int launch_step(const sns_ens* e, cudaStream_t stream) {
  for (int s = 0; s < kEnsStages; s++) {
    int rc = launch_stage(e, s, stream);
    if (rc) return rc;
  }
  return OK;
}

// Candidate configurations of stage s, defaults first.
std::vector<StageCfg> candidates(int s, int prec) {
  const int tmax = prec == PREC_C128 ? 512 : 768;
  std::vector<int> ts;
  if (s == 2)
    ts = {384, 192, 768};
  else if (s == 4)
    ts = prec == PREC_C128 ? std::vector<int>{192, 96, 384} : std::vector<int>{384, 192, 96, 768};
  else
    ts = {256, 128, 512};
  std::vector<int> ws = {1};
  if (s == 0 || s == 1 || s == 3)
    ws = prec == PREC_C128 ? std::vector<int>{8, 4, 16} : std::vector<int>{16, 8, 4};
  std::vector<StageCfg> out;
  for (int p = 0; p < 2; p++)
    for (int t : ts)
      if (t <= tmax)
        for (int w : ws) out.push_back(StageCfg{t, w, p});
  return out;
}

// Time `reps` launches of stage s (ms per launch).
int time_stage(sns_ens* e, int s, int reps, float* ms) {
  cudaEvent_t a, b;
  int rc = cuda_status(cudaEventCreate(&a), "sns_ens(tune)");
  if (rc) return rc;
  if ((rc = cuda_status(cudaEventCreate(&b), "sns_ens(tune)"))) {
    cudaEventDestroy(a);
    return rc;
  }
  rc = launch_stage(e, s, e->s);  // warm-up
  if (!rc) rc = cuda_status(cudaEventRecord(a, e->s), "sns_ens(tune)");
  for (int r = 0; r < reps && !rc; r++) rc = launch_stage(e, s, e->s);
  if (!rc) rc = cuda_status(cudaEventRecord(b, e->s), "sns_ens(tune)");
  if (!rc) rc = cuda_status(cudaEventSynchronize(b), "sns_ens(tune)");
  float t = 0;
  if (!rc) rc = cuda_status(cudaEventElapsedTime(&t, a, b), "sns_ens(tune)");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t / reps;
  return rc;
}

// Configure every stage: the first valid candidate, or the fastest when tuning.
int configure(sns_ens* e, bool tune) {
  for (int s = 0; s < kEnsStages; s++) {
    StageCfg best{};
    float best_ms = 1e30f;
    bool found = false;
    for (const StageCfg& cfg : candidates(s, e->prec)) {
      int rc = build_stage(e, s, cfg);
      if (rc == ERR_UNSUPPORTED) continue;
      if (rc) return rc;
      if (!tune) {
        best = cfg;
        found = true;
        break;
      }
      float ms = 0;
      if ((rc = time_stage(e, s, 4, &ms))) return rc;
      if (ms < best_ms) {
        best_ms = ms;
        best = cfg;
        found = true;
      }
    }
    if (!found) {
      set_error("sns_ens: no tile configuration fits every box of stage " + std::to_string(s));
      return ERR_UNSUPPORTED;
    }
    int rc = build_stage(e, s, best);
    if (rc) return rc;
  }
  return OK;
}

void release(sns_ens* e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  for (BoxHost& b : e->boxes) {
    for (int d = 0; d < 3; d++) {
      pool_free(b.V[d]);
      pool_free(b.C0[d]);
    }
    for (int i = 0; i < 6; i++) pool_free(b.U[i]);
    pool_free(b.stats);
  }
  pool_free(e->d_boxes);
  pool_free(e->d_cls);
  pool_free(e->d_parts_ens);
  pool_free(e->d_parts_seq);
  pool_free(e->d_stats);
  if (e->cap) cudaStreamDestroy(e->cap);
}

bool box_ok(const sns_ens* e, int box, const char* what) {
  if (!e) {
    set_error(std::string(what) + ": null ensemble");
    return false;
  }
  if (box < 0 || box >= (int)e->user_to_table.size()) {
    set_error(std::string(what) + ": box index out of range");
    return false;
  }
  return true;
}

bool vec3(const void* const v[3], const char* what) {
  if (!v || !v[0] || !v[1] || !v[2]) {
    set_error(std::string(what) + ": null field pointer");
    return false;
  }
  return true;
}

}  // namespace
}  // namespace sns

extern "C" {

int sns_ens_create(sns_ens** handle, int nboxes, const int64_t* dims, const double* nu, double dt,
                   int prec, int tune, void* stream) {
  if (!handle) {
    set_error("sns_ens_create: null output pointer");
    return ERR_ARG;
  }
  *handle = nullptr;
  if (nboxes < 1 || !dims || !nu) {
    set_error("sns_ens_create: need at least one box with dimensions and viscosity");
    return ERR_ARG;
  }
  if (prec != PREC_C64 && prec != PREC_C128) {
    set_error("precision must be SNS_C64 (0) or SNS_C128 (1)");
    return ERR_ARG;
  }
  // group the boxes by size, larger boxes first
  std::map<std::tuple<int64_t, int64_t, int64_t>, std::vector<int>> by_size;
  for (int i = 0; i < nboxes; i++) {
    const int64_t nx = dims[3 * i], ny = dims[3 * i + 1], nz = dims[3 * i + 2];
    for (int64_t n : {nx, ny, nz})
      if (!is_pow2(n) || n < kEnsMinLine || n > kEnsMaxLine) {
        set_error("sns_ens_create: box dimensions must be powers of two in [16, 256]");
        return ERR_UNSUPPORTED;
      }
    by_size[std::make_tuple(nx, ny, nz)].push_back(i);
  }
  if ((int)by_size.size() > kEnsMaxClasses) {
    set_error("sns_ens_create: at most 8 distinct box sizes");
    return ERR_UNSUPPORTED;
  }
  sns_ens* e = new sns_ens();
  e->prec = prec;
  e->dt = dt;
  e->s = reinterpret_cast<cudaStream_t>(stream);
  e->user_to_table.assign(nboxes, 0);
  int rc = OK;
  for (auto it = by_size.rbegin(); it != by_size.rend(); ++it) {
    ClassHost ch{};
    ch.nx = std::get<0>(it->first);
    ch.ny = std::get<1>(it->first);
    ch.nz = std::get<2>(it->first);
    ch.box0 = (int)e->boxes.size();
    ch.nboxes = (int)it->second.size();
    if (!rc) rc = ns_plan(ch.seq, (int)ch.nx, (int)ch.ny, (int)ch.nz, prec);
    ch.seq.use_xy = false;
    ch.seq.use_xyc = false;
    ch.seq.k1_lines = false;
    ch.seq.k1_tma = false;
    ch.seq.x_tma = false;
    ch.seq.z_tma = false;
    ch.seq.xy_chunk = 0;
    ch.seq.passes = kNSPasses;
    for (int user : it->second) {
      BoxHost b{};
      b.nx = ch.nx;
      b.ny = ch.ny;
      b.nz = ch.nz;
      b.nu = nu[user];
      b.cls = (int)e->classes.size();
      e->user_to_table[user] = (int)e->boxes.size();
      e->boxes.push_back(b);
    }
    e->classes.push_back(ch);
  }
  // fields: V, C0, U per box, zeroed; per-tile diagnostics
  const size_t esz = esize_of(prec);
  for (BoxHost& b : e->boxes) {
    const size_t bytes = esz * (size_t)b.nx * b.ny * b.nz;
    void** all[12];
    for (int d = 0; d < 3; d++) {
      all[d] = &b.V[d];
      all[3 + d] = &b.C0[d];
    }
    for (int i = 0; i < 6; i++) all[6 + i] = &b.U[i];
    for (int i = 0; i < 12 && !rc; i++) {
      rc = pool_malloc(all[i], bytes);
      if (!rc) rc = cuda_status(cudaMemsetAsync(*all[i], 0, bytes, e->s), "sns_ens_create");
    }
    // at most one tile per xy column in either mode
    if (!rc) rc = pool_malloc((void**)&b.stats, sizeof(double) * 4 * (size_t)b.nx * b.ny);
  }
  const int nb = (int)e->boxes.size(), nc = (int)e->classes.size();
  if (!rc) rc = pool_malloc((void**)&e->d_boxes, sizeof(EnsBox) * nb);
  if (!rc) rc = pool_malloc((void**)&e->d_cls, sizeof(EnsClass) * kEnsStages * nc);
  if (!rc) rc = pool_malloc((void**)&e->d_parts_ens, sizeof(int64_t) * nb);
  if (!rc) rc = pool_malloc((void**)&e->d_parts_seq, sizeof(int64_t) * nb);
  if (!rc) rc = pool_malloc((void**)&e->d_stats, sizeof(double) * 4 * nb);
  std::vector<EnsBox> hb(nb);
  std::vector<int64_t> seq_parts(nb);
  for (int i = 0; i < nb && !rc; i++) {
    const BoxHost& b = e->boxes[i];
    for (int d = 0; d < 3; d++) {
      hb[i].V[d] = b.V[d];
      hb[i].C0[d] = b.C0[d];
    }
    for (int q = 0; q < 6; q++) hb[i].U[q] = b.U[q];
    hb[i].stats = b.stats;
    hb[i].hK = dt / 2;
    hb[i].nuhK = b.nu * dt / 2;
    seq_parts[i] = e->classes[b.cls].seq.update_blocks;
  }
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(e->d_boxes, hb.data(), sizeof(EnsBox) * nb,
                                     cudaMemcpyHostToDevice, e->s),
                     "sns_ens_create");
  if (!rc)
    rc = cuda_status(cudaMemcpyAsync(e->d_parts_seq, seq_parts.data(), sizeof(int64_t) * nb,
                                     cudaMemcpyHostToDevice, e->s),
                     "sns_ens_create");
  if (!rc) rc = cuda_status(cudaStreamSynchronize(e->s), "sns_ens_create");
  // kernels may use the device's full shared memory
  for (int s = 0; s < kEnsStages && !rc; s++) {
    cudaError_t ce;
    if (prec == PREC_C128) {
      const cudaError_t r[5] = {set_attr<double, 0>(), set_attr<double, 1>(), set_attr<double, 2>(),
                                set_attr<double, 3>(), set_attr<double, 4>()};
      ce = r[s];
    } else {
      const cudaError_t r[5] = {set_attr<float, 0>(), set_attr<float, 1>(), set_attr<float, 2>(),
                                set_attr<float, 3>(), set_attr<float, 4>()};
      ce = r[s];
    }
    rc = cuda_status(ce, "cudaFuncSetAttribute(k_ens_stage)");
  }
  if (!rc) rc = configure(e, tune != 0);
  if (!rc) {
    // partials of the update stage per box = tiles of its class
    std::vector<int64_t> ens_parts(nb);
    for (int c = 0; c < nc; c++) {
      EnsClass k{};
      size_t sm = 0;
      make_class(e, 4, c, e->cfg[4], k, sm);
      for (int i = 0; i < e->classes[c].nboxes; i++) ens_parts[e->classes[c].box0 + i] = k.tiles;
    }
    rc = cuda_status(cudaMemcpyAsync(e->d_parts_ens, ens_parts.data(), sizeof(int64_t) * nb,
                                     cudaMemcpyHostToDevice, e->s),
                     "sns_ens_create");
    if (!rc) rc = cuda_status(cudaStreamSynchronize(e->s), "sns_ens_create");
  }
  if (!rc)
    rc = cuda_status(cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking), "sns_ens_create");
  if (rc) {
    release(e);
    delete e;
    return rc;
  }
  *handle = e;
  return OK;
}

int sns_ens_destroy(sns_ens* e) {
  if (!e) return OK;
  cudaStreamSynchronize(e->s);
  release(e);
  delete e;
  return OK;
}

int sns_ens_boxes(sns_ens* e) { return e ? (int)e->boxes.size() : ERR_ARG; }

int sns_ens_bootstrap(sns_ens* e, int box, const void* const V0[3], const void* const omega0[3]) {
  if (!box_ok(e, box, "sns_ens_bootstrap") || !vec3(V0, "sns_ens_bootstrap") ||
      !vec3(omega0, "sns_ens_bootstrap"))
    return ERR_ARG;
  BoxHost& b = e->boxes[e->user_to_table[box]];
  const Dims d{(int)b.nx, (int)b.ny, (int)b.nz};
  int rc = ns_bootstrap_fields(d, e->prec, b.nu, e->dt, V0, omega0, b.V, b.C0, b.U, e->s);
  if (rc) return rc;
  e->stepped = false;
  return OK;
}

int sns_ens_set_state(sns_ens* e, int box, const void* const V1[3], const void* const cross0[3]) {
  if (!box_ok(e, box, "sns_ens_set_state") || !vec3(V1, "sns_ens_set_state") ||
      !vec3(cross0, "sns_ens_set_state"))
    return ERR_ARG;
  BoxHost& b = e->boxes[e->user_to_table[box]];
  const size_t bytes = esize_of(e->prec) * (size_t)b.nx * b.ny * b.nz;
  for (int d = 0; d < 3; d++) {
    int rc = cuda_status(cudaMemcpyAsync(b.V[d], V1[d], bytes, cudaMemcpyDeviceToDevice, e->s),
                         "sns_ens_set_state");
    if (!rc)
      rc = cuda_status(cudaMemcpyAsync(b.C0[d], cross0[d], bytes, cudaMemcpyDeviceToDevice, e->s),
                       "sns_ens_set_state");
    if (rc) return rc;
  }
  e->stepped = false;
  return OK;
}

int sns_ens_get_state(sns_ens* e, int box, void* const V1[3], void* const omega1[3],
                      void* const cross0[3]) {
  if (!box_ok(e, box, "sns_ens_get_state")) return ERR_ARG;
  BoxHost& b = e->boxes[e->user_to_table[box]];
  const Dims d{(int)b.nx, (int)b.ny, (int)b.nz};
  const size_t bytes = esize_of(e->prec) * (size_t)d.n();
  int rc;
  for (int i = 0; i < 3; i++) {
    if (V1 && V1[i] &&
        (rc = cuda_status(cudaMemcpyAsync(V1[i], b.V[i], bytes, cudaMemcpyDeviceToDevice, e->s),
                          "sns_ens_get_state")))
      return rc;
    if (cross0 && cross0[i] &&
        (rc = cuda_status(cudaMemcpyAsync(cross0[i], b.C0[i], bytes, cudaMemcpyDeviceToDevice,
                                          e->s),
                          "sns_ens_get_state")))
      return rc;
  }
  if (omega1) {
    if (!vec3((const void* const*)omega1, "sns_ens_get_state")) return ERR_ARG;
    const void* v[3] = {b.V[0], b.V[1], b.V[2]};
    if ((rc = op_curl(v, omega1, d, e->prec, e->s))) return rc;
  }
  return OK;
}

int sns_ens_step(sns_ens* e, int nsteps, int mode) {
  if (!e) {
    set_error("sns_ens_step: null ensemble");
    return ERR_ARG;
  }
  if (nsteps < 0 || mode < SNS_ENS_GRAPH || mode > SNS_ENS_SEQUENTIAL) {
    set_error("sns_ens_step: bad step count or mode");
    return ERR_ARG;
  }
  int rc = OK;
  if (mode == SNS_ENS_GRAPH && nsteps > 0 && !e->exec) {
    // capture one ensemble step on the private stream, replayed on the caller's
    if ((rc = cuda_status(cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal),
                          "sns_ens_step(capture)")))
      return rc;
    const int lrc = launch_step(e, e->cap);
    cudaGraph_t g = nullptr;
    rc = cuda_status(cudaStreamEndCapture(e->cap, &g), "sns_ens_step(capture)");
    if (lrc || rc) {
      if (g) cudaGraphDestroy(g);
      return lrc ? lrc : rc;
    }
    if ((rc = cuda_status(cudaGraphInstantiate(&e->exec, g, 0), "sns_ens_step(instantiate)"))) {
      cudaGraphDestroy(g);
      e->exec = nullptr;
      return rc;
    }
    e->graph = g;
  }
  for (int t = 0; t < nsteps; t++) {
    if (mode == SNS_ENS_GRAPH) {
      rc = cuda_status(cudaGraphLaunch(e->exec, e->s), "sns_ens_step(graph)");
    } else if (mode == SNS_ENS_EAGER) {
      rc = launch_step(e, e->s);
    } else {
      for (const BoxHost& b : e->boxes) {
        void* V[3] = {b.V[0], b.V[1], b.V[2]};
        void* C0[3] = {b.C0[0], b.C0[1], b.C0[2]};
        void* U[6] = {b.U[0], b.U[1], b.U[2], b.U[3], b.U[4], b.U[5]};
        rc = ns_step_once(e->classes[b.cls].seq, V, C0, U, b.stats, nullptr, b.nu, e->dt, e->s);
        if (rc) break;
      }
    }
    if (rc) return rc;
    e->stepped = true;
    e->last_mode = mode;
  }
  return OK;
}

int sns_ens_stats(sns_ens* e, double* out) {
  if (!e || !out) {
    set_error("sns_ens_stats: null argument");
    return ERR_ARG;
  }
  if (!e->stepped) {
    set_error("sns_ens_stats: no step has run since the state was set");
    return ERR_ARG;
  }
  const int nb = (int)e->boxes.size();
  const int64_t* parts = e->last_mode == SNS_ENS_SEQUENTIAL ? e->d_parts_seq : e->d_parts_ens;
  k_ens_stats<<<nb, 256, 0, e->s>>>(e->d_boxes, parts, e->d_stats);
  SNS_CHECK_LAUNCH("k_ens_stats");
  std::vector<double> v(4 * (size_t)nb);
  int rc = cuda_status(cudaMemcpyAsync(v.data(), e->d_stats, sizeof(double) * v.size(),
                                       cudaMemcpyDeviceToHost, e->s),
                       "sns_ens_stats");
  if (!rc) rc = cuda_status(cudaStreamSynchronize(e->s), "sns_ens_stats");
  if (rc) return rc;
  for (int user = 0; user < nb; user++) {
    const int i = e->user_to_table[user];
    const BoxHost& b = e->boxes[i];
    const double N = (double)b.nx * b.ny * b.nz;
    out[4 * user + 0] = v[4 * i] / N;
    out[4 * user + 1] = 0.5 * v[4 * i + 1] / (N * N);
    out[4 * user + 2] = 0.5 * v[4 * i + 2] / (N * N);
    out[4 * user + 3] = v[4 * i + 3];
  }
  return OK;
}

int sns_ens_tuning(sns_ens* e, int* out, int max) {
  if (!e || !out || max < 0) {
    set_error("sns_ens_tuning: null argument");
    return ERR_ARG;
  }
  for (int s = 0; s < kEnsStages && 3 * s + 2 < max; s++) {
    out[3 * s] = e->cfg[s].threads;
    out[3 * s + 1] = e->cfg[s].wcap;
    out[3 * s + 2] = e->cfg[s].persistent;
  }
  return kEnsStages;
}

int sns_ens_stage_times(sns_ens* e, int nsteps, double* ms) {
  if (!e || !ms || nsteps < 1) {
    set_error("sns_ens_stage_times: null argument or no steps");
    return ERR_ARG;
  }
  std::vector<cudaEvent_t> ev((size_t)nsteps * (kEnsStages + 1), nullptr);
  int rc = OK;
  for (size_t i = 0; i < ev.size() && !rc; i++)
    rc = cuda_status(cudaEventCreate(&ev[i]), "sns_ens_stage_times");
  for (int t = 0; t < nsteps && !rc; t++) {
    cudaEvent_t* m = &ev[(size_t)t * (kEnsStages + 1)];
    rc = cuda_status(cudaEventRecord(m[0], e->s), "sns_ens_stage_times");
    for (int s = 0; s < kEnsStages && !rc; s++) {
      rc = launch_stage(e, s, e->s);
      if (!rc) rc = cuda_status(cudaEventRecord(m[s + 1], e->s), "sns_ens_stage_times");
    }
    if (!rc) {
      e->stepped = true;
      e->last_mode = SNS_ENS_EAGER;
    }
  }
  if (!rc) rc = cuda_status(cudaStreamSynchronize(e->s), "sns_ens_stage_times");
  for (int s = 0; s < kEnsStages; s++) ms[s] = 0;
  for (int t = 0; t < nsteps && !rc; t++) {
    cudaEvent_t* m = &ev[(size_t)t * (kEnsStages + 1)];
    for (int s = 0; s < kEnsStages && !rc; s++) {
      float x = 0;
      rc = cuda_status(cudaEventElapsedTime(&x, m[s], m[s + 1]), "sns_ens_stage_times");
      ms[s] += x / nsteps;
    }
  }
  for (cudaEvent_t x : ev)
    if (x) cudaEventDestroy(x);
  return rc ? rc : kEnsStages;
}

int sns_ens_launches_per_step(sns_ens* e, int mode) {
  if (!e) return ERR_ARG;
  if (mode == SNS_ENS_SEQUENTIAL) return kNSPasses * (int)e->boxes.size();
  return kEnsStages;
}

}  // extern "C"
