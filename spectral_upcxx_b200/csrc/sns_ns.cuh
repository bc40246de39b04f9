// Fused NS step (host interface).
#pragma once

#include <cuda_runtime.h>

#include "sns_xy.cuh"

namespace sns {

struct NSPlan {
  int nx, ny, nz, prec;
  int xG;             // rows per CTA of the x cross pass
  bool x_tma;         // the x cross pass as a persistent pass over TMA-staged rows
  bool x_occ;         // its direct-load form compiled for five CTAs of <= 192 threads per SM
  bool z_tma;         // the update pass as a persistent pass over TMA-staged z lines
  bool carry;         // the update pass also does the next step's K1 (z-inverse of
                      // the new V and its curl into U), so the next step skips K1
  bool carry_reload;  // ... reading the new V back from V (L1/L2) instead of keeping
                      // it in a second set of shared-memory rows
  bool z_pfself;      // the update pass asks L2 for each tile's V and C0 once the
                      // cross product's loads are in flight
  int k1W, k1G;       // K1 tile: adjacent z lines x groups (all six outputs per CTA)
  bool k1_fused;      // K1 loads V once per tile (else one output field per CTA)
  bool k1_reload;     // the fused K1 forms omega from reloads of V (L1), not shared memory
  bool k1_tma;        // the fused K1 as a persistent pass over TMA-staged tiles
  int k1_stages;      // its stages (1 or 2)
  bool k1_lines;      // K1 as a line pass of V and i kz V (5 fields into the work
                      // fields W), the curl formed in K2's prologue (PRO_OMEGA)
  int k1lW, k1lT;     // tile knobs of that z line pass (axis_geo wmax, tmax)
  int zW;             // adjacent z lines per CTA of the update pass
  int update_blocks;  // CTAs of the update pass (= diagnostics partials)
  int sgs_W;          // adjacent z lines per CTA of the closure update (9 fields)
  int sgs_blocks;     // its CTAs (= diagnostics partials of a closure step)
  bool use_xy;        // xy phase as one persistent dataflow launch
  bool use_xyc;       // xy phase as one cluster pass over each plane (sns_xyc.cu)
  XYPlan xy;
  int xy_chunk;       // planes per slab of the separate xy passes (0 = all)
  int lineW;          // adjacent lines per tile of the y/z line passes (0 = default)
  int lineT;          // threads per CTA up to which line groups are added (0 = default)
  int lineOrd;        // radix order of the y line passes (RadixOrder)
  int y_tma;          // the y line passes over TMA-staged tiles: 0 (direct loads), or
                      // the number of shared-memory stages (1, 2)
  bool tuned;         // the knobs above were chosen by measurement (ns_tune_plan)
  int pf_waves;       // L2 prefetch of each pass's tile this many waves ahead (0: none)
  int passes;         // timed phases per step: z-inverse, xy, z-forward+update
  bool real;          // half-spectrum fields of a real velocity (R2C / C2R along x)
  int nx_phys;        // physical nx (= nx, or 2 nx for a real-field run)
  double kc2;         // spectral cutoff |k|^2 <= kc2 of the evolved modes (1e300: none)
  double sgs_klo, sgs_kinv;  // closure: stress divergence weight clamp((|k|-klo) kinv, 0, 1)
};

// zW > 0 and lineW > 0 select tuned tile widths (0 = defaults).
// real = true: a real-field run on the half spectrum kx = 0 .. nx/2-1 (pl.nx
// is then nx/2, the stored row length; pl.nx_phys = nx).
int ns_plan(NSPlan& pl, int nx, int ny, int nz, int prec, int zW = 0, int lineW = 0,
            bool real = false);
// One step in place on V (Fourier velocity) and C0 (previous cross product),
// with six work fields U; per-block diagnostics go to `stats`
// (4 doubles x update_blocks).
// `ev`, when not null, holds kNSPasses + 1 events recorded around the passes.
// `sync_words` (xy_sync_words(nz) ints) serves the dataflow xy pass.  W: five
// more work fields, needed when pl.k1_lines (else may be null).
// `carried` (may be null: no carrying) tracks, for a plan with pl.carry,
// whether U already holds K1's output for the current V: when *carried is
// true the step skips K1 (its pass time is then empty); on return it says
// whether this step's K5 left the next step's K1 output in U.  Anything else
// that writes V or U must clear it.
constexpr int kNSPasses = 5;
constexpr int kNSLineWork = 5;
int ns_step_once(const NSPlan& pl, void* const V[3], void* const C0[3], void* const U[6],
                 double* stats, int* sync_words, double nu, double dt, cudaStream_t s,
                 cudaEvent_t* ev = nullptr, void* const* W = nullptr, bool* carried = nullptr);
// K1 alone (z-inverse of V and of i k x V into U[0..5]), for a carrying plan
// whose U does not hold it yet (before a captured steady-state step).
int ns_k1_once(const NSPlan& pl, void* const V[3], void* const U[6], int* sync_words,
               cudaStream_t s);
// The update pass (z-forward + AB2 / projection / CN update) on the fields of
// `a`; sgs adds the divergence of the Fourier eddy stress a.tau.
struct UpdateArgs;
// err: the step's error word (the TMA-staged form records its bounded waits
// there); null keeps the direct-load form.
int ns_update(const NSPlan& pl, const UpdateArgs& a, bool sgs, cudaStream_t s,
              int* err = nullptr);
// Autotuner of the plain complex or real step (the counterpart of the
// reference's FFTW_MEASURE planning, src/FFT1D.cpp:18-22): times the passes
// of candidate plans on the stepper's own fields -- which must hold no state
// yet: the timing steps fill V and C0 with seeded data, and the caller clears
// them after -- and keeps, pass by pass,
// the fastest: K1 tile (W x G, or one output field per CTA), the y passes'
// run width, thread cap and radix order, the x pass's rows per CTA and the
// update pass's width.  `max_blocks` is the capacity of `stats` in update
// blocks.  Plans of another pass structure (fused xy phases) are left as they
// are.
int ns_tune_plan(NSPlan& pl, void* const V[3], void* const C0[3], void* const U[6],
                 double* stats, int max_blocks, int* sync_words, cudaStream_t s,
                 void* const* W = nullptr);
// Reduce the per-block diagnostics into out4 (device): sum|div|, sum|V|^2,
// sum|i k x V|^2, max|div|.
int ns_stats_final(const double* partials, int blocks, double* out4, cudaStream_t s);
// out4 (device, from ns_stats_final) -> div_avg, energy, enstrophy, max_div of
// an N-point grid, as sns_ns_stats reports them.
int ns_stats_normalise(double* out4, double N, cudaStream_t s);

}  // namespace sns
