// Persistent dataflow kernel for the xy phase of the NS step (host interface).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <algorithm>

namespace sns {

struct XYArgs {
  void* U[6];
  int nx, ny, nz;
  int W;   // x columns per A/C item
  int G;   // rows per B item
  int nA, nB, nC;  // items per plane
  int D;   // plane lag between the item kinds in the ticket order
  double scale2;   // 1/N^2 for the cross product of unnormalised fields
  unsigned long long* ticket;
  int* cntA;  // per plane: finished A items
  int* cntB;  // per plane: finished B items
  int* err;   // set when a wait gives up
  long long spin_limit;
};

struct XYPlan {
  int nx, ny, nz, prec;
  int W, G, threads;
  size_t smem_bytes;
  int nA, nB, nC, D;
  int* sync_words;
  size_t sync_bytes_to_clear;
};

bool xy_supported(int nx, int ny, int prec);
int xy_plan(XYPlan& p, int nx, int ny, int nz, int prec);
// Number of ints the sync buffer needs: ticket (2), per-plane counters
// (2*nz), error word (1).  The error word is the last one.
size_t xy_sync_words(int nz);
// y-inverse (6 fields) + x cross + y-forward (3 fields) of U in place.
int xy_run(const XYPlan& p, void* const U[6], int* sync_words, cudaStream_t s);

// The same phase as one pass over each xy plane on a thread-block cluster
// (sns_xyc.cu): nx = ny = 128, or 256 in complex64, where a cluster fits.
bool xyc_supported(int nx, int ny, int prec);
int xyc_run(void* const U[6], int nx, int ny, int nz, int prec, cudaStream_t s);

}  // namespace sns
