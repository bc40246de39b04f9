// Tensor Memory Accelerator (TMA) loads of field tiles into shared memory,
// written from the PTX ISA's cp.async.bulk.tensor / mbarrier expect_tx
// descriptions and the driver API's cuTensorMapEncodeTiled.
//
// A field of nx * ny * nz complex elements (x fastest) is described to the
// TMA as a 3D tensor of 8-byte units: dims (nx * esz / 8, ny, nz), byte
// strides nx * esz and nx * ny * esz.  One load copies a box of
// (bw * esz / 8, bg, bz) units starting at (x0 * esz / 8, y0, z0) into shared
// memory, densely in [z][y][x] order, and signals completion on an mbarrier
// through its transaction count.  Loads read only this GPU's own fields and
// never use cluster multicast.
//
// Alignment (checked by the host before any launch): the field's base is 16
// byte aligned (every pool and cudaMalloc block is), bw * esz is a multiple of
// 16 bytes, and every x0 * esz a kernel asks for is a multiple of 16 bytes
// (x0 a multiple of bw).
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "sns_tc.cuh"

namespace sns {

// Host: the tensor map of a field for boxes of (bw, bg, bz) complex elements
// (bw, bg, bz <= 256 units each).  OK, or ERR_UNSUPPORTED when the driver
// lacks the entry point or refuses the map (the error text says which).
int field_tensor_map(CUtensorMap* map, const void* base, int nx, int ny, int nz, int esz, int bw,
                     int bg, int bz);
// Host: whether the TMA can load (bw, bg, bz) boxes of such a field.
bool field_box_ok(int nx, int ny, int nz, int esz, int bw, int bg, int bz);

namespace tma {

// Announce `bytes` of incoming transactions on the mbarrier and arrive once.
__device__ __forceinline__ void expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(mbar)),
               "r"(bytes)
               : "memory");
}

// Plain arrival (no transactions) on the mbarrier.
__device__ __forceinline__ void arrive(uint64_t* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(mbar)) : "memory");
}

// Box at coordinates (c0, c1, c2) of the tensor `map` (8-byte units along
// c0) into shared memory at dst; completes on mbar.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                        uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(tc::smem_u32(mbar))
      : "memory");
}

// Contiguous bytes [src, src + bytes) of global memory into shared memory at
// dst (both 16-byte aligned, bytes a multiple of 16); completes on mbar.
__device__ __forceinline__ void load_bulk(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(tc::smem_u32(mbar))
      : "memory");
}

// Order this thread's earlier generic-proxy accesses of shared memory before
// its later async-proxy ones (a TMA load into a buffer the CTA has read).
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Fetch the tensor map (a kernel parameter) into the TMA unit's cache.
__device__ __forceinline__ void prefetch_map(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace tma
}  // namespace sns
