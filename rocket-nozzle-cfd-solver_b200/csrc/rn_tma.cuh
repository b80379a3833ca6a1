// rn_tma.cuh -- tensor-memory-accelerator (TMA) staging of a tile's halo.
//
// The stage kernels start by copying the raw state of their tile plus its
// 2-cell halo (the A and B float4 planes) and the matching block of the solid
// mask from global memory into shared memory with 2-D tiled bulk tensor
// copies (cp.async.bulk.tensor), issued by one thread and completed on an
// mbarrier. Cells outside the grid arrive as zeros (the copy's out-of-bounds
// fill); the ghost-cell pass (FS_PRIM, solver.js:56-126) then overwrites them
// from the in-grid cells already in shared memory. The copies read this GPU's
// own memory only and never multicast.
//
// One TileMaps per tile shape and solver handle, in device memory: the box of
// a copy is part of its tensor map, and the box follows the tile shape.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace rn {

struct TileMaps {
  CUtensorMap a[3];     // state ring slots, plane A: box (PX x PY) float4 as 4*PX floats
  CUtensorMap b[3];     // plane B
  CUtensorMap mask;     // row-pitched copy of the solid mask: box (MW x PY) bytes
  CUtensorMap geoM;     // geoM with a 1-cell ring: box (TX+2) x (TY+2) float4 (shapes that stage it)
  CUtensorMap geoG;     // geoG of the tile: box TX x TY float4
};

// Width in bytes of the mask box of a tile whose halo row is PX cells wide:
// the box starts at the 16-byte boundary at or below the halo's first column
// (up to 15 bytes early), so it covers PX + 15 bytes, rounded up to 16.
__host__ __device__ constexpr int mask_box_width(int PX) { return ((PX + 15 + 15) / 16) * 16; }

#ifdef __CUDACC__
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  // make the initialised barrier visible to the copy engine before any copy names it
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// One 2-D tile of `map` at element coordinates (x, y) into shared memory at
// dst, completing `bar`. x times the element size is a multiple of 16 bytes
// at every call site (a float4 column times 16 bytes, or a mask column
// rounded down to a multiple of 16).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
          "r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase 0 of `bar` at most `limit` polls (each poll itself waits a
// short, hardware-defined time); false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned limit) {
  for (unsigned it = 0; it < limit; it++)
    if (mbar_try_wait(bar, 0)) return true;
  return false;
}
#endif

}  // namespace rn
