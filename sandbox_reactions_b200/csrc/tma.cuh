// tma.cuh — tiled TMA loads (cp.async.bulk.tensor, no multicast) of a CTA's halo'd tile of f32 planes into shared
// memory, completing on an mbarrier, and the host-side encoding of their tensor maps.
//
// A tensor map here describes `planes` f32 planes of w x h (channel-major, row-major inside a plane, w a multiple of 4
// so every row stride is a multiple of 16 bytes) as a 3-D tensor (x, y, plane); a box of bx x by x planes lands in
// shared memory as [plane][by][bx]. Elements outside the planes read as zero. The box's x origin must be a multiple of
// 4 elements (16 bytes); the other coordinates may be negative or run past the edge.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "common.cuh"
#include "tc.cuh"

namespace tma {

// Arms `mbar` for one phase that completes when `bytes` have landed (one arrival: the calling thread's).
__device__ __forceinline__ void expect_tx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(mbar)), "r"(bytes)
                 : "memory");
}

// The box at (x, y, plane 0) of `map` into shared memory at `dst` (128-byte aligned), completing on `mbar`.
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(tc::smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z),
        "r"(tc::smem_addr(mbar))
        : "memory");
}

}  // namespace tma

// Host: the tensor map of `planes` f32 planes of w x h at `base` (16-byte aligned), box bx x by x planes.
void tma_encode_planes(CUtensorMap* map, const float* base, int w, int h, int planes, int bx, int by);
