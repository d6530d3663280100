// Shared pieces of the TMA-staged fused stream + collide kernel for the 16-bit
// TRT step (bfx_stream_kernels.cuh): tile geometry, the launch interface and the
// mbarrier / bulk-tensor PTX wrappers.
//
// Pipeline.  A persistent CTA owns a strided set of tiles (64 cells along x,
// 4 rows along y, one z plane).  One producer thread issues, per tile, one 4-D
// TMA box load per direction q (the 19 source rows of the AA pull, plus a
// 2-cell x margin) into a ring of shared-memory stages; four consumer warps
// each take one row, two cells per lane, read the 19 populations from shared
// memory, release the stage, collide in packed f32x2 arithmetic and store
// straight to HBM.  Loads of later tiles are in flight while a tile computes,
// so the kernel is bounded by HBM bandwidth or by issue, not by load latency.
#pragma once

#include <cuda.h>

#include "bfx_bulk.cuh"

namespace bfx {

constexpr int kTileX = 64;                  // cells along x per tile (one warp row, two cells per lane)
constexpr int kTileY = 4;                   // rows per tile = consumer warps per CTA
constexpr int kStreamThreads = 32 * (kTileY + 1);

template <class T>
struct StreamGeom {
    // box row: 64 cells plus the -1 / +1 x neighbours, rounded to 16 bytes
    static constexpr int row = (((kTileX + 2) * (int)sizeof(T) + 15) / 16) * 16 / (int)sizeof(T);
    static constexpr int plane_bytes = ((kTileY * row * (int)sizeof(T) + 127) / 128) * 128;
    static constexpr int stage_bytes = 19 * plane_bytes;
    static constexpr int tx_bytes = 19 * kTileY * row * (int)sizeof(T);
    // ring depth: 3 stages of 12 KB (16-bit), four CTAs per SM, about 100 KB
    // of loads in flight per SM
    static constexpr int stages = 3;
    // stages, their full / empty mbarriers, and slack to align the base to 128 B
    static constexpr int smem_bytes = stages * stage_bytes + 2 * stages * 8 + 128;
};

struct StreamTiles {
    int tiles_x, tiles_y;
    int ntiles;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: every iteration is a hardware-suspended try_wait, so the limit
// ends a wait that can no longer complete after at most a few seconds.
constexpr int kWaitLimit = 1 << 20;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// One 4-D box of the population tensor (x, y, z, plane) into shared memory,
// completing on the stage's mbarrier.  x is a multiple of 64 cells, so the
// start is 16-byte aligned; coordinates past the array read as zero.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

// Launch of the staged kernel for a 16-bit format and a collision operator
// that staged_collision accepts (bfx_fluid_fast.cu); a null BulkArgs only
// prepares the instantiations (shared-memory limit, occupancy).
void launch_stream_fast(int storage, int collision, int rep_s, const GridDesc& g, const BulkArgs* a,
                        const CUtensorMap* map, int sm_count, cudaStream_t s);

}  // namespace bfx
