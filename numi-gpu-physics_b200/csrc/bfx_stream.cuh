// Shared pieces of the TMA-staged fused stream + collide kernel for the 16-bit
// TRT step (bfx_stream_kernels.cuh): tile geometry, the launch interface and the
// mbarrier / bulk-tensor PTX wrappers.
//
// Pipeline.  A persistent CTA (one per SM) owns a strided set of tiles: W
// consumer warps side by side along x (64 cells each), Y rows along y, one z
// plane (StreamShape).  One producer thread issues, per tile, one 4-D TMA box
// load per direction q (the 19 source rows of the AA pull, plus the x margin)
// into a ring of shared-memory stages; each consumer warp takes 64 cells of
// one row, two cells per lane, reads the 19 populations from shared memory,
// releases the stage, collides in packed f32x2 arithmetic and stores straight
// to HBM.  Loads of later tiles are in flight while a tile computes.
#pragma once

#include <cuda.h>

#include "bfx_bulk.cuh"

namespace bfx {

constexpr int kTileX = 64;  // cells along x per consumer warp (two per lane)

// Tile shape and ring depth per collision operator.  Measured on B200 on the
// 512x256x256 flapping plates in FP16 (kernel time per step):
//   TRT          64x4, 3 stages, 4 CTAs/SM 0.705 ms; 64x16, 2 stages 0.536 ms;
//                128x8, 2 stages 0.522 ms (chosen)
//   RR3          64x4, 3 stages 0.733 ms; 64x12, 2 stages 0.680 ms;
//                64x12, 3 stages 0.662 ms (chosen)
// Taller and wider boxes make fewer, longer TMA requests with less x-margin
// overhead per byte; for the memory-bound TRT step a shallow ring (about
// 85 KB of loads in flight per SM) is faster than a deep one, while the
// arithmetic-heavier regularized operators want twelve consumer warps and
// one more stage to cover their longer tiles.
template <int COLL>
struct StreamShape {
    static constexpr bool trt = COLL == BFX_COLLISION_TRT;
    static constexpr int W = trt ? 2 : 1;         // consumer warps per row
    static constexpr int Y = trt ? 8 : 15;        // rows per tile
    static constexpr int stages = trt ? 2 : 3;    // shared-memory ring depth
    static constexpr int consumers = W * Y;
    static constexpr int threads = 32 * (consumers + 1);  // + one producer warp
    // Register cap of a thread.  The TRT step needs 80 without spilling, which
    // leaves about 22 K of an SM's registers to the geometry kernels that the
    // pipelined build runs beside it; the regularized operators take what one
    // CTA of 16 warps can have.
    static constexpr int max_regs = trt ? 80 : 65536 / threads;
};

template <class T, int COLL>
struct StreamGeom {
    using SH = StreamShape<COLL>;
    // box row: the tile's cells plus the -1 / +1 x neighbours, rounded to 16 bytes
    static constexpr int row = (((kTileX * SH::W + 2) * (int)sizeof(T) + 15) / 16) * 16 / (int)sizeof(T);
    static constexpr int plane_bytes = ((SH::Y * row * (int)sizeof(T) + 127) / 128) * 128;
    static constexpr int stage_bytes = 19 * plane_bytes;
    static constexpr int tx_bytes = 19 * SH::Y * row * (int)sizeof(T);
    static constexpr int stages = SH::stages;
    // stages, their full / empty mbarriers, and slack to align the base to 128 B
    static constexpr int smem_bytes = stages * stage_bytes + 2 * stages * 8 + 128;
    static_assert(row <= 256 && SH::Y <= 256, "a TMA box spans at most 256 elements per dimension");
    static_assert(smem_bytes <= 227 * 1024, "shared memory of one CTA");
};

struct StreamTiles {
    int tiles_x, tiles_y;
    int ntiles;
    int step_x, step_y, step_z;  // the grid stride (CTAs) in tile coordinates
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
constexpr uint32_t kWaitLimit = 1u << 20;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
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
