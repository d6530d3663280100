// Kernel templates of the fused stream + collide step, shared by two
// translation units that differ only in floating-point contraction:
//   bfx_fluid.cu       --fmad=false  FP32 and FP64 storage, bit-identical to the
//                                    reference operation order (default)
//   bfx_fluid_fast.cu  --fmad=true   the 16-bit deviation formats and the
//                                    opt-in fast_math FP32 mode
// The including file defines BFX_VARIANT, the namespace that keeps the two
// sets of instantiations apart.
#pragma once

#include "bfx_device.cuh"
#include "bfx_internal.h"

namespace bfx {

struct BulkArgs {
    void* plane[19];        // A + q * padded cells: base of direction q's plane
    int32_t doff[19];       // c_q . (1, px, px*py): padded neighbour offset of direction q
    float far_eq_f[19];     // equilibrium(q, far density, far velocity), FP32
    double far_eq_d[19];    // same in FP64 (FP64 storage)
    float far_dev[19];      // (far_eq_f - w_q) x the storage's deviation scale (16-bit formats)
    // x-face values of the staged kernel (face_values 1; the halo fill then
    // skips the x faces): the stored deviation of what the fill writes for
    // direction q across face f (0: -x, 1: +x), read back as the kernel reads
    // a population
    int face_values;
    float face_dev[2][19];
    int box[3];             // geometry box extent (origin in DeviceState); rare-cell launch
    void* pops;
    const uint8_t* mask;
    const float4* wall;
    float* density;
    float4* velocity;
    DeviceState* state;
    void* tape;             // pre-collision (rho, u) per cell (capture == 2)
    Grid g;
    FluidParams fp;
    int capture;            // 0 none, 1 macroscopic fields, 2 adjoint tape
};

// Fused-step launch for the contracted variant (bfx_fluid_fast.cu).
void launch_bulk_fast(int storage, int collision, int rep_s, const GridDesc& g, const BulkArgs& a, cudaStream_t s);
// Solid / newly uncovered cells of the geometry box for the staged kernel (contracted variant).
void launch_rare_fast(int storage, int collision, int rep_s, const BulkArgs& a, cudaStream_t s);
// Host-side construction of BulkArgs (bfx_fluid.cu).
BulkArgs make_bulk_args(const GridDesc& gd, const FluidParams& fp, const FluidBuffers& b, int capture, int storage);
void cell_launch_shape(const GridDesc& g, dim3& grid, dim3& block);

// spongeFactor: BF.metal:2427-2446
__device__ __forceinline__ float sponge_factor(const Grid& g, const FluidParams& fp, int x, int y, int z) {
    unsigned dx = min((unsigned)x, (unsigned)(g.nx - 1 - x));
    unsigned dy = min((unsigned)y, (unsigned)(g.ny - 1 - y));
    unsigned dz = min((unsigned)z, (unsigned)(g.nz - 1 - z));
    float distance = (float)min(dx, min(dy, dz));
    float width = fp.sponge_width;
    if (distance >= width) return 0.0f;
    float nd = fminf(fmaxf((width - distance) / fmaxf(width, 1.0f), 0.0f), 1.0f);
    return fp.sponge_strength * nd * nd;
}

}  // namespace bfx
