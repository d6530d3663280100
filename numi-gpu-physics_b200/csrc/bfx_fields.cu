// Derived flow diagnostics of a captured field frame (deriveFlowDiagnostics,
// Sources/BirdFlowVisualization/Metal/Visualization.metal:270-308): vorticity
// and the Q criterion from central differences of the physical velocity, one
// thread per cell, with the reference's operation order.
//
// Cells on the lattice boundary and cells whose 7-point stencil touches the
// body of the captured step are marked invalid and get zeros (the reference
// excludes cells within one cell of its analytic bird; here the occupancy of
// the captured step stands in for that distance).
#include <cuda_runtime.h>

#include <cstdint>

#include "bfx_internal.h"

namespace bfx {
namespace {

constexpr uint8_t kSolidBits = 0x3F;  // part id bits of the mask byte

__global__ void __launch_bounds__(256) k_flow_diagnostics(const float4* __restrict__ velocity,
                                                          const uint8_t* __restrict__ mask, int nx, int ny, int nz,
                                                          float scale, float4* __restrict__ vorticity,
                                                          float* __restrict__ q_criterion, uint8_t* __restrict__ valid) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= nx) return;
    const int64_t sy = nx, sz = (int64_t)nx * ny;
    const int64_t gid = x + sy * y + sz * z;
    bool ok = x > 0 && y > 0 && z > 0 && x + 1 < nx && y + 1 < ny && z + 1 < nz;
    if (ok && mask) {
        const uint8_t m = mask[gid] | mask[gid - 1] | mask[gid + 1] | mask[gid - sy] | mask[gid + sy] |
                          mask[gid - sz] | mask[gid + sz];
        ok = (m & kSolidBits) == 0;
    }
    if (!ok) {
        vorticity[gid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        q_criterion[gid] = 0.0f;
        valid[gid] = 0;
        return;
    }
    const float4 xp = velocity[gid + 1], xm = velocity[gid - 1];
    const float4 yp = velocity[gid + sy], ym = velocity[gid - sy];
    const float4 zp = velocity[gid + sz], zm = velocity[gid - sz];
    // d_a = (u(a + 1) - u(a - 1)) * scale: the derivative of each component along a
    const float dxx = (xp.x - xm.x) * scale, dxy = (xp.y - xm.y) * scale, dxz = (xp.z - xm.z) * scale;
    const float dyx = (yp.x - ym.x) * scale, dyy = (yp.y - ym.y) * scale, dyz = (yp.z - ym.z) * scale;
    const float dzx = (zp.x - zm.x) * scale, dzy = (zp.y - zm.y) * scale, dzz = (zp.z - zm.z) * scale;
    const float cx = dyz - dzy, cy = dzx - dxz, cz = dxy - dyx;
    const float trace_square = dxx * dxx + dyy * dyy + dzz * dzz + 2.0f * (dxy * dyx + dxz * dzx + dyz * dzy);
    vorticity[gid] = make_float4(cx, cy, cz, sqrtf(cx * cx + cy * cy + cz * cz));
    q_criterion[gid] = -0.5f * trace_square;
    valid[gid] = 1;
}

}  // namespace

void launch_flow_diagnostics(const float4* velocity, const uint8_t* mask, int nx, int ny, int nz, float scale,
                             float4* vorticity, float* q_criterion, uint8_t* valid, cudaStream_t s) {
    const dim3 block(256), grid((unsigned)((nx + 255) / 256), (unsigned)ny, (unsigned)nz);
    k_flow_diagnostics<<<grid, block, 0, s>>>(velocity, mask, nx, ny, nz, scale, vorticity, q_criterion, valid);
}

}  // namespace bfx
