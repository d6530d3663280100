// Device helpers shared by the geometry kernels (bfx_geometry.cu) and the
// adjoint kernels (bfx_adjoint.cu): float3 arithmetic in the reference's
// operation order, quaternions, the triangle closest point, the geometry box,
// the link predicate and the fixed-order block reductions.
#pragma once

#include "bfx_device.cuh"
#include "bfx_internal.h"

namespace bfx {

struct GeomArgs {
    Grid g;
    FluidParams fp;
    int bx, by, bz;          // box extent
    int64_t box_cells;
    GeomBuffers b;
    void* pops;
};

// ---------------------------------------------------------------------------
// float3 helpers with the reference's operation order.
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 v3(const float4& a) { return V3{a.x, a.y, a.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
__device__ __forceinline__ float4 f4(V3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

__device__ __forceinline__ V3 cell_world(const FluidParams& fp, int x, int y, int z) {
    return v3(fp.origin[0] + ((float)x + 0.5f) * fp.dx, fp.origin[1] + ((float)y + 0.5f) * fp.dx,
              fp.origin[2] + ((float)z + 0.5f) * fp.dx);
}

// Quaternions (x, y, z, w).  Normalisation divides by the correctly rounded
// norm so host and device agree bit for bit.
__device__ __forceinline__ float4 qnormalize(float4 q) {
    float n2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
    if (n2 > 1.0e-20f) {
        float n = sqrtf(n2);
        return make_float4(q.x / n, q.y / n, q.z / n, q.w / n);
    }
    return make_float4(0.0f, 0.0f, 0.0f, 1.0f);
}
__device__ __forceinline__ V3 qrotate(float4 q, V3 v) {
    V3 qv = v3(q.x, q.y, q.z);
    V3 t = cross(qv, v);
    t = v3(t.x * 2.0f, t.y * 2.0f, t.z * 2.0f);
    V3 c2 = cross(qv, t);
    return v3(v.x + q.w * t.x + c2.x, v.y + q.w * t.y + c2.y, v.z + q.w * t.z + c2.z);
}
__device__ __forceinline__ V3 qunrotate(float4 q, V3 v) { return qrotate(make_float4(-q.x, -q.y, -q.z, q.w), v); }
// rotateAroundAxis (BF.metal:466-473) with the angle's sine and cosine given
__device__ __forceinline__ V3 rotate_axis_sc(V3 v, V3 axis, float s, float c) {
    V3 cr = cross(axis, v);
    float d = dot(axis, v);
    return v3(v.x * c + cr.x * s + axis.x * d * (1.0f - c), v.y * c + cr.y * s + axis.y * d * (1.0f - c),
              v.z * c + cr.z * s + axis.z * d * (1.0f - c));
}
// rotateAroundAxis: BF.metal:466-473
__device__ __forceinline__ V3 rotate_axis(V3 v, V3 axis, float angle) {
    return rotate_axis_sc(v, axis, bfx_sinf(angle), bfx_cosf(angle));
}
__device__ __forceinline__ V3 normalize3(V3 v) {
    float l = length(v);
    return v3(v.x / l, v.y / l, v.z / l);
}

// Cell of this thread in box block (bxi, byi, bzi) of a box launch.
__device__ __forceinline__ bool box_cell_at(const GeomArgs& a, int bxi, int byi, int bzi, int& x, int& y, int& z,
                                            int64_t& bidx) {
    int lx = bxi * blockDim.x + threadIdx.x;
    int ly = byi * blockDim.y + threadIdx.y;
    int lz = bzi;
    if (lx >= a.bx || ly >= a.by || lz >= a.bz) return false;
    const int32_t* o = a.b.state->box_origin;
    x = o[0] + lx;
    y = o[1] + ly;
    z = o[2] + lz;
    bidx = (int64_t)lx + (int64_t)a.bx * ((int64_t)ly + (int64_t)a.by * lz);
    return x < a.g.nx && y < a.g.ny && z < a.g.nz;
}
__device__ __forceinline__ bool box_cell(const GeomArgs& a, int& x, int& y, int& z, int64_t& bidx) {
    int lx = blockIdx.x * blockDim.x + threadIdx.x;
    int ly = blockIdx.y * blockDim.y + threadIdx.y;
    int lz = blockIdx.z;
    if (lx >= a.bx || ly >= a.by || lz >= a.bz) return false;
    const int32_t* o = a.b.state->box_origin;
    x = o[0] + lx;
    y = o[1] + ly;
    z = o[2] + lz;
    bidx = (int64_t)lx + (int64_t)a.bx * ((int64_t)ly + (int64_t)a.by * lz);
    return x < a.g.nx && y < a.g.ny && z < a.g.nz;
}

// Active bounds of the step: the cells of the geometry box within
// fp.act_margin of the mesh vertices' bounding box (the whole box for the
// analytic shapes).  Cells outside hold no key, no link and no topology
// change, and their mask bytes are 0 in both buffers.
__device__ __forceinline__ void active_bounds(const GeomArgs& a, int (&lo)[3], int (&hi)[3]) {
    const DeviceState* st = a.b.state;
    const int ext[3] = {a.bx, a.by, a.bz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int l = st->act_lo[k] - a.fp.act_margin, h = st->act_hi[k] + a.fp.act_margin;
        lo[k] = l > st->box_origin[k] ? l : st->box_origin[k];
        const int top = st->box_origin[k] + ext[k] - 1;
        hi[k] = h < top ? h : top;
    }
}
// Slab launches: a block covers kSlabZ consecutive z slices of its (x, y)
// tile, one cell per thread and slice, so empty parts of the box cost a
// quarter of the blocks.
constexpr int kSlabZ = 4;
__device__ __forceinline__ bool slab_cell(const GeomArgs& a, int k, int& x, int& y, int& z, int64_t& bidx) {
    int lx = blockIdx.x * blockDim.x + threadIdx.x;
    int ly = blockIdx.y * blockDim.y + threadIdx.y;
    int lz = blockIdx.z * kSlabZ + k;
    if (lx >= a.bx || ly >= a.by || lz >= a.bz) return false;
    const int32_t* o = a.b.state->box_origin;
    x = o[0] + lx;
    y = o[1] + ly;
    z = o[2] + lz;
    bidx = (int64_t)lx + (int64_t)a.bx * ((int64_t)ly + (int64_t)a.by * lz);
    return x < a.g.nx && y < a.g.ny && z < a.g.nz;
}
// Every cell of the slab block lies outside the active bounds (uniform over the block).
__device__ __forceinline__ bool slab_inactive(const GeomArgs& a) {
    int lo[3], hi[3];
    active_bounds(a, lo, hi);
    const int32_t* o = a.b.state->box_origin;
    const int x0 = o[0] + (int)(blockIdx.x * blockDim.x), x1 = x0 + (int)blockDim.x - 1;
    const int y0 = o[1] + (int)(blockIdx.y * blockDim.y), y1 = y0 + (int)blockDim.y - 1;
    const int z0 = o[2] + (int)blockIdx.z * kSlabZ, z1 = z0 + kSlabZ - 1;
    return x1 < lo[0] || x0 > hi[0] || y1 < lo[1] || y0 > hi[1] || z1 < lo[2] || z0 > hi[2];
}

// The cells of box_cell's block all lie outside the active bounds (uniform
// over the block).
__device__ __forceinline__ bool block_inactive_at(const GeomArgs& a, int bxi, int byi, int bzi) {
    int lo[3], hi[3];
    active_bounds(a, lo, hi);
    const int32_t* o = a.b.state->box_origin;
    const int x0 = o[0] + bxi * (int)blockDim.x, x1 = x0 + (int)blockDim.x - 1;
    const int y0 = o[1] + byi * (int)blockDim.y, y1 = y0 + (int)blockDim.y - 1;
    const int z = o[2] + bzi;
    return x1 < lo[0] || x0 > hi[0] || y1 < lo[1] || y0 > hi[1] || z < lo[2] || z > hi[2];
}
__device__ __forceinline__ bool block_inactive(const GeomArgs& a) {
    return block_inactive_at(a, blockIdx.x, blockIdx.y, blockIdx.z);
}
__device__ __forceinline__ bool in_bounds(const int (&lo)[3], const int (&hi)[3], int x, int y, int z) {
    return x >= lo[0] && x <= hi[0] && y >= lo[1] && y <= hi[1] && z >= lo[2] && z <= hi[2];
}
__device__ __forceinline__ bool cell_active(const GeomArgs& a, int x, int y, int z) {
    int lo[3], hi[3];
    active_bounds(a, lo, hi);
    return in_bounds(lo, hi, x, y, z);
}

__device__ __forceinline__ uint8_t topo_flags(uint8_t part, uint8_t prev_part, int has_prev) {
    if (!has_prev) return part;
    if (part && !prev_part) return (uint8_t)(part | kCovered);
    if (!part && prev_part) return kUncovered;
    return part;
}


// ---------------------------------------------------------------------------
// Triangle mesh (BF.metal:1529-1583 closest point, 1638-1686 raster,
// 1697-1738 / 1978-2039 resolve).  Keys are 64-bit: quantised distance
// (1/65536 cell) in the high word, triangle id in the low word, so meshes are
// not limited to the reference's 4,096 triangles and ties stay deterministic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ V3 closest_point(V3 p, V3 a, V3 b, V3 c, V3& bary) {
    V3 ab = b - a, ac = c - a, ap = p - a;
    float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        bary = v3(1, 0, 0);
        return a;
    }
    V3 bp = p - b;
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
        bary = v3(0, 1, 0);
        return b;
    }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float v = d1 / (d1 - d3);
        bary = v3(1.0f - v, v, 0);
        return v3(a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z);
    }
    V3 cp = p - c;
    float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) {
        bary = v3(0, 0, 1);
        return c;
    }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float w = d2 / (d2 - d6);
        bary = v3(1.0f - w, 0, w);
        return v3(a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z);
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        bary = v3(0, 1.0f - w, w);
        return v3(b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z));
    }
    float inv = 1.0f / fmaxf(va + vb + vc, 1.0e-20f);
    float v = vb * inv, w = vc * inv;
    bary = v3(1.0f - v - w, v, w);
    return v3(a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w);
}

// Articulated vertex placement: segment 0 rides the body frame, 1 / 2 the left
// / right wing frames (the indexed surface preparation of BF.metal:1589-1622,

__device__ __forceinline__ void tri_vertices(const GeomArgs& a, uint32_t t, V3& A, V3& B, V3& C) {
    A = v3(a.b.mesh_pos[a.b.mesh_tris[3 * t]]);
    B = v3(a.b.mesh_pos[a.b.mesh_tris[3 * t + 1]]);
    C = v3(a.b.mesh_pos[a.b.mesh_tris[3 * t + 2]]);
}


// ---------------------------------------------------------------------------
// Link predicate and link fractions.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool persistent_fluid(uint8_t m_next, uint8_t m_prev) {
    return (m_next & (kPartMask | kUncovered)) == 0 && (m_prev & kPartMask) == 0;
}
// Solid source of link (x, q) or -1.
__device__ __forceinline__ int64_t link_source(const Grid& g, const uint8_t* mask_next, int x, int y, int z, int q,
                                               int& sx, int& sy, int& sz) {
    sx = x - cx(q);
    sy = y - cy(q);
    sz = z - cz(q);
    if (!wrap(g, sx, sy, sz)) return -1;
    int64_t s = flat(g, sx, sy, sz);
    return (mask_next[s] & kPartMask) ? s : -1;
}

// Solid link sources of cell (x, y, z): bit q set when the source x - c_q is
// solid, i.e. a cut link in direction q.  The 18 mask bytes are loaded in two
// groups of nine, each group's loads issued together so their latencies
// overlap (all 18 at once would cost the callers' occupancy in registers).
__device__ __forceinline__ uint32_t link_sources(const Grid& g, const uint8_t* mask_next, int x, int y, int z) {
    uint32_t bits = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        uint8_t m[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const int q = 1 + 9 * h + k;
            int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
            m[k] = wrap(g, sx, sy, sz) ? mask_next[flat(g, sx, sy, sz)] : (uint8_t)0;
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) bits |= (m[k] & kPartMask) ? 1u << (1 + 9 * h + k) : 0u;
    }
    return bits;
}

// Ten-iteration bisection from the fluid node toward the solid node on the

__device__ __forceinline__ float tri_distance(const GeomArgs& a, uint32_t t, V3 w) {
    V3 A, B, C, bary;
    tri_vertices(a, t, A, B, C);
    V3 cp = closest_point(w, A, B, C, bary);
    return length(w - cp);
}

__device__ __forceinline__ unsigned long long box_key(const GeomArgs& a, int x, int y, int z) {
    const int32_t* o = a.b.state->box_origin;
    int lx = x - o[0], ly = y - o[1], lz = z - o[2];
    if (lx < 0 || ly < 0 || lz < 0 || lx >= a.bx || ly >= a.by || lz >= a.bz) return 0xFFFFFFFFFFFFFFFFull;
    return a.b.keys[(int64_t)lx + (int64_t)a.bx * ((int64_t)ly + (int64_t)a.by * lz)];
}

// Wall position along the link as the bracketed root of

// ---------------------------------------------------------------------------
// Block reductions in a fixed order (deterministic).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int linear_tid() { return threadIdx.x + blockDim.x * threadIdx.y; }

// Fixed-order tree over the (up to 256) threads of a block; every thread
// receives the block total.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double (*sh)[256]) {
    const int t = linear_tid();
    const int nt = blockDim.x * blockDim.y;
    for (int k = 0; k < K; ++k) sh[k][t] = v[k];
    for (int k = 0; k < K; ++k)
        if (t + nt < 256) sh[k][t + nt] = 0.0;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (t < s)
            for (int k = 0; k < K; ++k) sh[k][t] += sh[k][t + s];
        __syncthreads();
    }
    for (int k = 0; k < K; ++k) v[k] = sh[k][0];
    __syncthreads();
}

// FP64 load contribution: lattice force fl applied at point pt (both in the
// precision the step computes in), torque about the FP64 body position.
template <class R>
__device__ __forceinline__ void add_load(double (&acc)[8], R flx, R fly, R flz, R ptx, R pty, R ptz,
                                         const double* body, float f2p) {
    double fp[3] = {(double)flx * (double)f2p, (double)fly * (double)f2p, (double)flz * (double)f2p};
    double r[3] = {(double)ptx - body[0], (double)pty - body[1], (double)ptz - body[2]};
    acc[0] += (double)flx;
    acc[1] += (double)fly;
    acc[2] += (double)flz;
    acc[3] += r[1] * fp[2] - r[2] * fp[1];
    acc[4] += r[2] * fp[0] - r[0] * fp[2];
    acc[5] += r[0] * fp[1] - r[1] * fp[0];
}

static inline GeomArgs make_geom(const GridDesc& gd, const FluidParams& fp, const BoxDesc& box, const GeomBuffers& gb,
                          void* pops) {
    GeomArgs a;
    a.g = device_grid(gd);
    a.fp = fp;
    a.bx = box.sx;
    a.by = box.sy;
    a.bz = box.sz;
    a.box_cells = box.cells;
    a.b = gb;
    a.pops = pops;
    return a;
}

static inline void box_shape(const BoxDesc& box, dim3& grid, dim3& block) {
    int bx = box.sx >= 64 ? 64 : ((box.sx + 31) / 32) * 32;
    if (bx < 32) bx = 32;
    int by = 256 / bx;
    block = dim3(bx, by, 1);
    grid = dim3((box.sx + bx - 1) / bx, (box.sy + by - 1) / by, box.sz);
}
static inline void slab_shape(const BoxDesc& box, dim3& grid, dim3& block) {
    box_shape(box, grid, block);
    grid.z = (unsigned)((box.sz + kSlabZ - 1) / kSlabZ);
}

}  // namespace bfx
