// Device-side building blocks of the D3Q19 moving-boundary step: lattice
// constants, population storage formats, the in-place AA addressing and the
// equilibrium.  All arithmetic follows the operation order of the reference
// fluid kernel (Sources/BirdFlowMetal/Metal/BirdFlow.metal, stepFluidTRT
// 2507-3236) so the FP32 path is bit-identical to a non-contracted CPU
// evaluation; the library is compiled with --fmad=false for that reason.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "bfx_portable_math.h"
#include "bfx_types.h"

namespace bfx {

// ---------------------------------------------------------------------------
// D3Q19 velocity set in the reference order (BF.metal:7-43).  constexpr
// functions fold to immediates inside unrolled loops.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int cx(int q) {
    return (q == 1 || q == 7 || q == 9 || q == 11 || q == 13) ? 1
         : (q == 2 || q == 8 || q == 10 || q == 12 || q == 14) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int q) {
    return (q == 3 || q == 7 || q == 10 || q == 15 || q == 17) ? 1
         : (q == 4 || q == 8 || q == 9 || q == 16 || q == 18) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int q) {
    return (q == 5 || q == 11 || q == 14 || q == 15 || q == 18) ? 1
         : (q == 6 || q == 12 || q == 13 || q == 16 || q == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
// weight class: 0 rest (1/3), 1 axis (1/18), 2 diagonal (1/36)
__host__ __device__ constexpr int wclass(int q) { return q == 0 ? 0 : (q <= 6 ? 1 : 2); }

template <class R> struct Lat;
template <> struct Lat<float> {
    static constexpr float w0 = 1.0f / 3.0f, w1 = 1.0f / 18.0f, w2 = 1.0f / 36.0f;
    static constexpr float cs2 = 1.0f / 3.0f;
};
template <> struct Lat<double> {
    static constexpr double w0 = 1.0 / 3.0, w1 = 1.0 / 18.0, w2 = 1.0 / 36.0;
    static constexpr double cs2 = 1.0 / 3.0;
};
template <class R> __host__ __device__ constexpr R wq(int q) {
    return wclass(q) == 0 ? Lat<R>::w0 : (wclass(q) == 1 ? Lat<R>::w1 : Lat<R>::w2);
}

// dot(float3(C[q]), u) with the zero products dropped.  Dropping x + 0*y only
// changes the sign of an exact zero, which cannot change any value the step
// produces (every use adds it to 1 or squares it).
template <int Q, class R> __device__ __forceinline__ R cdot(R ux, R uy, R uz) {
    R r = R(0);
    bool first = true;
    if (cx(Q) != 0) { r = cx(Q) > 0 ? ux : -ux; first = false; }
    if (cy(Q) != 0) { r = first ? (cy(Q) > 0 ? uy : -uy) : (cy(Q) > 0 ? r + uy : r - uy); first = false; }
    if (cz(Q) != 0) { r = first ? (cz(Q) > 0 ? uz : -uz) : (cz(Q) > 0 ? r + uz : r - uz); }
    return r;
}

// Same for a direction index that is a constant after loop unrolling.
template <class R> __device__ __forceinline__ R cdotq(int q, R ux, R uy, R uz) {
    R r = R(0);
    bool first = true;
    if (cx(q) != 0) { r = cx(q) > 0 ? ux : -ux; first = false; }
    if (cy(q) != 0) { r = first ? (cy(q) > 0 ? uy : -uy) : (cy(q) > 0 ? r + uy : r - uy); first = false; }
    if (cz(q) != 0) { r = first ? (cz(q) > 0 ? uz : -uz) : (cz(q) > 0 ? r + uz : r - uz); }
    return r;
}
template <class R> __device__ __forceinline__ R feqq(int q, R rho, R ux, R uy, R uz, R u2) {
    R cu = cdotq<R>(q, ux, uy, uz);
    return wq<R>(q) * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * u2);
}

// equilibrium(q, rho, u) = W[q]*rho*(1 + 3cu + 4.5cu^2 - 1.5u^2)  (BF.metal:478-484)
template <int Q, class R> __device__ __forceinline__ R feq(R rho, R ux, R uy, R uz, R u2) {
    R cu = cdot<Q, R>(ux, uy, uz);
    return wq<R>(Q) * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * u2);
}
// Runtime-direction variant for the sparse boundary kernels.
template <class R> __device__ __forceinline__ R feq_rt(int q, R rho, R ux, R uy, R uz) {
    R cu = R(cx(q)) * ux + R(cy(q)) * uy + R(cz(q)) * uz;
    R u2 = ux * ux + uy * uy + uz * uz;
    R w = wclass(q) == 0 ? Lat<R>::w0 : (wclass(q) == 1 ? Lat<R>::w1 : Lat<R>::w2);
    return w * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * u2);
}

// ---------------------------------------------------------------------------
// Storage formats.  Compute type R is float except for the FP64 run.
// Deviation formats store f - w_q (the equilibrium at rest), halving the bytes
// per cell; FP16 additionally scales by 2^12 to keep small deviations normal.
// ---------------------------------------------------------------------------
//
// Stochastic rounding (BF16).  bfloat16 keeps 8 significant bits of f - w_q, so
// a fluid update smaller than half a unit in the last place of the stored
// deviation (a slowly decaying low-amplitude flow changes by ~1e-4 of itself
// per step) is lost every step under round-to-nearest and the flow freezes.
// The BF16 fluid stores therefore round up with probability equal to the
// discarded fraction: 16 pseudo-random bits are added to the FP32 bit pattern
// below the kept bits before truncation, an unbiased rounding whose expected
// value is the FP32 result.  The bits come from a hash of (cell, step) advanced
// by the Numerical Recipes linear congruential step per direction, so a run is
// reproducible bit for bit and independent of how steps are batched.
__device__ __forceinline__ uint32_t sr_seed(uint32_t cell, uint32_t step) {
    uint32_t h = cell * 0x9E3779B1u + step * 0x85EBCA77u;  // golden-ratio and Murmur3-finaliser odd constants
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    return h;
}
__device__ __forceinline__ uint32_t sr_next(uint32_t x) { return x * 1664525u + 1013904223u; }
__device__ __forceinline__ __nv_bfloat16 bf16_stochastic(float v, uint32_t x) {
    // the high half of the LCG state: its low bits are the weak ones
    const uint32_t b = __float_as_uint(v) + (x >> 16);
    return __ushort_as_bfloat16((unsigned short)(b >> 16));
}

struct StoreF32 {
    using T = float;
    using R = float;
    static constexpr bool kStochastic = false;
    template <int Q> __device__ __forceinline__ static R ld(const T* p) { return *p; }
    template <int Q> __device__ __forceinline__ static void st(T* p, R v) { *p = v; }
    __device__ __forceinline__ static R ld_rt(const T* p, int) { return *p; }
    __device__ __forceinline__ static void st_rt(T* p, int, R v) { *p = v; }
    __device__ __forceinline__ static void st_rt_sr(T* p, int, R v, uint32_t) { *p = v; }
};
struct StoreF64 {
    using T = double;
    using R = double;
    static constexpr bool kStochastic = false;
    template <int Q> __device__ __forceinline__ static R ld(const T* p) { return *p; }
    template <int Q> __device__ __forceinline__ static void st(T* p, R v) { *p = v; }
    __device__ __forceinline__ static R ld_rt(const T* p, int) { return *p; }
    __device__ __forceinline__ static void st_rt(T* p, int, R v) { *p = v; }
    __device__ __forceinline__ static void st_rt_sr(T* p, int, R v, uint32_t) { *p = v; }
};
constexpr float kF16Scale = 4096.0f;
constexpr float kF16InvScale = 1.0f / 4096.0f;
// The 16-bit conversions use explicit fused multiply-adds: they are not part of
// the FP32 parity contract, and one FMA per conversion keeps the 16-bit step
// from becoming instruction-bound.
struct StoreF16Dev {
    using T = __half;
    using R = float;
    template <int Q> __device__ __forceinline__ static R ld(const T* p) {
        return __fmaf_rn(__half2float(*p), kF16InvScale, wq<float>(Q));
    }
    template <int Q> __device__ __forceinline__ static void st(T* p, R v) {
        *p = __float2half_rn(__fmaf_rn(v, kF16Scale, -wq<float>(Q) * kF16Scale));
    }
    __device__ __forceinline__ static R ld_rt(const T* p, int q) {
        return __fmaf_rn(__half2float(*p), kF16InvScale,
                         q == 0 ? Lat<float>::w0 : (q <= 6 ? Lat<float>::w1 : Lat<float>::w2));
    }
    __device__ __forceinline__ static void st_rt(T* p, int q, R v) {
        float w = q == 0 ? Lat<float>::w0 : (q <= 6 ? Lat<float>::w1 : Lat<float>::w2);
        *p = __float2half_rn(__fmaf_rn(v, kF16Scale, -w * kF16Scale));
    }
    __device__ __forceinline__ static void st_rt_sr(T* p, int q, R v, uint32_t) { st_rt(p, q, v); }
    // the stored value itself: the deviation f - w_q scaled by kDevScale
    static constexpr float kDevScale = kF16Scale;
    static constexpr bool kStochastic = false;
    __device__ __forceinline__ static float ld_dev(const T* p) { return __half2float(*p); }
    __device__ __forceinline__ static void st_dev(T* p, float v) { *p = __float2half_rn(v); }
    __device__ __forceinline__ static void st_dev_sr(T* p, float v, uint32_t) { *p = __float2half_rn(v); }
};
struct StoreBF16Dev {
    using T = __nv_bfloat16;
    using R = float;
    template <int Q> __device__ __forceinline__ static R ld(const T* p) {
        return __bfloat162float(*p) + wq<float>(Q);
    }
    template <int Q> __device__ __forceinline__ static void st(T* p, R v) {
        *p = __float2bfloat16_rn(v - wq<float>(Q));
    }
    __device__ __forceinline__ static R ld_rt(const T* p, int q) {
        return __bfloat162float(*p) + (q == 0 ? Lat<float>::w0 : (q <= 6 ? Lat<float>::w1 : Lat<float>::w2));
    }
    __device__ __forceinline__ static void st_rt(T* p, int q, R v) {
        float w = q == 0 ? Lat<float>::w0 : (q <= 6 ? Lat<float>::w1 : Lat<float>::w2);
        *p = __float2bfloat16_rn(v - w);
    }
    // fluid updates: stochastic rounding with the LCG state x (see sr_seed)
    __device__ __forceinline__ static void st_rt_sr(T* p, int q, R v, uint32_t x) {
        float w = q == 0 ? Lat<float>::w0 : (q <= 6 ? Lat<float>::w1 : Lat<float>::w2);
        *p = bf16_stochastic(v - w, x);
    }
    static constexpr float kDevScale = 1.0f;
    static constexpr bool kStochastic = true;
    __device__ __forceinline__ static float ld_dev(const T* p) { return __bfloat162float(*p); }
    __device__ __forceinline__ static void st_dev(T* p, float v) { *p = __float2bfloat16_rn(v); }
    __device__ __forceinline__ static void st_dev_sr(T* p, float v, uint32_t x) { *p = bf16_stochastic(v, x); }
};

// ---------------------------------------------------------------------------
// Grid geometry and the in-place AA addressing.
//
// The canonical state after a step is the post-collision field f*_q(x).  It is
// stored in one of two representations that alternate every step:
//   rep E (after an even number of steps): f*_q(x) at slot opp(q) of cell x;
//   rep S (after an odd number):          f*_q(x) at slot q of cell x + c_q.
// A step that starts from rep E pulls f_q(x) = A[opp q][x - c_q] and pushes
// its result to A[q][x + c_q]; a step from rep S reads A[q][x] and writes
// A[opp q][x].  Each cell reads and writes the same 19 slots, so the update is
// race-free in place.
//
// The population array carries a one-cell halo around the lattice (padded
// extent (px, ny+2, nz+2), the row pitch px = nx + 2 rounded up to 8 cells so
// every row starts on a 16-byte boundary; columns past nx + 1 are unused).  Values pushed across a face land in the halo,
// and a small fill kernel writes the values the boundary cells will pull
// (periodic copies, face rules) before each step, so the fused kernel uses the
// same uniform addressing for every real cell.  Masks, wall velocities and
// captured fields stay unpadded.
// ---------------------------------------------------------------------------
struct Grid {
    int nx, ny, nz;
    int per_x, per_y, per_z;  // periodic axes
    int64_t n;                // real cells
    int64_t nxy;
    int px, py, pz;           // padded extent (px: row pitch, at least nx + 2)
    int64_t pxy, pn;          // padded plane and total
};

// Cell counts are limited to 2^32 - 1 (GridSize, SimulationConfiguration.swift:32-44),
// so 32-bit division suffices.
__device__ __forceinline__ void unflat(const Grid& g, int64_t gid, int& x, int& y, int& z) {
    uint32_t id = (uint32_t)gid;
    uint32_t nxy = (uint32_t)g.nxy;
    uint32_t zz = id / nxy;
    uint32_t r = id - zz * nxy;
    uint32_t yy = r / (uint32_t)g.nx;
    z = (int)zz;
    y = (int)yy;
    x = (int)(r - yy * (uint32_t)g.nx);
}
__device__ __forceinline__ int64_t flat(const Grid& g, int x, int y, int z) {
    return (int64_t)x + (int64_t)g.nx * ((int64_t)y + (int64_t)g.ny * z);
}
// Padded index of (x, y, z), valid for -1 <= x <= nx (and likewise y, z).
__device__ __forceinline__ int64_t pflat(const Grid& g, int x, int y, int z) {
    return (int64_t)(x + 1) + (int64_t)g.px * ((int64_t)(y + 1) + (int64_t)g.py * (z + 1));
}
__device__ __forceinline__ bool inside(const Grid& g, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < g.nx && y < g.ny && z < g.nz;
}
// Wraps periodic axes; returns false if the point is still outside.
__device__ __forceinline__ bool wrap(const Grid& g, int& x, int& y, int& z) {
    if (g.per_x) x = x < 0 ? g.nx - 1 : (x >= g.nx ? 0 : x);
    if (g.per_y) y = y < 0 ? g.ny - 1 : (y >= g.ny ? 0 : y);
    if (g.per_z) z = z < 0 ? g.nz - 1 : (z >= g.nz ? 0 : z);
    return inside(g, x, y, z);
}

// Face of the first out-of-range axis (x, then y, then z): 0..5 = -x,+x,-y,+y,-z,+z.
__device__ __forceinline__ int exit_face(const Grid& g, int x, int y, int z) {
    if (x < 0) return 0;
    if (x >= g.nx) return 1;
    if (y < 0) return 2;
    if (y >= g.ny) return 3;
    return z < 0 ? 4 : 5;
}

// Canonical accessor f*_q(x) of a real cell in the current representation.
template <class S>
__device__ __forceinline__ typename S::R canon_load(const typename S::T* A, const Grid& g, int rep_s, int q, int x,
                                                    int y, int z) {
    if (!rep_s) return S::ld_rt(A + (int64_t)opp(q) * g.pn + pflat(g, x, y, z), opp(q));
    return S::ld_rt(A + (int64_t)q * g.pn + pflat(g, x + cx(q), y + cy(q), z + cz(q)), q);
}
template <class S>
__device__ __forceinline__ void canon_store(typename S::T* A, const Grid& g, int rep_s, int q, int x, int y, int z,
                                            typename S::R v) {
    if (!rep_s) S::st_rt(A + (int64_t)opp(q) * g.pn + pflat(g, x, y, z), opp(q), v);
    else S::st_rt(A + (int64_t)q * g.pn + pflat(g, x + cx(q), y + cy(q), z + cz(q)), q, v);
}
// Slot that real cell (x,y,z) reads as its incoming direction q in the NEXT
// step: rep E pulls A[opp q][x - c_q] (possibly a halo cell), rep S reads A[q][x].
template <class S>
__device__ __forceinline__ typename S::T* incoming_slot(typename S::T* A, const Grid& g, int rep_s, int q, int x,
                                                        int y, int z, int& slot_dir) {
    if (rep_s) {
        slot_dir = q;
        return A + (int64_t)q * g.pn + pflat(g, x, y, z);
    }
    slot_dir = opp(q);
    return A + (int64_t)opp(q) * g.pn + pflat(g, x - cx(q), y - cy(q), z - cz(q));
}

// Cell t of the halo shell of the padded array (the -z / +z planes, then the
// -y / +y rows, then the -x / +x columns), in padded coordinates.
__device__ __forceinline__ bool padded_shell_cell(const Grid& g, int64_t t, int& x, int& y, int& z) {
    const int64_t fz = (int64_t)g.px * g.py;
    if (t < 2 * fz) {
        z = t < fz ? 0 : g.pz - 1;
        const int64_t r = t < fz ? t : t - fz;
        y = (int)(r / g.px);
        x = (int)(r - (int64_t)y * g.px);
        return true;
    }
    t -= 2 * fz;
    const int64_t fy = (int64_t)g.px * (g.pz - 2);
    if (t < 2 * fy) {
        y = t < fy ? 0 : g.py - 1;
        const int64_t r = t < fy ? t : t - fy;
        z = 1 + (int)(r / g.px);
        x = (int)(r - (int64_t)(z - 1) * g.px);
        return true;
    }
    t -= 2 * fy;
    const int64_t fx = (int64_t)(g.py - 2) * (g.pz - 2);
    if (t < 2 * fx) {
        x = t < fx ? 0 : g.nx + 1;
        const int64_t r = t < fx ? t : t - fx;
        z = 1 + (int)(r / (g.py - 2));
        y = 1 + (int)(r - (int64_t)(z - 1) * (g.py - 2));
        return true;
    }
    return false;
}

// Mask byte: bits 0-5 part id (0 = fluid), bit 6 newly uncovered, bit 7 newly covered.
constexpr uint8_t kPartMask = 0x3F;
constexpr uint8_t kUncovered = 0x40;
constexpr uint8_t kCovered = 0x80;

}  // namespace bfx
