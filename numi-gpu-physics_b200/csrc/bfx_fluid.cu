// Fused D3Q19 stream + collide on the in-place AA population layout.
//
// One thread per cell, one launch per step.  The kernel restates the fluid,
// solid and newly-uncovered branches of the reference's stepFluidTRT
// (Sources/BirdFlowMetal/Metal/BirdFlow.metal:2507-3236) in the same FP32
// operation order; moving-wall bounce-back and the body loads are applied
// before this kernel by the link kernels (bfx_geometry.cu), which write the
// reconstructed populations into the slots this kernel reads.  That keeps the
// bulk of the lattice branch-free: interior cells load 19 values, collide and
// store 19 values (152 B per cell in FP32, 76 B in the 16-bit formats).
#include "bfx_device.cuh"
#include "bfx_internal.h"

namespace bfx {

struct BulkArgs {
    void* pops;
    void* spill;
    const void* ghost;
    const uint8_t* mask;
    const float4* wall;
    float* density;
    float4* velocity;
    DeviceState* state;
    Grid g;
    Spill sp;
    Spill gh;
    FluidParams fp;
    int capture;
};

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

// Value pulled from outside the lattice through face f (see bfx.h bfx_face_bc).
template <class S>
__device__ __forceinline__ typename S::R face_value(const BulkArgs& a, int f, int q, int x, int y, int z) {
    using R = typename S::R;
    const FluidParams& fp = a.fp;
    int bc = fp.face_bc[f];
    if (bc == BFX_BC_OUTFLOW) {
        const typename S::T* gh = (const typename S::T*)a.ghost;
        return S::ld_rt(gh + a.gh.off[f] + face_index(a.g, f, x, y, z) * 5 + face_slot(f ^ 1, q), q);
    }
    float ux = fp.far[0], uy = fp.far[1], uz = fp.far[2];
    if (bc == BFX_BC_VELOCITY) {
        ux = fp.face_u[f][0];
        uy = fp.face_u[f][1];
        uz = fp.face_u[f][2];
    }
    return feq_rt<R>(q, (R)fp.far[3], (R)ux, (R)uy, (R)uz);
}

template <class R, int COLL>
__device__ __forceinline__ void collide(const R (&f)[19], R rho, R ux, R uy, R uz, R omega_p, R omega_m,
                                        R (&post)[19], float& activation, float& restriction) {
    const R cs2 = Lat<R>::cs2;
    R u2 = ux * ux + uy * uy + uz * uz;
    R feqv[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) feqv[q] = feqq<R>(q, rho, ux, uy, uz, u2);

    if (COLL == BFX_COLLISION_REGULARIZED || COLL == BFX_COLLISION_RR3) {
        // BF.metal:2917-3062
        R dsx = 0, dsy = 0, dsz = 0, odx = 0, ody = 0, odz = 0;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const R dx = (R)cx(q), dy = (R)cy(q), dz = (R)cz(q);
            R ne = f[q] - feqv[q];
            dsx += ne * (dx * dx - cs2);
            dsy += ne * (dy * dy - cs2);
            dsz += ne * (dz * dz - cs2);
            odx += ne * (dx * dy);
            ody += ne * (dx * dz);
            odz += ne * (dy * dz);
        }
        R aXxy = R(2) * ux * odx + uy * dsx;
        R aXxz = R(2) * ux * ody + uz * dsx;
        R aXyy = ux * dsy + R(2) * uy * odx;
        R aXzz = ux * dsz + R(2) * uz * ody;
        R aYyz = R(2) * uy * odz + uz * dsy;
        R aYzz = uy * dsz + R(2) * uz * odz;
        R unb[19];
        R scale = R(1);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const R dx = (R)cx(q), dy = (R)cy(q), dz = (R)cz(q);
            R hx = dx * dx - cs2, hy = dy * dy - cs2, hz = dz * dz - cs2;
            R contraction = (hx * dsx + hy * dsy + hz * dsz) + R(2) * ((dx * dy) * odx + (dx * dz) * ody + (dy * dz) * odz);
            R third = 0;
            if (COLL == BFX_COLLISION_RR3) {
                third = dy * (dx * dx - cs2) * aXxy + dz * (dx * dx - cs2) * aXxz + dx * (dy * dy - cs2) * aXyy +
                        dx * (dz * dz - cs2) * aXzz + dz * (dy * dy - cs2) * aYyz + dy * (dz * dz - cs2) * aYzz;
            }
            R rne = wq<R>(q) * R(4.5) * contraction;
            if (COLL == BFX_COLLISION_RR3) rne += wq<R>(q) * R(13.5) * third;
            R cand = feqv[q] + (R(1) - omega_p) * rne;
            unb[q] = cand;
            R fl = R(1.0e-6) * (feqv[q] > R(0) ? feqv[q] : R(0));
            R floor_ = R(1.0e-12) > fl ? R(1.0e-12) : fl;
            if (cand < floor_) {
                R den = feqv[q] - cand;
                den = den > R(1.0e-30) ? den : R(1.0e-30);
                R adm = (feqv[q] - floor_) / den;
                adm = adm < R(0) ? R(0) : (adm > R(1) ? R(1) : adm);
                scale = scale < adm ? scale : adm;
            }
        }
        if (scale < R(1)) {
            activation = 1.0f;
            restriction = (float)(R(1) - scale);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) post[q] = feqv[q] + scale * (unb[q] - feqv[q]);
    } else if (COLL == BFX_COLLISION_TRT) {
        // BF.metal:3063-3093
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int qo = opp(q);
            R fp_ = R(0.5) * (f[q] + f[qo]);
            R fm = R(0.5) * (f[q] - f[qo]);
            R ep = R(0.5) * (feqv[q] + feqv[qo]);
            R em = R(0.5) * (feqv[q] - feqv[qo]);
            post[q] = f[q] - omega_p * (fp_ - ep) - omega_m * (fm - em);
        }
    } else {
        // symmetric positivity limiter: BF.metal:3094-3174
        R si[19], ai[19];
        R sscale = R(1);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int qo = opp(q);
            R fp_ = R(0.5) * (f[q] + f[qo]);
            R fm = R(0.5) * (f[q] - f[qo]);
            R ep = R(0.5) * (feqv[q] + feqv[qo]);
            R em = R(0.5) * (feqv[q] - feqv[qo]);
            R sv = -omega_p * (fp_ - ep);
            R av = -omega_m * (fm - em);
            si[q] = sv;
            ai[q] = av;
            if (sv < R(0)) {
                R base = f[q] + av;
                R fl = R(1.0e-6) * (feqv[q] > R(0) ? feqv[q] : R(0));
                R floor_ = R(1.0e-12) > fl ? R(1.0e-12) : fl;
                if (base + sv < floor_) {
                    R den = -sv > R(1.0e-30) ? -sv : R(1.0e-30);
                    R cand = (base - floor_) / den;
                    cand = cand < R(0) ? R(0) : (cand > R(1) ? R(1) : cand);
                    sscale = sscale < cand ? sscale : cand;
                }
            }
        }
        if (sscale < R(1)) {
            activation = 1.0f;
            restriction = (float)(R(1) - sscale);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (sscale < R(1)) {
                post[q] = f[q] + sscale * si[q] + ai[q];
            } else {
                const int qo = opp(q);
                R fp_ = R(0.5) * (f[q] + f[qo]);
                R fm = R(0.5) * (f[q] - f[qo]);
                R ep = R(0.5) * (feqv[q] + feqv[qo]);
                R em = R(0.5) * (feqv[q] - feqv[qo]);
                post[q] = f[q] - omega_p * (fp_ - ep) - omega_m * (fm - em);
            }
        }
    }
}

template <class S, int REP_S>
__device__ __forceinline__ void store_post(const BulkArgs& a, typename S::T* A, int64_t gid, int x, int y, int z,
                                           bool boundary, const typename S::R (&post)[19]) {
    const Grid& g = a.g;
    if (REP_S) {
#pragma unroll
        for (int q = 0; q < 19; ++q) S::st_rt(A + (int64_t)opp(q) * g.n + gid, opp(q), post[q]);
        return;
    }
    if (!boundary) {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int64_t off = (int64_t)cx(q) + (int64_t)g.nx * cy(q) + g.nxy * cz(q);
            S::st_rt(A + (int64_t)q * g.n + gid + off, q, post[q]);
        }
        return;
    }
    typename S::T* spill = (typename S::T*)a.spill;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        int tx = x + cx(q), ty = y + cy(q), tz = z + cz(q);
        if (wrap(g, tx, ty, tz)) {
            S::st_rt(A + (int64_t)q * g.n + flat(g, tx, ty, tz), q, post[q]);
        } else {
            int f = exit_face(g, tx, ty, tz);
            S::st_rt(spill + a.sp.off[f] + face_index(g, f, x, y, z) * 5 + face_slot(f, q), q, post[q]);
        }
    }
}

template <class S, int REP_S, int COLL>
__global__ void __launch_bounds__(256) k_bulk(const BulkArgs a) {
    using T = typename S::T;
    using R = typename S::R;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const int64_t gid = (int64_t)x + (int64_t)g.nx * ((int64_t)y + (int64_t)g.ny * z);
    T* A = (T*)a.pops;
    const uint8_t m = a.mask ? a.mask[gid] : (uint8_t)0;
    const bool boundary = x == 0 || y == 0 || z == 0 || x == g.nx - 1 || y == g.ny - 1 || z == g.nz - 1;
    R post[19];

    if (m & kPartMask) {
        // Solid: moving-wall equilibrium eq(1, u_wall) (BF.metal:2557-2570).
        const float4 w = a.wall[gid];
        const R ux = w.x, uy = w.y, uz = w.z;
        const R u2 = ux * ux + uy * uy + uz * uz;
#pragma unroll
        for (int q = 0; q < 19; ++q) post[q] = feqq<R>(q, R(1), ux, uy, uz, u2);
        store_post<S, REP_S>(a, A, gid, x, y, z, boundary, post);
        if (a.capture) {
            a.density[gid] = 1.0f;
            a.velocity[gid] = make_float4(w.x, w.y, w.z, 0.0f);
        }
        return;
    }

    R f[19];
    if (m & kUncovered) {
        // Newly uncovered: refill from the local moving-wall state (BF.metal:2610-2625).
        const float4 w = a.wall[gid];
        const R ux = w.x, uy = w.y, uz = w.z;
        const R u2 = ux * ux + uy * uy + uz * uz;
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = feqq<R>(q, R(1), ux, uy, uz, u2);
    } else if (!boundary) {
        if (REP_S) {
#pragma unroll
            for (int q = 0; q < 19; ++q) f[q] = S::ld_rt(A + (int64_t)q * g.n + gid, q);
        } else {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const int64_t off = (int64_t)cx(q) + (int64_t)g.nx * cy(q) + g.nxy * cz(q);
                f[q] = S::ld_rt(A + (int64_t)opp(q) * g.n + gid - off, opp(q));
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
            if (wrap(g, sx, sy, sz)) {
                f[q] = REP_S ? S::ld_rt(A + (int64_t)q * g.n + gid, q)
                             : S::ld_rt(A + (int64_t)opp(q) * g.n + flat(g, sx, sy, sz), opp(q));
            } else {
                f[q] = face_value<S>(a, exit_face(g, sx, sy, sz), q, x, y, z);
            }
        }
    }

    // Moments in the reference order (rho over q = 0..18, momentum componentwise).
    R rho = 0, mx = 0, my = 0, mz = 0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        rho += f[q];
        if (cx(q) > 0) mx += f[q];
        if (cx(q) < 0) mx -= f[q];
        if (cy(q) > 0) my += f[q];
        if (cy(q) < 0) my -= f[q];
        if (cz(q) > 0) mz += f[q];
        if (cz(q) < 0) mz -= f[q];
    }
    rho = rho > R(1.0e-8) ? rho : R(1.0e-8);
    const R ux = mx / rho, uy = my / rho, uz = mz / rho;
    float activation = 0.0f, restriction = 0.0f;
    collide<R, COLL>(f, rho, ux, uy, uz, (R)a.fp.omega_p, (R)a.fp.omega_m, post, activation, restriction);

    if (a.fp.has_sponge) {
        const float sp = sponge_factor(g, a.fp, x, y, z);
        if (sp > 0.0f) {
            const R fx = a.fp.far[0], fy = a.fp.far[1], fz = a.fp.far[2];
            const R fu2 = fx * fx + fy * fy + fz * fz;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const R farv = feqq<R>(q, (R)a.fp.far[3], fx, fy, fz, fu2);
                post[q] = post[q] + (farv - post[q]) * (R)sp;
            }
        }
    }
    store_post<S, REP_S>(a, A, gid, x, y, z, boundary, post);

    if (a.capture) {
        R cd = 0, cmx = 0, cmy = 0, cmz = 0;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            cd += post[q];
            if (cx(q) > 0) cmx += post[q];
            if (cx(q) < 0) cmx -= post[q];
            if (cy(q) > 0) cmy += post[q];
            if (cy(q) < 0) cmy -= post[q];
            if (cz(q) > 0) cmz += post[q];
            if (cz(q) < 0) cmz -= post[q];
        }
        cd = cd > R(1.0e-8) ? cd : R(1.0e-8);
        a.density[gid] = (float)cd;
        a.velocity[gid] = make_float4((float)(cmx / cd), (float)(cmy / cd), (float)(cmz / cd), 0.0f);
    }
    if (COLL != BFX_COLLISION_TRT && activation != 0.0f) {
        atomicAdd(&a.state->limiter_count, 1.0);
        atomicMax(&a.state->limiter_max_bits, __float_as_uint(restriction));
    }
}

// ---------------------------------------------------------------------------
// Zero-gradient outflow: ghost value for (face cell, inward direction q) is
// the population the interior neighbour receives, f*_q(x - n - c_q).
// ---------------------------------------------------------------------------
template <class S>
__global__ void k_ghost(const BulkArgs a, int rep_s, int f) {
    using T = typename S::T;
    const Grid& g = a.g;
    const int axis = f >> 1;
    const int hi = f & 1;
    const int du = axis == 0 ? g.ny : g.nx;
    const int dv = axis == 2 ? g.ny : g.nz;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    if (u >= du || v >= dv) return;
    int x, y, z;
    if (axis == 0) { x = hi ? g.nx - 1 : 0; y = u; z = v; }
    else if (axis == 1) { y = hi ? g.ny - 1 : 0; x = u; z = v; }
    else { z = hi ? g.nz - 1 : 0; x = u; y = v; }
    const int nxo = axis == 0 ? (hi ? 1 : -1) : 0;
    const int nyo = axis == 1 ? (hi ? 1 : -1) : 0;
    const int nzo = axis == 2 ? (hi ? 1 : -1) : 0;
    const T* A = (const T*)a.pops;
    const T* spill = (const T*)a.spill;
    T* gh = (T*)a.ghost;
    for (int q = 1; q < 19; ++q) {
        const int c = axis == 0 ? cx(q) : (axis == 1 ? cy(q) : cz(q));
        if (c != (hi ? -1 : 1)) continue;  // inward through this face
        int tx = x - nxo - cx(q), ty = y - nyo - cy(q), tz = z - nzo - cz(q);
        typename S::R val;
        bool ok = wrap(g, tx, ty, tz);
        if (ok && (a.mask == nullptr || (a.mask[flat(g, tx, ty, tz)] & kPartMask) == 0)) {
            val = canon_load<S>(A, g, a.sp, spill, rep_s, q, tx, ty, tz);
        } else {
            val = (typename S::R)feq_rt<float>(q, a.fp.far[3], a.fp.far[0], a.fp.far[1], a.fp.far[2]);
        }
        S::st_rt(gh + a.gh.off[f] + face_index(g, f, x, y, z) * 5 + face_slot(f ^ 1, q), q, val);
    }
}

// ---------------------------------------------------------------------------
// Initialisation (rep E), canonical read-out / write-in, macroscopic fields.
// ---------------------------------------------------------------------------
template <class S>
__global__ void k_init(const BulkArgs a, int kind, float amplitude) {
    using R = typename S::R;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const int64_t gid = flat(g, x, y, z);
    float u[3];
    if (kind == BFX_INIT_SHEAR_WAVE_Y || kind == BFX_INIT_SHEAR_WAVE_Z) {
        // initializeShearWave: BF.metal:2132-2162
        int coord = kind == BFX_INIT_SHEAR_WAVE_Z ? z : y;
        int extent = kind == BFX_INIT_SHEAR_WAVE_Z ? g.nz : g.ny;
        float phase = 2.0f * 3.14159265358979323846f * (float)coord / (float)extent;
        u[0] = amplitude * bfx_sinf(phase);
        u[1] = 0.0f;
        u[2] = 0.0f;
    } else if (a.mask && (a.mask[gid] & kPartMask)) {
        const float4 w = a.wall[gid];
        u[0] = w.x;
        u[1] = w.y;
        u[2] = w.z;
    } else {
        u[0] = a.fp.far[0];
        u[1] = a.fp.far[1];
        u[2] = a.fp.far[2];
    }
    typename S::T* A = (typename S::T*)a.pops;
    for (int q = 0; q < 19; ++q) {
        float v = feq_rt<float>(q, 1.0f, u[0], u[1], u[2]);
        S::st_rt(A + (int64_t)opp(q) * g.n + gid, opp(q), (R)v);
    }
    if (a.density) {
        a.density[gid] = 1.0f;
        a.velocity[gid] = make_float4(u[0], u[1], u[2], 0.0f);
    }
}

template <class S>
__global__ void k_readout(const BulkArgs a, int rep_s, float* out) {
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const int64_t gid = flat(g, x, y, z);
    for (int q = 0; q < 19; ++q)
        out[(int64_t)q * g.n + gid] =
            (float)canon_load<S>((const typename S::T*)a.pops, g, a.sp, (const typename S::T*)a.spill, rep_s, q, x, y, z);
}

template <class S>
__global__ void k_writein(const BulkArgs a, int rep_s, const float* in) {
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const int64_t gid = flat(g, x, y, z);
    for (int q = 0; q < 19; ++q)
        canon_store<S>((typename S::T*)a.pops, g, a.sp, (typename S::T*)a.spill, rep_s, q, x, y, z,
                       (typename S::R)in[(int64_t)q * g.n + gid]);
}

// extractMacroscopicFields: BF.metal:2107-2127
template <class S>
__global__ void k_macroscopic(const BulkArgs a, int rep_s) {
    using R = typename S::R;
    const Grid& g = a.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const int64_t gid = flat(g, x, y, z);
    R rho = 0, mx = 0, my = 0, mz = 0;
    for (int q = 0; q < 19; ++q) {
        R v = canon_load<S>((const typename S::T*)a.pops, g, a.sp, (const typename S::T*)a.spill, rep_s, q, x, y, z);
        rho += v;
        mx += v * (R)cx(q);
        my += v * (R)cy(q);
        mz += v * (R)cz(q);
    }
    rho = rho > R(1.0e-8) ? rho : R(1.0e-8);
    a.density[gid] = (float)rho;
    a.velocity[gid] = make_float4((float)(mx / rho), (float)(my / rho), (float)(mz / rho), 0.0f);
}

// FP64 mass and momentum of fluid cells: fixed-order block tree, then one
// single-block pass over the partials (deterministic).
template <class S>
__global__ void __launch_bounds__(256) k_mass_momentum(const BulkArgs a, int rep_s, double* partials) {
    __shared__ double sh[4][256];
    const Grid& g = a.g;
    double acc[4] = {0, 0, 0, 0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < g.n; gid += stride) {
        if (a.mask && (a.mask[gid] & kPartMask)) continue;
        int x, y, z;
        unflat(g, gid, x, y, z);
        for (int q = 0; q < 19; ++q) {
            double v = (double)canon_load<S>((const typename S::T*)a.pops, g, a.sp, (const typename S::T*)a.spill,
                                             rep_s, q, x, y, z);
            acc[0] += v;
            acc[1] += v * cx(q);
            acc[2] += v * cy(q);
            acc[3] += v * cz(q);
        }
    }
    for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) partials[4 * blockIdx.x + k] = sh[k][0];
}

__global__ void k_sum_partials4(const double* partials, int count, double* out) {
    __shared__ double sh[4][256];
    double acc[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < count; i += blockDim.x)
        for (int k = 0; k < 4; ++k) acc[k] += partials[4 * i + k];
    for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) out[k] = sh[k][0];
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static BulkArgs make_args(const GridDesc& gd, const FluidParams& fp, const FluidBuffers& b, int capture) {
    BulkArgs a;
    a.pops = b.pops;
    a.spill = b.spill;
    a.ghost = b.ghost;
    a.mask = b.mask;
    a.wall = b.wall;
    a.density = b.density;
    a.velocity = b.velocity;
    a.state = b.state;
    a.g.nx = gd.nx;
    a.g.ny = gd.ny;
    a.g.nz = gd.nz;
    a.g.per_x = gd.per_x;
    a.g.per_y = gd.per_y;
    a.g.per_z = gd.per_z;
    a.g.n = gd.n;
    a.g.nxy = gd.nxy;
    for (int f = 0; f < 6; ++f) {
        a.sp.off[f] = gd.spill_off[f];
        a.gh.off[f] = gd.ghost_off[f];
    }
    a.fp = fp;
    a.capture = capture;
    return a;
}

static void cell_launch_shape(const GridDesc& g, dim3& grid, dim3& block) {
    int bx = g.nx >= 128 ? 128 : ((g.nx + 31) / 32) * 32;
    int by = 256 / bx;
    block = dim3(bx, by, 1);
    grid = dim3((g.nx + bx - 1) / bx, (g.ny + by - 1) / by, g.nz);
}

template <class S, int REP, int COLL>
static void bulk_t(const BulkArgs& a, const GridDesc& g, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    k_bulk<S, REP, COLL><<<grid, block, 0, s>>>(a);
}

template <class S>
static void bulk_s(const BulkArgs& a, const GridDesc& g, int collision, int rep_s, cudaStream_t s) {
    switch (collision * 2 + rep_s) {
    case 0: bulk_t<S, 0, BFX_COLLISION_TRT>(a, g, s); break;
    case 1: bulk_t<S, 1, BFX_COLLISION_TRT>(a, g, s); break;
    case 2: bulk_t<S, 0, BFX_COLLISION_TRT_LIMITER>(a, g, s); break;
    case 3: bulk_t<S, 1, BFX_COLLISION_TRT_LIMITER>(a, g, s); break;
    case 4: bulk_t<S, 0, BFX_COLLISION_REGULARIZED>(a, g, s); break;
    case 5: bulk_t<S, 1, BFX_COLLISION_REGULARIZED>(a, g, s); break;
    case 6: bulk_t<S, 0, BFX_COLLISION_RR3>(a, g, s); break;
    default: bulk_t<S, 1, BFX_COLLISION_RR3>(a, g, s); break;
    }
}

#define BFX_DISPATCH_STORAGE(storage, FN, ...)                 \
    switch (storage) {                                         \
    case BFX_STORAGE_F16_DEVIATION: FN<StoreF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_BF16_DEVIATION: FN<StoreBF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_F64: FN<StoreF64>(__VA_ARGS__); break;    \
    default: FN<StoreF32>(__VA_ARGS__); break;                 \
    }

void launch_bulk(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, int capture, cudaStream_t s) {
    BulkArgs a = make_args(g, fp, b, capture);
    BFX_DISPATCH_STORAGE(storage, bulk_s, a, g, collision, rep_s, s);
}

template <class S>
static void ghost_s(const BulkArgs& a, const GridDesc& g, int rep_s, cudaStream_t s) {
    for (int f = 0; f < 6; ++f) {
        if (a.fp.face_bc[f] != BFX_BC_OUTFLOW) continue;
        int axis = f >> 1;
        int du = axis == 0 ? g.ny : g.nx;
        int dv = axis == 2 ? g.ny : g.nz;
        k_ghost<S><<<dim3((du + 127) / 128, dv), 128, 0, s>>>(a, rep_s, f);
    }
}
void launch_ghost(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                  cudaStream_t s) {
    BulkArgs a = make_args(g, fp, b, 0);
    BFX_DISPATCH_STORAGE(storage, ghost_s, a, g, rep_s, s);
}

template <class S>
static void init_s(const BulkArgs& a, const GridDesc& g, int kind, float amplitude, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    k_init<S><<<grid, block, 0, s>>>(a, kind, amplitude);
}
void launch_init(int storage, int init_kind, float amplitude, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, cudaStream_t s) {
    BulkArgs a = make_args(g, fp, b, 0);
    BFX_DISPATCH_STORAGE(storage, init_s, a, g, init_kind, amplitude, s);
}

template <class S>
static void readout_s(const BulkArgs& a, const GridDesc& g, int rep_s, float* out, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    k_readout<S><<<grid, block, 0, s>>>(a, rep_s, out);
}
void launch_readout(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, float* out, cudaStream_t s) {
    FluidParams fp = {};
    BulkArgs a = make_args(g, fp, b, 0);
    BFX_DISPATCH_STORAGE(storage, readout_s, a, g, rep_s, out, s);
}

template <class S>
static void writein_s(const BulkArgs& a, const GridDesc& g, int rep_s, const float* in, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    k_writein<S><<<grid, block, 0, s>>>(a, rep_s, in);
}
void launch_writein(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, const float* in,
                    cudaStream_t s) {
    FluidParams fp = {};
    BulkArgs a = make_args(g, fp, b, 0);
    BFX_DISPATCH_STORAGE(storage, writein_s, a, g, rep_s, in, s);
}

template <class S>
static void macro_s(const BulkArgs& a, const GridDesc& g, int rep_s, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    k_macroscopic<S><<<grid, block, 0, s>>>(a, rep_s);
}
void launch_macroscopic(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, cudaStream_t s) {
    FluidParams fp = {};
    BulkArgs a = make_args(g, fp, b, 0);
    BFX_DISPATCH_STORAGE(storage, macro_s, a, g, rep_s, s);
}

template <class S>
static void mass_s(const BulkArgs& a, int rep_s, double* partials, int blocks, double* result, cudaStream_t s) {
    k_mass_momentum<S><<<blocks, 256, 0, s>>>(a, rep_s, partials);
    k_sum_partials4<<<1, 256, 0, s>>>(partials, blocks, result);
}
void launch_mass_momentum(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, double* partials,
                          int blocks, double* result, cudaStream_t s) {
    FluidParams fp = {};
    BulkArgs a = make_args(g, fp, b, 0);
    BFX_DISPATCH_STORAGE(storage, mass_s, a, rep_s, partials, blocks, result, s);
}

}  // namespace bfx
