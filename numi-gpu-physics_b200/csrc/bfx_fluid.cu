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
    void* plane[19];        // A + q*N: base of direction q's plane
    int32_t doff[19];       // c_q . (1, nx, nx*ny): neighbour offset of direction q
    float far_eq_f[19];     // equilibrium(q, far density, far velocity), FP32
    double far_eq_d[19];    // same in FP64 (FP64 storage)
    int64_t shell_cells;
    int box[3];             // geometry box extent (origin in DeviceState)
    int64_t box_cells;
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

// Collision (BF.metal:2907-3174).  Directions are processed in opposite pairs
// (q odd, q+1 = opp(q)): the equilibrium, TRT and regularized terms of the pair
// share their even parts and negate their odd parts, and in IEEE arithmetic
// -(a-b) == b-a, (-a)*b == -(a*b), x-(-y) == x+y exactly.  Every value is
// therefore bit-identical to evaluating the reference expression once per
// direction, at about half the instruction count.
template <class R, int COLL>
__device__ __forceinline__ void collide(const R (&f)[19], R rho, R ux, R uy, R uz, R omega_p, R omega_m,
                                        R (&post)[19], float& activation, float& restriction) {
    const R cs2 = Lat<R>::cs2;
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R t15 = R(1.5) * u2;
    const R wr0 = Lat<R>::w0 * rho, wr1 = Lat<R>::w1 * rho, wr2 = Lat<R>::w2 * rho;
    R feqv[19];
    feqv[0] = wr0 * (R(1) + R(3) * R(0) + R(4.5) * R(0) * R(0) - t15);
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        // equilibrium(q, rho, u) = W rho (1 + 3cu + 4.5cu^2 - 1.5u^2) for q and opp(q) (cu -> -cu)
        const R cu = cdotq<R>(q, ux, uy, uz);
        const R t3 = R(3) * cu;
        const R t45 = R(4.5) * cu * cu;
        const R wr = q <= 6 ? wr1 : wr2;
        feqv[q] = wr * (R(1) + t3 + t45 - t15);
        feqv[q + 1] = wr * (R(1) - t3 + t45 - t15);
    }

    if (COLL == BFX_COLLISION_REGULARIZED || COLL == BFX_COLLISION_RR3) {
        // Projected second-order non-equilibrium stress; products with a zero
        // lattice coefficient are dropped and +-1 products become sign flips
        // (exact for finite values).
        R dsx = 0, dsy = 0, dsz = 0, odx = 0, ody = 0, odz = 0;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            R ne = f[q] - feqv[q];
            dsx += ne * ((R)(cx(q) * cx(q)) - cs2);
            dsy += ne * ((R)(cy(q) * cy(q)) - cs2);
            dsz += ne * ((R)(cz(q) * cz(q)) - cs2);
            if (cx(q) * cy(q) > 0) odx += ne;
            if (cx(q) * cy(q) < 0) odx -= ne;
            if (cx(q) * cz(q) > 0) ody += ne;
            if (cx(q) * cz(q) < 0) ody -= ne;
            if (cy(q) * cz(q) > 0) odz += ne;
            if (cy(q) * cz(q) < 0) odz -= ne;
        }
        R aXxy = R(2) * ux * odx + uy * dsx;
        R aXxz = R(2) * ux * ody + uz * dsx;
        R aXyy = ux * dsy + R(2) * uy * odx;
        R aXzz = ux * dsz + R(2) * uz * ody;
        R aYyz = R(2) * uy * odz + uz * dsy;
        R aYzz = uy * dsz + R(2) * uz * odz;
        const R one_minus = R(1) - omega_p;
        R scale = R(1);
        auto admit = [&](R fe, R cand) {
            R fl = R(1.0e-6) * (fe > R(0) ? fe : R(0));
            R floor_ = R(1.0e-12) > fl ? R(1.0e-12) : fl;
            if (cand < floor_) {
                R den = fe - cand;
                den = den > R(1.0e-30) ? den : R(1.0e-30);
                R adm = (fe - floor_) / den;
                adm = adm < R(0) ? R(0) : (adm > R(1) ? R(1) : adm);
                scale = scale < adm ? scale : adm;
            }
        };
        {
            // rest direction: contraction = -cs2 (dsx + dsy + dsz), no third-order part
            const R h = -cs2;
            const R contraction = h * dsx + h * dsy + h * dsz;
            const R rne = Lat<R>::w0 * R(4.5) * contraction;
            post[0] = feqv[0] + one_minus * rne;
            admit(feqv[0], post[0]);
        }
#pragma unroll
        for (int q = 1; q < 19; q += 2) {
            // the contraction is even in c (shared by q and opp q), the third-order sum is odd
            const R hx = (R)(cx(q) * cx(q)) - cs2, hy = (R)(cy(q) * cy(q)) - cs2, hz = (R)(cz(q) * cz(q)) - cs2;
            R contraction = hx * dsx + hy * dsy + hz * dsz;
            {
                const int xy = cx(q) * cy(q), xz = cx(q) * cz(q), yz = cy(q) * cz(q);
                if (xy != 0) contraction = contraction + R(2) * (xy > 0 ? odx : -odx);
                else if (xz != 0) contraction = contraction + R(2) * (xz > 0 ? ody : -ody);
                else if (yz != 0) contraction = contraction + R(2) * (yz > 0 ? odz : -odz);
            }
            const R a = wq<R>(q) * R(4.5) * contraction;
            R rq = a, ro = a;
            if (COLL == BFX_COLLISION_RR3) {
                R third = R(0);
                bool any = false;
                auto add = [&](int da, R hb, R amp) {
                    if (da == 0) return;
                    R t = ((R)da * hb) * amp;
                    third = any ? third + t : t;
                    any = true;
                };
                add(cy(q), hx, aXxy);
                add(cz(q), hx, aXxz);
                add(cx(q), hy, aXyy);
                add(cx(q), hz, aXzz);
                add(cz(q), hy, aYyz);
                add(cy(q), hz, aYzz);
                const R b = wq<R>(q) * R(13.5) * third;
                rq = a + b;
                ro = a - b;
            }
            post[q] = feqv[q] + one_minus * rq;
            post[q + 1] = feqv[q + 1] + one_minus * ro;
            admit(feqv[q], post[q]);
            admit(feqv[q + 1], post[q + 1]);
        }
        if (scale < R(1)) {
            activation = 1.0f;
            restriction = (float)(R(1) - scale);
#pragma unroll
            for (int q = 0; q < 19; ++q) post[q] = feqv[q] + scale * (post[q] - feqv[q]);
        } else {
            // scale == 1: feq + 1 * (cand - feq) == cand only up to rounding, so keep
            // the reference expression
#pragma unroll
            for (int q = 0; q < 19; ++q) post[q] = feqv[q] + scale * (post[q] - feqv[q]);
        }
    } else if (COLL == BFX_COLLISION_TRT) {
        // BF.metal:3063-3093, pairwise
        post[0] = f[0] - omega_p * (f[0] - feqv[0]);
#pragma unroll
        for (int q = 1; q < 19; q += 2) {
            const R fp_ = R(0.5) * (f[q] + f[q + 1]);
            const R fm = R(0.5) * (f[q] - f[q + 1]);
            const R ep = R(0.5) * (feqv[q] + feqv[q + 1]);
            const R em = R(0.5) * (feqv[q] - feqv[q + 1]);
            const R A = omega_p * (fp_ - ep);
            const R B = omega_m * (fm - em);
            post[q] = f[q] - A - B;
            post[q + 1] = f[q + 1] - A + B;
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

// Cell of the domain shell (the six faces) with index t: both z faces, then
// both y faces without their z edges, then both x faces without y/z edges.
__device__ __forceinline__ bool shell_cell(const Grid& g, int64_t t, int& x, int& y, int& z) {
    const int64_t fz = (int64_t)g.nx * g.ny;
    if (t < 2 * fz) {
        z = t < fz ? 0 : g.nz - 1;
        const int64_t r = t < fz ? t : t - fz;
        y = (int)(r / g.nx);
        x = (int)(r - (int64_t)y * g.nx);
        return true;
    }
    t -= 2 * fz;
    const int64_t fy = (int64_t)g.nx * (g.nz - 2);
    if (t < 2 * fy) {
        y = t < fy ? 0 : g.ny - 1;
        const int64_t r = t < fy ? t : t - fy;
        z = 1 + (int)(r / g.nx);
        x = (int)(r - (int64_t)(z - 1) * g.nx);
        return true;
    }
    t -= 2 * fy;
    const int64_t fx = (int64_t)(g.ny - 2) * (g.nz - 2);
    if (t < 2 * fx) {
        x = t < fx ? 0 : g.nx - 1;
        const int64_t r = t < fx ? t : t - fx;
        z = 1 + (int)(r / (g.ny - 2));
        y = 1 + (int)(r - (int64_t)(z - 1) * (g.ny - 2));
        return true;
    }
    return false;
}

// Generic cell update, used for the domain shell: periodic wrap, face rules,
// spill planes, solid and uncovered cells.
template <class S, int REP_S, int COLL, int MODE>
__global__ void __launch_bounds__(128) k_bulk_generic(const BulkArgs a) {
    using T = typename S::T;
    using R = typename S::R;
    const Grid& g = a.g;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int x, y, z;
    if (MODE == 0) {
        if (t >= a.shell_cells) return;
        if (!shell_cell(g, t, x, y, z)) return;
    } else {
        // interior cells of the geometry box that are solid or newly uncovered
        if (t >= a.box_cells) return;
        const int lz = (int)(t / ((int64_t)a.box[0] * a.box[1]));
        const int64_t r = t - (int64_t)lz * a.box[0] * a.box[1];
        const int ly = (int)(r / a.box[0]);
        const int lx = (int)(r - (int64_t)ly * a.box[0]);
        x = a.state->box_origin[0] + lx;
        y = a.state->box_origin[1] + ly;
        z = a.state->box_origin[2] + lz;
        if (x < 1 || y < 1 || z < 1 || x >= g.nx - 1 || y >= g.ny - 1 || z >= g.nz - 1) return;
        if (a.mask[(int64_t)x + (int64_t)g.nx * ((int64_t)y + (int64_t)g.ny * z)] == 0) return;
    }
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
// Interior cells: one fluid path with no domain-face logic.  Directions are
// addressed through per-direction plane pointers and 32-bit neighbour offsets
// held in the kernel parameters; solid and newly uncovered cells (rare) take a
// separate non-inlined path so the hot instruction stream stays short.
// ---------------------------------------------------------------------------
template <class S, int REP_S>
__device__ __forceinline__ void store_interior(const BulkArgs& a, uint32_t gid, const typename S::R (&post)[19]) {
    using T = typename S::T;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (REP_S) S::st_rt((T*)a.plane[opp(q)] + gid, opp(q), post[q]);
        else S::st_rt((T*)a.plane[q] + (uint32_t)(gid + (uint32_t)a.doff[q]), q, post[q]);
    }
}

template <class S, int COLL, int CAPTURE>
__device__ __forceinline__ void finish_interior(const BulkArgs& a, uint32_t gid, int x, int y, int z,
                                                typename S::R (&post)[19], float activation, float restriction) {
    using R = typename S::R;
    if (a.fp.has_sponge) {
        const float sp = sponge_factor(a.g, a.fp, x, y, z);
        if (sp > 0.0f) {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const R farv = sizeof(R) == 8 ? (R)a.far_eq_d[q] : (R)a.far_eq_f[q];
                post[q] = post[q] + (farv - post[q]) * (R)sp;
            }
        }
    }
    if (CAPTURE) {
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

template <class S, int REP_S, int COLL, int CAPTURE>
__global__ void __launch_bounds__(256, sizeof(typename S::R) == 8 ? 1 : (COLL == BFX_COLLISION_TRT ? 4 : 2))
    k_bulk_interior(const BulkArgs a) {
    using T = typename S::T;
    using R = typename S::R;
    const int x = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int y = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    const int z = 1 + blockIdx.z;
    if (x >= a.g.nx - 1 || y >= a.g.ny - 1) return;
    const uint32_t gid = (uint32_t)x + (uint32_t)a.g.nx * ((uint32_t)y + (uint32_t)a.g.ny * (uint32_t)z);
    // solid and newly uncovered cells are updated by k_bulk_generic over the geometry box
    if (a.mask && a.mask[gid]) return;
    R f[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (REP_S) f[q] = S::ld_rt((const T*)a.plane[q] + gid, q);
        else f[q] = S::ld_rt((const T*)a.plane[opp(q)] + (uint32_t)(gid - (uint32_t)a.doff[q]), opp(q));
    }
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
    R post[19];
    float activation = 0.0f, restriction = 0.0f;
    collide<R, COLL>(f, rho, mx / rho, my / rho, mz / rho, (R)a.fp.omega_p, (R)a.fp.omega_m, post, activation,
                     restriction);
    finish_interior<S, COLL, CAPTURE>(a, gid, x, y, z, post, activation, restriction);
    store_interior<S, REP_S>(a, gid, post);
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
// Equilibrium with the reference's FP32 (or FP64) operation order, on the host
// (compiled with -ffp-contract=off, so it matches the device values bit for bit).
template <class R>
static R host_feq(int q, R rho, R ux, R uy, R uz) {
    R cu = (R)cx(q) * ux + (R)cy(q) * uy + (R)cz(q) * uz;
    R u2 = ux * ux + uy * uy + uz * uz;
    R w = q == 0 ? Lat<R>::w0 : (q <= 6 ? Lat<R>::w1 : Lat<R>::w2);
    return w * rho * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * u2);
}

static size_t elem_bytes(int storage) {
    return storage == BFX_STORAGE_F64 ? 8 : (storage == BFX_STORAGE_F32 ? 4 : 2);
}

static BulkArgs make_args(const GridDesc& gd, const FluidParams& fp, const FluidBuffers& b, int capture,
                          int storage = BFX_STORAGE_F32) {
    BulkArgs a;
    for (int q = 0; q < 19; ++q) {
        a.plane[q] = (char*)b.pops + (size_t)q * (size_t)gd.n * elem_bytes(storage);
        a.doff[q] = (int32_t)((int64_t)cx(q) + (int64_t)gd.nx * cy(q) + gd.nxy * cz(q));
        a.far_eq_f[q] = host_feq<float>(q, fp.far[3], fp.far[0], fp.far[1], fp.far[2]);
        a.far_eq_d[q] = host_feq<double>(q, (double)fp.far[3], (double)fp.far[0], (double)fp.far[1], (double)fp.far[2]);
    }
    a.shell_cells = 2 * (int64_t)gd.nx * gd.ny + 2 * (int64_t)gd.nx * (gd.nz - 2) + 2 * (int64_t)(gd.ny - 2) * (gd.nz - 2);
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
    GridDesc in = g;
    in.nx = g.nx - 2;
    in.ny = g.ny - 2;
    in.nz = g.nz - 2;
    dim3 grid, block;
    cell_launch_shape(in, grid, block);
    if (a.capture) k_bulk_interior<S, REP, COLL, 1><<<grid, block, 0, s>>>(a);
    else k_bulk_interior<S, REP, COLL, 0><<<grid, block, 0, s>>>(a);
}

template <class S, int REP, int COLL>
static void shell_t(const BulkArgs& a, cudaStream_t s) {
    k_bulk_generic<S, REP, COLL, 0><<<(unsigned)((a.shell_cells + 127) / 128), 128, 0, s>>>(a);
    if (a.mask && a.box_cells > 0)
        k_bulk_generic<S, REP, COLL, 1><<<(unsigned)((a.box_cells + 127) / 128), 128, 0, s>>>(a);
}

template <class S>
static void bulk_s(const BulkArgs& a, const GridDesc& g, int collision, int rep_s, int part, cudaStream_t s) {
#define BFX_PART(REP, COLL) (part == 0 ? bulk_t<S, REP, COLL>(a, g, s) : shell_t<S, REP, COLL>(a, s))
    switch (collision * 2 + rep_s) {
    case 0: BFX_PART(0, BFX_COLLISION_TRT); break;
    case 1: BFX_PART(1, BFX_COLLISION_TRT); break;
    case 2: BFX_PART(0, BFX_COLLISION_TRT_LIMITER); break;
    case 3: BFX_PART(1, BFX_COLLISION_TRT_LIMITER); break;
    case 4: BFX_PART(0, BFX_COLLISION_REGULARIZED); break;
    case 5: BFX_PART(1, BFX_COLLISION_REGULARIZED); break;
    case 6: BFX_PART(0, BFX_COLLISION_RR3); break;
    default: BFX_PART(1, BFX_COLLISION_RR3); break;
    }
#undef BFX_PART
}

#define BFX_DISPATCH_STORAGE(storage, FN, ...)                 \
    switch (storage) {                                         \
    case BFX_STORAGE_F16_DEVIATION: FN<StoreF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_BF16_DEVIATION: FN<StoreBF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_F64: FN<StoreF64>(__VA_ARGS__); break;    \
    default: FN<StoreF32>(__VA_ARGS__); break;                 \
    }

void launch_bulk(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, int capture, int part, const int* box, cudaStream_t s) {
    BulkArgs a = make_args(g, fp, b, capture, storage);
    a.box[0] = box ? box[0] : 0;
    a.box[1] = box ? box[1] : 0;
    a.box[2] = box ? box[2] : 0;
    a.box_cells = box ? (int64_t)box[0] * box[1] * box[2] : 0;
    BFX_DISPATCH_STORAGE(storage, bulk_s, a, g, collision, rep_s, part, s);
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
