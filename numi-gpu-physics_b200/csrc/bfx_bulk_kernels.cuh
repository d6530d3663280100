// Fused-step kernel templates (see bfx_bulk.cuh); included once per variant.
#include "bfx_bulk.cuh"

#ifndef BFX_VARIANT
#error "define BFX_VARIANT before including bfx_bulk_kernels.cuh"
#endif

namespace bfx {
namespace BFX_VARIANT {

#ifdef BFX_CONTRACTED
#include "bfx_pair_math.cuh"
#endif

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
        // Positivity admission (BF.metal:3035-3052).  The floor test runs on
        // every population; the admissible scale, which only a population below
        // its floor changes, is evaluated afterwards in the same direction order
        // for the rare cell that has one.
        bool need = false;
        auto below = [&](R fe, R cand) {
            R fl = R(1.0e-6) * (fe > R(0) ? fe : R(0));
            R floor_ = R(1.0e-12) > fl ? R(1.0e-12) : fl;
            need = need || cand < floor_;
        };
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
            below(feqv[0], post[0]);
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
            below(feqv[q], post[q]);
            below(feqv[q + 1], post[q + 1]);
        }
        if (need) {
#pragma unroll
            for (int q = 0; q < 19; ++q) admit(feqv[q], post[q]);
        }
        if (scale < R(1)) {
            activation = 1.0f;
            restriction = (float)(R(1) - scale);
#pragma unroll
            for (int q = 0; q < 19; ++q) post[q] = feqv[q] + scale * (post[q] - feqv[q]);
        } else if (scale == R(1)) {
            // 1 * d == d exactly, but feq + (cand - feq) equals cand only up to
            // rounding, so the rest of the reference expression stays
#pragma unroll
            for (int q = 0; q < 19; ++q) post[q] = feqv[q] + (post[q] - feqv[q]);
        } else {
            // NaN scale (a non-finite equilibrium): the reference expression as is
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

// ---------------------------------------------------------------------------
// Per-cell pieces shared by the fused kernel and the rare-cell kernel.
// ---------------------------------------------------------------------------
template <class S, int REP_S>
__device__ __forceinline__ void load_cell(const BulkArgs& a, uint32_t pid, typename S::R (&f)[19]) {
    using T = typename S::T;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (REP_S) f[q] = S::ld_rt((const T*)a.plane[q] + pid, q);
        else f[q] = S::ld_rt((const T*)a.plane[opp(q)] + (uint32_t)(pid - (uint32_t)a.doff[q]), opp(q));
    }
}

template <class S, int REP_S>
__device__ __forceinline__ void store_cell(const BulkArgs& a, uint32_t pid, const typename S::R (&post)[19]) {
    using T = typename S::T;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (REP_S) S::st_rt((T*)a.plane[opp(q)] + pid, opp(q), post[q]);
        else S::st_rt((T*)a.plane[q] + (uint32_t)(pid + (uint32_t)a.doff[q]), q, post[q]);
    }
}

// Moments in the reference order (rho over q = 0..18, momentum componentwise).
template <class R>
__device__ __forceinline__ void moments(const R (&f)[19], R& rho, R& ux, R& uy, R& uz) {
    R r = 0, mx = 0, my = 0, mz = 0;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        r += f[q];
        if (cx(q) > 0) mx += f[q];
        if (cx(q) < 0) mx -= f[q];
        if (cy(q) > 0) my += f[q];
        if (cy(q) < 0) my -= f[q];
        if (cz(q) > 0) mz += f[q];
        if (cz(q) < 0) mz -= f[q];
    }
    r = r > R(1.0e-8) ? r : R(1.0e-8);
    rho = r;
#ifdef BFX_CONTRACTED
    // contracted variant: one reciprocal instead of three correctly rounded divisions
    const R inv = R(1) / r;
    ux = mx * inv;
    uy = my * inv;
    uz = mz * inv;
#else
    ux = mx / r;
    uy = my / r;
    uz = mz / r;
#endif
}

// Sponge relaxation toward the far field, captured fields, limiter statistics.
template <class S, int COLL>
__device__ __forceinline__ void finish_cell(const BulkArgs& a, uint32_t gid, int x, int y, int z, bool capture,
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
    if (capture) {
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

// Solid cells write the moving-wall equilibrium eq(1, u_wall)
// (BF.metal:2557-2570); newly uncovered cells refill from it and collide
// (BF.metal:2610-2625).  Called for a cell whose mask byte is nonzero (only
// cells of the geometry box have one) by the fused kernels.
template <class S, int REP_S, int COLL>
__device__ __forceinline__ void rare_cell(const BulkArgs& a, uint32_t gid, int x, int y, int z, uint32_t pid,
                                       uint8_t m) {
    using R = typename S::R;
    const float4 w = a.wall[gid];
    const R ux = w.x, uy = w.y, uz = w.z;
    const R u2 = ux * ux + uy * uy + uz * uz;
    R post[19];
    if (m & kPartMask) {
#pragma unroll
        for (int q = 0; q < 19; ++q) post[q] = feqq<R>(q, R(1), ux, uy, uz, u2);
        store_cell<S, REP_S>(a, pid, post);
        if (a.capture == 1) {
            a.density[gid] = 1.0f;
            a.velocity[gid] = make_float4(w.x, w.y, w.z, 0.0f);
        }
        return;
    }
    R f[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = feqq<R>(q, R(1), ux, uy, uz, u2);
    R rho, vx, vy, vz;
    moments<R>(f, rho, vx, vy, vz);
    float activation = 0.0f, restriction = 0.0f;
    collide<R, COLL>(f, rho, vx, vy, vz, (R)a.fp.omega_p, (R)a.fp.omega_m, post, activation, restriction);
    finish_cell<S, COLL>(a, gid, x, y, z, a.capture == 1, post, activation, restriction);
    store_cell<S, REP_S>(a, pid, post);
}

// ---------------------------------------------------------------------------
// The fused kernel: every cell of the lattice; solid and newly uncovered
// cells (flagged in the mask) take rare_cell.
// ---------------------------------------------------------------------------
template <class S, int REP_S, int COLL, int CAPTURE>
__global__ void __launch_bounds__(256, sizeof(typename S::R) == 8 ? 1 : (COLL == BFX_COLLISION_TRT_LIMITER ? 2 : 4))
    k_bulk(const BulkArgs a) {
    using R = typename S::R;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= a.g.nx || y >= a.g.ny) return;
    const uint32_t gid = (uint32_t)x + (uint32_t)a.g.nx * ((uint32_t)y + (uint32_t)a.g.ny * (uint32_t)z);
    const uint32_t pid =
        (uint32_t)(x + 1) + (uint32_t)a.g.px * ((uint32_t)(y + 1) + (uint32_t)a.g.py * (uint32_t)(z + 1));
    if (a.mask) {
        const uint8_t m = a.mask[gid];
        if (m) {
            rare_cell<S, REP_S, COLL>(a, gid, x, y, z, pid, m);
            return;
        }
    }
    R f[19];
    load_cell<S, REP_S>(a, pid, f);
    R post[19];
    float activation = 0.0f, restriction = 0.0f;
#ifdef BFX_CONTRACTED
    if constexpr (COLL == BFX_COLLISION_RR3 || COLL == BFX_COLLISION_REGULARIZED) {
        float act[1] = {0.0f}, res[1] = {0.0f};
        collide_pairs<R, COLL>(f, a.fp.omega_p, post, act, res);
        activation = act[0];
        restriction = res[0];
    } else
#endif
    {
        R rho, ux, uy, uz;
        moments<R>(f, rho, ux, uy, uz);
        if (CAPTURE == 2) {
            // adjoint tape: the collision Jacobian depends on the pre-collision moments only
            R* t = (R*)a.tape + 4 * (size_t)gid;
            t[0] = rho;
            t[1] = ux;
            t[2] = uy;
            t[3] = uz;
        }
        collide<R, COLL>(f, rho, ux, uy, uz, (R)a.fp.omega_p, (R)a.fp.omega_m, post, activation, restriction);
    }
    finish_cell<S, COLL>(a, gid, x, y, z, CAPTURE == 1, post, activation, restriction);
    store_cell<S, REP_S>(a, pid, post);
}

// Solid / newly uncovered cells of the geometry box in a launch of their own
// (the staged kernel skips them).  A thread scans kRareZ cells along z of one
// (x, y) column of the box, all mask bytes loaded before the first is used.
constexpr int kRareZ = 8;
template <class S, int REP_S, int COLL>
__global__ void __launch_bounds__(128) k_rare(const BulkArgs a) {
    const int lx = blockIdx.x * blockDim.x + threadIdx.x;
    if (lx >= a.box[0]) return;
    const int x = a.state->box_origin[0] + lx;
    const int y = a.state->box_origin[1] + (int)blockIdx.y;
    const int z0 = a.state->box_origin[2] + (int)blockIdx.z * kRareZ;
    if (x < 0 || x >= a.g.nx || y < 0 || y >= a.g.ny) return;
    const int lz_end = a.box[2] - (int)blockIdx.z * kRareZ;
    const uint32_t plane = (uint32_t)a.g.nx * (uint32_t)a.g.ny;
    uint8_t m[kRareZ];
#pragma unroll
    for (int k = 0; k < kRareZ; ++k) {
        const int z = z0 + k;
        m[k] = (k < lz_end && z >= 0 && z < a.g.nz)
                   ? a.mask[(uint32_t)x + (uint32_t)a.g.nx * (uint32_t)y + plane * (uint32_t)z]
                   : (uint8_t)0;
    }
#pragma unroll 1
    for (int k = 0; k < kRareZ; ++k) {
        if (m[k] == 0) continue;
        const int z = z0 + k;
        const uint32_t gid = (uint32_t)x + (uint32_t)a.g.nx * (uint32_t)y + plane * (uint32_t)z;
        const uint32_t pid =
            (uint32_t)(x + 1) + (uint32_t)a.g.px * ((uint32_t)(y + 1) + (uint32_t)a.g.py * (uint32_t)(z + 1));
        rare_cell<S, REP_S, COLL>(a, gid, x, y, z, pid, m[k]);
    }
}

template <class S>
static void rare_s(const BulkArgs& a, int collision, int rep_s, cudaStream_t s) {
    const dim3 grid((unsigned)((a.box[0] + 127) / 128), (unsigned)a.box[1],
                    (unsigned)((a.box[2] + kRareZ - 1) / kRareZ));
    switch (collision * 2 + rep_s) {
    case 0: k_rare<S, 0, BFX_COLLISION_TRT><<<grid, 128, 0, s>>>(a); break;
    case 1: k_rare<S, 1, BFX_COLLISION_TRT><<<grid, 128, 0, s>>>(a); break;
    case 2: k_rare<S, 0, BFX_COLLISION_TRT_LIMITER><<<grid, 128, 0, s>>>(a); break;
    case 3: k_rare<S, 1, BFX_COLLISION_TRT_LIMITER><<<grid, 128, 0, s>>>(a); break;
    case 4: k_rare<S, 0, BFX_COLLISION_REGULARIZED><<<grid, 128, 0, s>>>(a); break;
    case 5: k_rare<S, 1, BFX_COLLISION_REGULARIZED><<<grid, 128, 0, s>>>(a); break;
    case 6: k_rare<S, 0, BFX_COLLISION_RR3><<<grid, 128, 0, s>>>(a); break;
    default: k_rare<S, 1, BFX_COLLISION_RR3><<<grid, 128, 0, s>>>(a); break;
    }
}

template <class S, int REP, int COLL>
static void bulk_t(const BulkArgs& a, const GridDesc& g, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    if (a.capture == 1) k_bulk<S, REP, COLL, 1><<<grid, block, 0, s>>>(a);
#ifndef BFX_CONTRACTED
    else if (a.capture == 2 && COLL == BFX_COLLISION_TRT) k_bulk<S, REP, BFX_COLLISION_TRT, 2><<<grid, block, 0, s>>>(a);
#endif
    else k_bulk<S, REP, COLL, 0><<<grid, block, 0, s>>>(a);
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

}  // namespace BFX_VARIANT
}  // namespace bfx
