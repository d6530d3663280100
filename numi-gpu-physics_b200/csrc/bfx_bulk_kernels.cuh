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

// Sums over the pairs (q odd) of c_a(q) v[q] (B < 0) or c_a(q) c_b(q) v[q],
// the first nonzero term taken as is or negated, then added or subtracted in
// direction order.
template <int A, int B, class R>
__device__ __forceinline__ R pair_sum(const R (&v)[19]) {
    R r = R(0);
    bool first = true;
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const int ca = A == 0 ? cx(q) : (A == 1 ? cy(q) : cz(q));
        const int cb = B < 0 ? 1 : (B == 0 ? cx(q) : (B == 1 ? cy(q) : cz(q)));
        const int c = ca * cb;
        if (c == 0) continue;
        r = first ? (c > 0 ? v[q] : -v[q]) : (c > 0 ? r + v[q] : r - v[q]);
        first = false;
    }
    return r;
}

// Regularized / RR3 collision (BF.metal:2917-3062) evaluated on
// opposite-direction pairs (q odd, q + 1 = opp q), the oracle's
// regularized_pairs operation for operation (FP32 results bit-identical to
// it; the reference's literal per-direction order agrees with it to FP32
// rounding):
//   moments from pair sums p = f_q + f_q' and differences m = f_q - f_q';
//   feq_q = E + O, feq_q' = E - O with E = w rho (1 - 1.5u^2 + 4.5cu^2),
//   O = 3 w rho cu;
//   stress from the pair non-equilibria n = p - 2E:
//   ds_a = sum_{c_a != 0} n - cs2 (ne_0 + sum n), od_ab = sum sign(c_a c_b) n;
//   post_q = X + Y, post_q' = X - Y with X = E + (1 - w+) w 4.5 H2:ds,
//   Y = O + (1 - w+) w 13.5 H3:a3;
//   positivity admission over every direction, and the scaled blend
//   feq + s (cand - feq) only where s < 1.
// It takes about two thirds of the literal form's instructions.  A cheap
// superset test (min over the populations against 1e-12 + 1e-6 max feq, with
// E + |O| bounding each pair's equilibria) skips the exact admission for the
// cells that cannot need it; the exact test then decides as the oracle does.
template <class R, int COLL>
__device__ __forceinline__ void regularized_pairs(const R (&f)[19], R omega_p, R (&post)[19], float& activation,
                                                  float& restriction) {
    const R cs2 = Lat<R>::cs2;
    R ps[19], md[19], E[19], O[19], nps[19];
    R rho = f[0];
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        ps[q] = f[q] + f[q + 1];
        md[q] = f[q] - f[q + 1];
        rho = rho + ps[q];
    }
    const R mx = pair_sum<0, -1>(md), my = pair_sum<1, -1>(md), mz = pair_sum<2, -1>(md);
    rho = rho > R(1.0e-8) ? rho : R(1.0e-8);
    const R ux = mx / rho, uy = my / rho, uz = mz / rho;
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R base = R(1) - R(1.5) * u2;
    const R wr1 = Lat<R>::w1 * rho, wr2 = Lat<R>::w2 * rho;
    const R feq0 = (Lat<R>::w0 * rho) * base;
    R ntot = f[0] - feq0;
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const R cu = cdotq<R>(q, ux, uy, uz);
        const R wr = q <= 6 ? wr1 : wr2;
        E[q] = wr * (base + (R(4.5) * cu) * cu);
        O[q] = wr * (R(3) * cu);
        nps[q] = ps[q] - R(2) * E[q];
        ntot = ntot + nps[q];
    }
    const R dsx = pair_sum<0, 0>(nps) - cs2 * ntot;
    const R dsy = pair_sum<1, 1>(nps) - cs2 * ntot;
    const R dsz = pair_sum<2, 2>(nps) - cs2 * ntot;
    const R odx = pair_sum<0, 1>(nps), ody = pair_sum<0, 2>(nps), odz = pair_sum<1, 2>(nps);
    const R aXxy = (R(2) * ux) * odx + uy * dsx;
    const R aXxz = (R(2) * ux) * ody + uz * dsx;
    const R aXyy = ux * dsy + (R(2) * uy) * odx;
    const R aXzz = ux * dsz + (R(2) * uz) * ody;
    const R aYyz = (R(2) * uy) * odz + uz * dsy;
    const R aYzz = uy * dsz + (R(2) * uz) * odz;
    const R trace = dsx + dsy + dsz;
    const R cax = dsx - cs2 * trace, cay = dsy - cs2 * trace, caz = dsz - cs2 * trace;
    const R om = R(1) - omega_p;
    const R om0 = om * (Lat<R>::w0 * R(4.5) * -cs2);
    const R om1 = om * (Lat<R>::w1 * R(4.5)), om2 = om * (Lat<R>::w2 * R(4.5));
    const R ot1 = om * (Lat<R>::w1 * R(13.5)), ot2 = om * (Lat<R>::w2 * R(13.5));
    post[0] = feq0 + om0 * trace;
    R lo = post[0], hi = feq0;
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        R contraction;
        if (cx(q) != 0 && cy(q) != 0) contraction = (cax + dsy) + R(2) * (cx(q) * cy(q) > 0 ? odx : -odx);
        else if (cx(q) != 0 && cz(q) != 0) contraction = (cax + dsz) + R(2) * (cx(q) * cz(q) > 0 ? ody : -ody);
        else if (cy(q) != 0 && cz(q) != 0) contraction = (cay + dsz) + R(2) * (cy(q) * cz(q) > 0 ? odz : -odz);
        else contraction = cx(q) != 0 ? cax : (cy(q) != 0 ? cay : caz);
        const R X = E[q] + (q <= 6 ? om1 : om2) * contraction;
        R Y = O[q];
        if (COLL == BFX_COLLISION_RR3) {
            const R hx = (R)(cx(q) * cx(q)) - cs2, hy = (R)(cy(q) * cy(q)) - cs2, hz = (R)(cz(q) * cz(q)) - cs2;
            R third = R(0);
            bool any = false;
            auto add = [&](int da, R hb, R amp) {
                if (da == 0) return;
                const R t = ((R)da * hb) * amp;
                third = any ? third + t : t;
                any = true;
            };
            add(cy(q), hx, aXxy);
            add(cz(q), hx, aXxz);
            add(cx(q), hy, aXyy);
            add(cx(q), hz, aXzz);
            add(cz(q), hy, aYyz);
            add(cy(q), hz, aYzz);
            Y = Y + (q <= 6 ? ot1 : ot2) * third;
        }
        post[q] = X + Y;
        post[q + 1] = X - Y;
        lo = fmin(lo, fmin(post[q], post[q + 1]));
        hi = fmax(hi, E[q] + fabs(O[q]));
    }
    // every floor max(1e-12, 1e-6 max(feq_q, 0)) is at most 1e-12 + 1e-6 max(hi, 0)
    if (!(lo < R(1.0e-12) + R(1.0e-6) * fmax(hi, R(0)))) return;
    R scale = R(1);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const R fe = q == 0 ? feq0 : ((q & 1) ? E[q] + O[q] : E[q - 1] - O[q - 1]);
        const R fl = R(1.0e-6) * (fe > R(0) ? fe : R(0));
        const R floor_ = R(1.0e-12) > fl ? R(1.0e-12) : fl;
        if (post[q] < floor_) {
            R den = fe - post[q];
            den = den > R(1.0e-30) ? den : R(1.0e-30);
            R adm = (fe - floor_) / den;
            adm = adm < R(0) ? R(0) : (adm > R(1) ? R(1) : adm);
            scale = scale < adm ? scale : adm;
        }
    }
    if (scale < R(1)) {
        activation = 1.0f;
        restriction = (float)(R(1) - scale);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const R fe = q == 0 ? feq0 : ((q & 1) ? E[q] + O[q] : E[q - 1] - O[q - 1]);
            post[q] = fe + scale * (post[q] - fe);
        }
    }
}

// TRT and symmetric-limiter collision (BF.metal:3063-3174; the regularized
// operators are regularized_pairs).  Directions are processed in opposite pairs
// (q odd, q+1 = opp(q)): the equilibrium and TRT terms of the pair
// share their even parts and negate their odd parts, and in IEEE arithmetic
// -(a-b) == b-a, (-a)*b == -(a*b), x-(-y) == x+y exactly.  Every value is
// therefore bit-identical to evaluating the reference expression once per
// direction, at about half the instruction count.
template <class R, int COLL>
__device__ __forceinline__ void collide(const R (&f)[19], R rho, R ux, R uy, R uz, R omega_p, R omega_m,
                                        R (&post)[19], float& activation, float& restriction) {
    static_assert(COLL == BFX_COLLISION_TRT || COLL == BFX_COLLISION_TRT_LIMITER,
                  "the regularized operators run through regularized_pairs");
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

    if (COLL == BFX_COLLISION_TRT) {
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

// A fluid cell's collided populations: stochastic rounding for BF16 (the
// stream of cell gid at the step the device state counts), plain stores else.
template <class S, int REP_S>
__device__ __forceinline__ void store_fluid_cell(const BulkArgs& a, uint32_t gid, uint32_t pid,
                                                 const typename S::R (&post)[19]) {
    using T = typename S::T;
    if constexpr (S::kStochastic) {
        uint32_t x = sr_seed(gid, (uint32_t)a.state->step);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            x = sr_next(x);
            if (REP_S) S::st_rt_sr((T*)a.plane[opp(q)] + pid, opp(q), post[q], x);
            else S::st_rt_sr((T*)a.plane[q] + (uint32_t)(pid + (uint32_t)a.doff[q]), q, post[q], x);
        }
    } else {
        store_cell<S, REP_S>(a, pid, post);
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
    float activation = 0.0f, restriction = 0.0f;
    if constexpr (COLL == BFX_COLLISION_RR3 || COLL == BFX_COLLISION_REGULARIZED) {
        regularized_pairs<R, COLL>(f, (R)a.fp.omega_p, post, activation, restriction);
    } else {
        R rho, vx, vy, vz;
        moments<R>(f, rho, vx, vy, vz);
        collide<R, COLL>(f, rho, vx, vy, vz, (R)a.fp.omega_p, (R)a.fp.omega_m, post, activation, restriction);
    }
    finish_cell<S, COLL>(a, gid, x, y, z, a.capture == 1, post, activation, restriction);
    store_fluid_cell<S, REP_S>(a, gid, pid, post);
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
    if constexpr (COLL == BFX_COLLISION_RR3 || COLL == BFX_COLLISION_REGULARIZED) {
#ifdef BFX_CONTRACTED
        float act[1] = {0.0f}, res[1] = {0.0f};
        collide_pairs<R, COLL>(f, a.fp.omega_p, post, act, res);
        activation = act[0];
        restriction = res[0];
#else
        regularized_pairs<R, COLL>(f, (R)a.fp.omega_p, post, activation, restriction);
#endif
    } else {
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
    store_fluid_cell<S, REP_S>(a, gid, pid, post);
}

// Solid / newly uncovered cells of the geometry box in a launch of their own
// (the staged kernel skips them).  A thread scans kRareZ cells along z of one
// (x, y) column of the box, all mask bytes loaded before the first is used.
constexpr int kRareZ = 8;
template <class S, int REP_S, int COLL>
__global__ void __launch_bounds__(128) k_rare(const BulkArgs a) {
    const int lx = blockIdx.x * blockDim.x + threadIdx.x;
    if (lx >= a.box[0]) return;
    const DeviceState* st = a.state;
    const int x = st->box_origin[0] + lx;
    const int y = st->box_origin[1] + (int)blockIdx.y;
    const int z0 = st->box_origin[2] + (int)blockIdx.z * kRareZ;
    if (x < 0 || x >= a.g.nx || y < 0 || y >= a.g.ny) return;
    // flagged cells lie within the geometry's active bounds
    const int am = a.fp.act_margin;
    if (x < st->act_lo[0] - am || x > st->act_hi[0] + am || y < st->act_lo[1] - am || y > st->act_hi[1] + am ||
        z0 + kRareZ - 1 < st->act_lo[2] - am || z0 > st->act_hi[2] + am)
        return;
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
