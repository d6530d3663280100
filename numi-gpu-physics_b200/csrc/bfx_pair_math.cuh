// Arithmetic of the contracted variant (bfx_fluid_fast.cu): packed f32x2 pairs
// (two cells per lane) and the regularized / RR3 collision restated on
// opposite-direction pairs.  Included inside namespace bfx::BFX_VARIANT by
// bfx_bulk_kernels.cuh when BFX_CONTRACTED is defined.
//
// The restatement evaluates the same operator as collide<R, COLL> (the
// reference's BF.metal:2917-3062) with a different operation order:
//   * moments from pair sums p_q = f_q + f_q' and differences m_q = f_q - f_q'
//     (q' = opp q);
//   * the equilibrium split into its even part E_q = w rho (1 - 1.5u^2 + 4.5cu^2)
//     and odd part O_q = 3 w rho cu, so feq_q = E_q + O_q, feq_q' = E_q - O_q;
//   * the second-order non-equilibrium stress from the pair non-equilibria
//     n_q = p_q - 2 E_q (the sums of (f - feq) over each pair):
//       ds_a = sum_{c_a != 0} n_q - cs2 * sum_all n,  od_ab = sum sign(c_a c_b) n_q;
//   * the post-collision pair as X +- Y with X = E_q + (1 - omega) w 4.5 H2:Pi
//     and Y = O_q + (1 - omega) w 13.5 H3:a3;
//   * the positivity admission tested on every population, with the scaled
//     blend feq + s (cand - feq) evaluated only for a cell where some
//     population falls below its floor (s < 1).
// Every quantity is a cancellation of the same size as in the literal form,
// so the rounding stays at the FP32 level; the 16-bit formats' quantisation is
// about 100x larger.

using P2 = float2;
__device__ __forceinline__ P2 pv(float s) { return make_float2(s, s); }
#define BFX_F32X2_OP(NAME, INSTR)                                                                   \
    __device__ __forceinline__ P2 NAME(P2 a, P2 b) {                                               \
        P2 r;                                                                                      \
        asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n " INSTR     \
            " d, a, b;\n mov.b64 {%0, %1}, d;\n}"                                                  \
            : "=f"(r.x), "=f"(r.y)                                                                 \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                             \
        return r;                                                                                  \
    }
BFX_F32X2_OP(padd, "add.rn.f32x2")
BFX_F32X2_OP(psub, "sub.rn.f32x2")
BFX_F32X2_OP(pmul, "mul.rn.f32x2")
#undef BFX_F32X2_OP
__device__ __forceinline__ P2 operator+(P2 a, P2 b) { return padd(a, b); }
__device__ __forceinline__ P2 operator-(P2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ P2 operator-(P2 a, P2 b) { return psub(a, b); }
__device__ __forceinline__ P2 operator*(P2 a, P2 b) { return pmul(a, b); }
__device__ __forceinline__ P2 operator*(float s, P2 a) { return pmul(make_float2(s, s), a); }
__device__ __forceinline__ P2 operator*(P2 a, float s) { return pmul(a, make_float2(s, s)); }

// Lane access for one cell (float) or two cells (P2).
template <class V> struct Lanes;
template <> struct Lanes<float> {
    static constexpr int n = 1;
    __device__ __forceinline__ static float splat(float s) { return s; }
    __device__ __forceinline__ static float get(float v, int) { return v; }
    __device__ __forceinline__ static void set(float& v, int, float s) { v = s; }
};
template <> struct Lanes<P2> {
    static constexpr int n = 2;
    __device__ __forceinline__ static P2 splat(float s) { return make_float2(s, s); }
    __device__ __forceinline__ static float get(P2 v, int l) { return l ? v.y : v.x; }
    __device__ __forceinline__ static void set(P2& v, int l, float s) {
        if (l) v.y = s;
        else v.x = s;
    }
};

// sum over the pairs (q odd) of c_axis(q) * v[q], zero coefficients dropped
template <int AX, class V>
__device__ __forceinline__ V pair_dot(const V (&v)[19]) {
    V r = Lanes<V>::splat(0.0f);
    bool first = true;
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const int c = AX == 0 ? cx(q) : (AX == 1 ? cy(q) : cz(q));
        if (c == 0) continue;
        r = first ? (c > 0 ? v[q] : -v[q]) : (c > 0 ? r + v[q] : r - v[q]);
        first = false;
    }
    return r;
}

// sum over the pairs of c_a(q)^2 * v[q] (AX = a) or c_a c_b v[q] (cross terms)
template <int A, int B, class V>
__device__ __forceinline__ V pair_second(const V (&v)[19]) {
    V r = Lanes<V>::splat(0.0f);
    bool first = true;
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const int ca = A == 0 ? cx(q) : (A == 1 ? cy(q) : cz(q));
        const int cb = B == 0 ? cx(q) : (B == 1 ? cy(q) : cz(q));
        const int c = ca * cb;
        if (c == 0) continue;
        r = first ? (c > 0 ? v[q] : -v[q]) : (c > 0 ? r + v[q] : r - v[q]);
        first = false;
    }
    return r;
}

template <class V>
__device__ __forceinline__ V cdot_pair(int q, V ux, V uy, V uz) {
    V r = Lanes<V>::splat(0.0f);
    bool first = true;
    if (cx(q) != 0) { r = cx(q) > 0 ? ux : -ux; first = false; }
    if (cy(q) != 0) { r = first ? (cy(q) > 0 ? uy : -uy) : (cy(q) > 0 ? r + uy : r - uy); first = false; }
    if (cz(q) != 0) { r = first ? (cz(q) > 0 ? uz : -uz) : (cz(q) > 0 ? r + uz : r - uz); }
    return r;
}

// Positivity floor of the admission step: max(1e-12, 1e-6 max(feq, 0)).
__device__ __forceinline__ float admit_floor(float fe) {
    const float fl = 1.0e-6f * (fe > 0.0f ? fe : 0.0f);
    return 1.0e-12f > fl ? 1.0e-12f : fl;
}

// Regularized / RR3 collision of one (float) or two (P2) cells from their
// incoming populations: moments, equilibrium, projected non-equilibrium and
// positivity admission.  post receives the post-collision populations.
template <class V, int COLL>
__device__ __forceinline__ void collide_pairs(const V (&f)[19], float omega_p, V (&post)[19],
                                              float (&activation)[Lanes<V>::n],
                                              float (&restriction)[Lanes<V>::n]) {
    using L = Lanes<V>;
    constexpr float cs2 = Lat<float>::cs2;
    V ps[19], md[19];
    V rho = f[0];
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        ps[q] = f[q] + f[q + 1];
        md[q] = f[q] - f[q + 1];
        rho = rho + ps[q];
    }
    const V mx = pair_dot<0>(md), my = pair_dot<1>(md), mz = pair_dot<2>(md);
    V inv;
#pragma unroll
    for (int l = 0; l < L::n; ++l) {
        float r = L::get(rho, l);
        r = r > 1.0e-8f ? r : 1.0e-8f;
        L::set(rho, l, r);
        L::set(inv, l, 1.0f / r);
    }
    const V ux = mx * inv, uy = my * inv, uz = mz * inv;
    const V u2 = ux * ux + uy * uy + uz * uz;
    const V base = L::splat(1.0f) - 1.5f * u2;
    const V wr1 = Lat<float>::w1 * rho, wr2 = Lat<float>::w2 * rho;
    const V feq0 = (Lat<float>::w0 * rho) * base;
    V E[19], O[19], nps[19];
    V ntot = f[0] - feq0;
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const V cu = cdot_pair(q, ux, uy, uz);
        const V wr = q <= 6 ? wr1 : wr2;
        E[q] = wr * (base + (4.5f * cu) * cu);
        O[q] = wr * (3.0f * cu);
        nps[q] = ps[q] - 2.0f * E[q];
        ntot = ntot + nps[q];
    }
    const V dsx = pair_second<0, 0>(nps) - cs2 * ntot;
    const V dsy = pair_second<1, 1>(nps) - cs2 * ntot;
    const V dsz = pair_second<2, 2>(nps) - cs2 * ntot;
    const V odx = pair_second<0, 1>(nps), ody = pair_second<0, 2>(nps), odz = pair_second<1, 2>(nps);
    const V aXxy = (2.0f * ux) * odx + uy * dsx;
    const V aXxz = (2.0f * ux) * ody + uz * dsx;
    const V aXyy = ux * dsy + (2.0f * uy) * odx;
    const V aXzz = ux * dsz + (2.0f * uz) * ody;
    const V aYyz = (2.0f * uy) * odz + uz * dsy;
    const V aYzz = uy * dsz + (2.0f * uz) * odz;
    const V trace = (dsx + dsy) + dsz;
    // h:ds for one axis direction is ds_a - cs2 * trace; a diagonal adds ds_b
    const V cax = dsx - cs2 * trace, cay = dsy - cs2 * trace, caz = dsz - cs2 * trace;
    const float om = 1.0f - omega_p;
    const float om0 = om * (Lat<float>::w0 * 4.5f * -cs2);
    const float om1 = om * (Lat<float>::w1 * 4.5f), om2 = om * (Lat<float>::w2 * 4.5f);
    const float ot1 = om * (Lat<float>::w1 * 13.5f), ot2 = om * (Lat<float>::w2 * 13.5f);
    bool need[L::n];
    post[0] = feq0 + om0 * trace;
#pragma unroll
    for (int l = 0; l < L::n; ++l) need[l] = L::get(post[0], l) < admit_floor(L::get(feq0, l));
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const float hx = (float)(cx(q) * cx(q)) - cs2, hy = (float)(cy(q) * cy(q)) - cs2,
                    hz = (float)(cz(q) * cz(q)) - cs2;
        V contraction;
        if (cx(q) != 0 && cy(q) != 0) contraction = (cax + dsy) + 2.0f * (cx(q) * cy(q) > 0 ? odx : -odx);
        else if (cx(q) != 0 && cz(q) != 0) contraction = (cax + dsz) + 2.0f * (cx(q) * cz(q) > 0 ? ody : -ody);
        else if (cy(q) != 0 && cz(q) != 0) contraction = (cay + dsz) + 2.0f * (cy(q) * cz(q) > 0 ? odz : -odz);
        else contraction = cx(q) != 0 ? cax : (cy(q) != 0 ? cay : caz);
        const V X = E[q] + (q <= 6 ? om1 : om2) * contraction;
        V Y = O[q];
        if (COLL == BFX_COLLISION_RR3) {
            V third = L::splat(0.0f);
            bool any = false;
            auto add = [&](int da, float hb, V amp) {
                if (da == 0) return;
                const V t = ((float)da * hb) * amp;
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
        const V fq = E[q] + O[q], fo = E[q] - O[q];
#pragma unroll
        for (int l = 0; l < L::n; ++l) {
            need[l] = need[l] || L::get(post[q], l) < admit_floor(L::get(fq, l));
            need[l] = need[l] || L::get(post[q + 1], l) < admit_floor(L::get(fo, l));
        }
    }
    // rare: some population below its floor; scale the non-equilibrium part
#pragma unroll
    for (int l = 0; l < L::n; ++l) {
        if (!need[l]) continue;
        const float r = L::get(rho, l), vx = L::get(ux, l), vy = L::get(uy, l), vz = L::get(uz, l);
        float scale = 1.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const float fe = feq_rt<float>(q, r, vx, vy, vz);
            const float cand = L::get(post[q], l);
            const float floor_ = admit_floor(fe);
            if (cand < floor_) {
                float den = fe - cand;
                den = den > 1.0e-30f ? den : 1.0e-30f;
                float adm = (fe - floor_) / den;
                adm = adm < 0.0f ? 0.0f : (adm > 1.0f ? 1.0f : adm);
                scale = scale < adm ? scale : adm;
            }
        }
        if (scale < 1.0f) {
            activation[l] = 1.0f;
            restriction[l] = 1.0f - scale;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                const float fe = feq_rt<float>(q, r, vx, vy, vz);
                L::set(post[q], l, fe + scale * (L::get(post[q], l) - fe));
            }
        }
    }
}
