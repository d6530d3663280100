/*
 * CPU oracle for the D3Q19 moving-boundary step — TEST INFRASTRUCTURE ONLY.
 * See bfx_oracle.h for scope.  Every function cites the reference code it
 * restates (paths relative to the Numi2/numi-gpu-physics project root).
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fno-fast-math -shared -fPIC
 * (oracle/Makefile).  Contraction must stay off: the reference's FP32
 * operation order is part of the parity contract.
 */
#include "bfx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../numi-gpu-physics_b200/csrc/bfx_portable_math.h"

/* D3Q19 velocity set, opposite table and weights:
 * Sources/BirdFlowCore/D3Q19.swift:8-45, BF.metal:7-43. */
static const int C[19][3] = {
    {0, 0, 0},
    {1, 0, 0}, {-1, 0, 0},
    {0, 1, 0}, {0, -1, 0},
    {0, 0, 1}, {0, 0, -1},
    {1, 1, 0}, {-1, -1, 0},
    {1, -1, 0}, {-1, 1, 0},
    {1, 0, 1}, {-1, 0, -1},
    {1, 0, -1}, {-1, 0, 1},
    {0, 1, 1}, {0, -1, -1},
    {0, 1, -1}, {0, -1, 1}};
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
#define W0 (1.0f / 3.0f)
#define W1 (1.0f / 18.0f)
#define W2 (1.0f / 36.0f)
static const float W[19] = {W0, W1, W1, W1, W1, W1, W1, W2, W2, W2, W2, W2, W2, W2, W2, W2, W2, W2, W2};
static const float CS2 = 1.0f / 3.0f;

void or_lattice(int32_t* c, int32_t* opp, float* w) {
    for (int q = 0; q < 19; ++q) {
        c[3 * q] = C[q][0];
        c[3 * q + 1] = C[q][1];
        c[3 * q + 2] = C[q][2];
        opp[q] = OPP[q];
        w[q] = W[q];
    }
}

/* dot(float3(C[q]), u) as the reference writes it: x + y + z products. */
static inline float cdot(int q, const float u[3]) {
    return (float)C[q][0] * u[0] + (float)C[q][1] * u[1] + (float)C[q][2] * u[2];
}
static inline float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void cross3(const float a[3], const float b[3], float r[3]) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline float lengthf(const float v[3]) { return sqrtf(dot3(v, v)); }
static inline float mixf(float a, float b, float t) { return a + (b - a) * t; }
static inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

/* equilibrium: BF.metal:478-484; D3Q19.swift:48-58 */
float or_equilibrium(int q, float rho, const float u[3]) {
    float cu = cdot(q, u);
    float u2 = dot3(u, u);
    return W[q] * rho * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * u2);
}

/* D3Q19.trtCollision: D3Q19.swift:84-108 */
void or_trt_collision(const float* f, float rho, const float u[3], float omega_p, float omega_m, float* out) {
    float eq[19];
    for (int q = 0; q < 19; ++q) eq[q] = or_equilibrium(q, rho, u);
    for (int q = 0; q < 19; ++q) {
        int qo = OPP[q];
        float fp = 0.5f * (f[q] + f[qo]);
        float fm = 0.5f * (f[q] - f[qo]);
        float ep = 0.5f * (eq[q] + eq[qo]);
        float em = 0.5f * (eq[q] - eq[qo]);
        out[q] = f[q] - omega_p * (fp - ep) - omega_m * (fm - em);
    }
}

static inline int64_t ncells(const or_params* p) { return (int64_t)p->nx * p->ny * p->nz; }
static inline int64_t flat(const or_params* p, int x, int y, int z) {
    return (int64_t)x + (int64_t)p->nx * ((int64_t)y + (int64_t)p->ny * z);
}
static inline int inside3(const or_params* p, int x, int y, int z) {
    return x >= 0 && y >= 0 && z >= 0 && x < p->nx && y < p->ny && z < p->nz;
}
/* cellPosition: BF.metal:449-452 */
static inline void cell_world(const or_params* p, int x, int y, int z, float w[3]) {
    w[0] = p->origin[0] + ((float)x + 0.5f) * p->dx;
    w[1] = p->origin[1] + ((float)y + 0.5f) * p->dx;
    w[2] = p->origin[2] + ((float)z + 0.5f) * p->dx;
}
static inline int axis_periodic(const or_params* p, int a) {
    return p->face_bc[2 * a] == OR_BC_PERIODIC && p->face_bc[2 * a + 1] == OR_BC_PERIODIC;
}

/* spongeFactor: BF.metal:2427-2446 */
static float sponge_factor(const or_params* p, int x, int y, int z) {
    unsigned dxm = (unsigned)x < (unsigned)(p->nx - 1 - x) ? (unsigned)x : (unsigned)(p->nx - 1 - x);
    unsigned dym = (unsigned)y < (unsigned)(p->ny - 1 - y) ? (unsigned)y : (unsigned)(p->ny - 1 - y);
    unsigned dzm = (unsigned)z < (unsigned)(p->nz - 1 - z) ? (unsigned)z : (unsigned)(p->nz - 1 - z);
    unsigned m = dxm < dym ? dxm : dym;
    m = m < dzm ? m : dzm;
    float distance = (float)m;
    float width = p->sponge_width;
    if (distance >= width) return 0.0f;
    float n = clampf((width - distance) / fmaxf(width, 1.0f), 0.0f, 1.0f);
    return p->sponge_strength * n * n;
}

/* ------------------------------------------------------------------ */
/* Initialisation: initializePopulations BF.metal:2078-2103,           */
/* initializeShearWave BF.metal:2132-2162, extractMacroscopicFields     */
/* BF.metal:2107-2127.                                                 */
/* ------------------------------------------------------------------ */
void or_init_equilibrium(const or_params* p, float* pops, const uint8_t* mask, const float* wall,
                         float* density, float* velocity) {
    int64_t n = ncells(p);
#pragma omp parallel for schedule(static)
    for (int64_t gid = 0; gid < n; ++gid) {
        float u[3];
        if (mask && mask[gid] != 0) {
            u[0] = wall[4 * gid];
            u[1] = wall[4 * gid + 1];
            u[2] = wall[4 * gid + 2];
        } else {
            u[0] = p->far[0];
            u[1] = p->far[1];
            u[2] = p->far[2];
        }
        for (int q = 0; q < 19; ++q) pops[q * n + gid] = or_equilibrium(q, 1.0f, u);
        if (density) density[gid] = 1.0f;
        if (velocity) {
            velocity[4 * gid] = u[0];
            velocity[4 * gid + 1] = u[1];
            velocity[4 * gid + 2] = u[2];
            velocity[4 * gid + 3] = 0.0f;
        }
    }
}

void or_init_shear_wave(const or_params* p, float amplitude, int axis, float* pops, float* density, float* velocity) {
    int64_t n = ncells(p);
#pragma omp parallel for schedule(static)
    for (int64_t gid = 0; gid < n; ++gid) {
        int64_t xy = (int64_t)p->nx * p->ny;
        int z = (int)(gid / xy);
        int64_t rem = gid - (int64_t)z * xy;
        int y = (int)(rem / p->nx);
        int coord = axis == 2 ? z : y;
        int extent = axis == 2 ? p->nz : p->ny;
        float phase = 2.0f * 3.14159265358979323846f * (float)coord / (float)extent;
        float u[3] = {amplitude * bfx_sinf(phase), 0.0f, 0.0f};
        for (int q = 0; q < 19; ++q) pops[q * n + gid] = or_equilibrium(q, 1.0f, u);
        if (density) density[gid] = 1.0f;
        if (velocity) {
            velocity[4 * gid] = u[0];
            velocity[4 * gid + 1] = 0.0f;
            velocity[4 * gid + 2] = 0.0f;
            velocity[4 * gid + 3] = 0.0f;
        }
    }
}

void or_macroscopic(const or_params* p, const float* pops, float* density, float* velocity) {
    int64_t n = ncells(p);
#pragma omp parallel for schedule(static)
    for (int64_t gid = 0; gid < n; ++gid) {
        float rho = 0.0f, m[3] = {0.0f, 0.0f, 0.0f};
        for (int q = 0; q < 19; ++q) {
            float v = pops[q * n + gid];
            rho += v;
            m[0] += v * (float)C[q][0];
            m[1] += v * (float)C[q][1];
            m[2] += v * (float)C[q][2];
        }
        rho = fmaxf(rho, 1.0e-8f);
        density[gid] = rho;
        velocity[4 * gid] = m[0] / rho;
        velocity[4 * gid + 1] = m[1] / rho;
        velocity[4 * gid + 2] = m[2] / rho;
        velocity[4 * gid + 3] = 0.0f;
    }
}

/* ------------------------------------------------------------------ */
/* FP64 load accumulator: one contribution = lattice force fl (float,   */
/* computed literally) applied at point pt (float world position).      */
/* ------------------------------------------------------------------ */
typedef struct {
    double f[3];
    double t[3];
    double act;
    double rmax;
    int64_t links, covered, uncovered;
} acc64;

static inline void acc_add(acc64* a, const float fl[3], const float pt[3], const double body[3], float f2p) {
    double fp[3] = {(double)fl[0] * (double)f2p, (double)fl[1] * (double)f2p, (double)fl[2] * (double)f2p};
    double r[3] = {(double)pt[0] - body[0], (double)pt[1] - body[1], (double)pt[2] - body[2]};
    a->f[0] += (double)fl[0];
    a->f[1] += (double)fl[1];
    a->f[2] += (double)fl[2];
    a->t[0] += r[1] * fp[2] - r[2] * fp[1];
    a->t[1] += r[2] * fp[0] - r[0] * fp[2];
    a->t[2] += r[0] * fp[1] - r[1] * fp[0];
}

/* Value of a population pulled from outside the domain after periodic
 * wrapping failed (far field, inlet velocity, or zero-gradient outflow). The
 * reference only has the far-field rule (BF.metal:2696-2725); the velocity and
 * outflow faces are this library's additions. */
static float outside_value(const or_params* p, int q, int cx, int cy, int cz, int sx, int sy, int sz,
                           const float* pin, const uint8_t* mcur) {
    int face;
    if (sx < 0 || sx >= p->nx) face = sx < 0 ? 0 : 1;
    else if (sy < 0 || sy >= p->ny) face = sy < 0 ? 2 : 3;
    else face = sz < 0 ? 4 : 5;
    int bc = p->face_bc[face];
    if (bc == OR_BC_VELOCITY) return or_equilibrium(q, p->far[3], p->face_velocity[face]);
    if (bc == OR_BC_OUTFLOW) {
        /* zero gradient: the population the interior neighbour receives */
        int a = face >> 1;
        int sgn = (face & 1) ? 1 : -1;
        int ix = cx - (a == 0 ? sgn : 0), iy = cy - (a == 1 ? sgn : 0), iz = cz - (a == 2 ? sgn : 0);
        int tx = ix - C[q][0], ty = iy - C[q][1], tz = iz - C[q][2];
        if (axis_periodic(p, 0)) tx = tx < 0 ? p->nx - 1 : (tx >= p->nx ? 0 : tx);
        if (axis_periodic(p, 1)) ty = ty < 0 ? p->ny - 1 : (ty >= p->ny ? 0 : ty);
        if (axis_periodic(p, 2)) tz = tz < 0 ? p->nz - 1 : (tz >= p->nz ? 0 : tz);
        if (inside3(p, tx, ty, tz)) {
            int64_t t = flat(p, tx, ty, tz);
            if (mcur[t] == 0) return pin[(int64_t)q * ncells(p) + t];
        }
    }
    return or_equilibrium(q, p->far[3], p->far);
}

/* ------------------------------------------------------------------ */
/* Regularized / RR3 collision (BF.metal:2917-3062).                    */
/* ------------------------------------------------------------------ */
/* The reference's literal per-direction evaluation: the projected
 * second-order non-equilibrium stress summed over q, the third-order
 * Hermite closure per direction, positivity admission and the scaled blend
 * feq + scale (cand - feq) for every direction. */
static void regularized_literal(const float f[19], const float u[3], const float feq[19], float omega_p, int rr3,
                                float post[19], float* act, float* restr) {
    float ds[3] = {0, 0, 0}, od[3] = {0, 0, 0};
    for (int q = 0; q < 19; ++q) {
        float d[3] = {(float)C[q][0], (float)C[q][1], (float)C[q][2]};
        float ne = f[q] - feq[q];
        ds[0] += ne * (d[0] * d[0] - CS2);
        ds[1] += ne * (d[1] * d[1] - CS2);
        ds[2] += ne * (d[2] * d[2] - CS2);
        od[0] += ne * (d[0] * d[1]);
        od[1] += ne * (d[0] * d[2]);
        od[2] += ne * (d[1] * d[2]);
    }
    float aXxy = 2.0f * u[0] * od[0] + u[1] * ds[0];
    float aXxz = 2.0f * u[0] * od[1] + u[2] * ds[0];
    float aXyy = u[0] * ds[1] + 2.0f * u[1] * od[0];
    float aXzz = u[0] * ds[2] + 2.0f * u[2] * od[1];
    float aYyz = 2.0f * u[1] * od[2] + u[2] * ds[1];
    float aYzz = u[1] * ds[2] + 2.0f * u[2] * od[2];
    float unb[19];
    float scale = 1.0f;
    for (int q = 0; q < 19; ++q) {
        float d[3] = {(float)C[q][0], (float)C[q][1], (float)C[q][2]};
        float h[3] = {d[0] * d[0] - CS2, d[1] * d[1] - CS2, d[2] * d[2] - CS2};
        float o[3] = {d[0] * d[1], d[0] * d[2], d[1] * d[2]};
        float contraction = dot3(h, ds) + 2.0f * dot3(o, od);
        float third = 0.0f;
        if (rr3) {
            third = d[1] * (d[0] * d[0] - CS2) * aXxy + d[2] * (d[0] * d[0] - CS2) * aXxz +
                    d[0] * (d[1] * d[1] - CS2) * aXyy + d[0] * (d[2] * d[2] - CS2) * aXzz +
                    d[2] * (d[1] * d[1] - CS2) * aYyz + d[1] * (d[2] * d[2] - CS2) * aYzz;
        }
        float rne = W[q] * 4.5f * contraction;
        if (rr3) rne += W[q] * 13.5f * third;
        float cand = feq[q] + (1.0f - omega_p) * rne;
        unb[q] = cand;
        float floor_ = fmaxf(1.0e-12f, 1.0e-6f * fmaxf(feq[q], 0.0f));
        if (cand < floor_) {
            float adm = clampf((feq[q] - floor_) / fmaxf(feq[q] - cand, 1.0e-30f), 0.0f, 1.0f);
            scale = fminf(scale, adm);
        }
    }
    if (scale < 1.0f) {
        *act = 1.0f;
        *restr = 1.0f - scale;
    }
    for (int q = 0; q < 19; ++q) post[q] = feq[q] + scale * (unb[q] - feq[q]);
}

/* The first nonzero term taken as is (or negated), the rest added or
 * subtracted in direction order: sum over the odd (pair-leading) q of
 * c_a(q) v[q] (b < 0) or c_a(q) c_b(q) v[q]. */
static float pair_sum(const float v[19], int a, int b) {
    float r = 0.0f;
    int first = 1;
    for (int q = 1; q < 19; q += 2) {
        const int c = b < 0 ? C[q][a] : C[q][a] * C[q][b];
        if (c == 0) continue;
        if (first) r = c > 0 ? v[q] : -v[q];
        else r = c > 0 ? r + v[q] : r - v[q];
        first = 0;
    }
    return r;
}
/* c_q . u over the nonzero components of c_q. */
static float cdot_nz(int q, const float u[3]) {
    float r = 0.0f;
    int first = 1;
    for (int k = 0; k < 3; ++k) {
        if (C[q][k] == 0) continue;
        if (first) r = C[q][k] > 0 ? u[k] : -u[k];
        else r = C[q][k] > 0 ? r + u[k] : r - u[k];
        first = 0;
    }
    return r;
}

/* The same operator evaluated on opposite-direction pairs (q odd, q + 1 =
 * OPP[q]), the order the FP32 fluid kernel uses:
 *   moments from pair sums p = f_q + f_q' and differences m = f_q - f_q';
 *   feq_q = E + O, feq_q' = E - O with E = w rho (1 - 1.5u^2 + 4.5cu^2),
 *   O = 3 w rho cu;
 *   stress from the pair non-equilibria n = p - 2E:
 *   ds_a = sum_{c_a != 0} n - cs2 (ne_0 + sum n), od_ab = sum sign(c_a c_b) n;
 *   post_q = X + Y, post_q' = X - Y with X = E + (1 - w+) w 4.5 (H2 : ds),
 *   Y = O + (1 - w+) w 13.5 (H3 : a3).
 * Mathematically the literal operator; the two orders agree to FP32
 * rounding.  The scaled blend runs only where the admission scale is below
 * one (a blend with scale 1 is the identity up to rounding). */
static void regularized_pairs(const float f[19], float omega_p, int rr3, float post[19], float* act, float* restr) {
    float ps[19], md[19], E[19], O[19], nps[19];
    float rho = f[0];
    for (int q = 1; q < 19; q += 2) {
        ps[q] = f[q] + f[q + 1];
        md[q] = f[q] - f[q + 1];
        rho = rho + ps[q];
    }
    const float mx = pair_sum(md, 0, -1), my = pair_sum(md, 1, -1), mz = pair_sum(md, 2, -1);
    rho = rho > 1.0e-8f ? rho : 1.0e-8f;
    const float u[3] = {mx / rho, my / rho, mz / rho};
    const float u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float base = 1.0f - 1.5f * u2;
    const float wr1 = W1 * rho, wr2 = W2 * rho;
    const float feq0 = (W0 * rho) * base;
    float ntot = f[0] - feq0;
    for (int q = 1; q < 19; q += 2) {
        const float cu = cdot_nz(q, u);
        const float wr = q <= 6 ? wr1 : wr2;
        E[q] = wr * (base + (4.5f * cu) * cu);
        O[q] = wr * (3.0f * cu);
        nps[q] = ps[q] - 2.0f * E[q];
        ntot = ntot + nps[q];
    }
    const float dsx = pair_sum(nps, 0, 0) - CS2 * ntot;
    const float dsy = pair_sum(nps, 1, 1) - CS2 * ntot;
    const float dsz = pair_sum(nps, 2, 2) - CS2 * ntot;
    const float odx = pair_sum(nps, 0, 1), ody = pair_sum(nps, 0, 2), odz = pair_sum(nps, 1, 2);
    const float aXxy = (2.0f * u[0]) * odx + u[1] * dsx;
    const float aXxz = (2.0f * u[0]) * ody + u[2] * dsx;
    const float aXyy = u[0] * dsy + (2.0f * u[1]) * odx;
    const float aXzz = u[0] * dsz + (2.0f * u[2]) * ody;
    const float aYyz = (2.0f * u[1]) * odz + u[2] * dsy;
    const float aYzz = u[1] * dsz + (2.0f * u[2]) * odz;
    const float trace = dsx + dsy + dsz;
    const float cax = dsx - CS2 * trace, cay = dsy - CS2 * trace, caz = dsz - CS2 * trace;
    const float om = 1.0f - omega_p;
    const float om0 = om * (W0 * 4.5f * -CS2);
    const float om1 = om * (W1 * 4.5f), om2 = om * (W2 * 4.5f);
    const float ot1 = om * (W1 * 13.5f), ot2 = om * (W2 * 13.5f);
    float fe[19];
    fe[0] = feq0;
    post[0] = feq0 + om0 * trace;
    for (int q = 1; q < 19; q += 2) {
        const int x = C[q][0], y = C[q][1], z = C[q][2];
        float contraction;
        if (x != 0 && y != 0) contraction = (cax + dsy) + 2.0f * (x * y > 0 ? odx : -odx);
        else if (x != 0 && z != 0) contraction = (cax + dsz) + 2.0f * (x * z > 0 ? ody : -ody);
        else if (y != 0 && z != 0) contraction = (cay + dsz) + 2.0f * (y * z > 0 ? odz : -odz);
        else contraction = x != 0 ? cax : (y != 0 ? cay : caz);
        const float X = E[q] + (q <= 6 ? om1 : om2) * contraction;
        float Y = O[q];
        if (rr3) {
            const float hx = (float)(x * x) - CS2, hy = (float)(y * y) - CS2, hz = (float)(z * z) - CS2;
            const int da[6] = {y, z, x, x, z, y};
            const float hb[6] = {hx, hx, hy, hz, hy, hz};
            const float amp[6] = {aXxy, aXxz, aXyy, aXzz, aYyz, aYzz};
            float third = 0.0f;
            int any = 0;
            for (int k = 0; k < 6; ++k) {
                if (da[k] == 0) continue;
                const float t = ((float)da[k] * hb[k]) * amp[k];
                third = any ? third + t : t;
                any = 1;
            }
            Y = Y + (q <= 6 ? ot1 : ot2) * third;
        }
        post[q] = X + Y;
        post[q + 1] = X - Y;
        fe[q] = E[q] + O[q];
        fe[q + 1] = E[q] - O[q];
    }
    float scale = 1.0f;
    for (int q = 0; q < 19; ++q) {
        const float fl = 1.0e-6f * (fe[q] > 0.0f ? fe[q] : 0.0f);
        const float floor_ = 1.0e-12f > fl ? 1.0e-12f : fl;
        if (post[q] < floor_) {
            float den = fe[q] - post[q];
            den = den > 1.0e-30f ? den : 1.0e-30f;
            float adm = (fe[q] - floor_) / den;
            adm = adm < 0.0f ? 0.0f : (adm > 1.0f ? 1.0f : adm);
            scale = scale < adm ? scale : adm;
        }
    }
    if (scale < 1.0f) {
        *act = 1.0f;
        *restr = 1.0f - scale;
        for (int q = 0; q < 19; ++q) post[q] = fe[q] + scale * (post[q] - fe[q]);
    }
}

void or_collide_regularized(int order, const float* f, float omega_p, int rr3, float* post, float* activation,
                            float* restriction) {
    *activation = 0.0f;
    *restriction = 0.0f;
    if (order == 1) {
        regularized_pairs(f, omega_p, rr3, post, activation, restriction);
        return;
    }
    float rho = 0.0f, mom[3] = {0.0f, 0.0f, 0.0f};
    for (int q = 0; q < 19; ++q) {
        rho += f[q];
        mom[0] += f[q] * (float)C[q][0];
        mom[1] += f[q] * (float)C[q][1];
        mom[2] += f[q] * (float)C[q][2];
    }
    rho = fmaxf(rho, 1.0e-8f);
    const float u[3] = {mom[0] / rho, mom[1] / rho, mom[2] / rho};
    float feq[19];
    for (int q = 0; q < 19; ++q) feq[q] = or_equilibrium(q, rho, u);
    regularized_literal(f, u, feq, omega_p, rr3, post, activation, restriction);
}

/* ------------------------------------------------------------------ */
/* stepFluidTRT: BF.metal:2507-3236 (all branches).                     */
/* ------------------------------------------------------------------ */
void or_step(const or_params* p, const float* pin, float* pout,
             const uint8_t* mprev, const uint8_t* mcur, const float* wall, const float* covered,
             float* density, float* velocity, const float body_f[3], const double body_d[3],
             or_loads* loads, float* per_cell_loads) {
    const int64_t n = ncells(p);
    const int nz = p->nz;
    const int accumulate = p->accumulate_loads != 0;
    const int sel = p->interpolated != 0;
    const int comp = sel ? p->load_component : 0;
    const int mode = sel ? p->force_mode : 6;
    const int include_link = !sel || comp != 2;
    const int include_topo = !sel || comp != 1;
    const int coll = p->collision;
    const int rr3 = coll == OR_COLLISION_RR3;
    const int regularized = coll == OR_COLLISION_RR3 || coll == OR_COLLISION_REGULARIZED;
    const int limiter = coll == OR_COLLISION_TRT_LIMITER;
    const float omega_p = p->omega_p, omega_m = p->omega_m;
    const float f2p = p->f2p;
    const int per[3] = {axis_periodic(p, 0), axis_periodic(p, 1), axis_periodic(p, 2)};

    acc64* slab = (acc64*)calloc((size_t)nz, sizeof(acc64));

#pragma omp parallel for schedule(dynamic, 1)
    for (int z = 0; z < nz; ++z) {
        acc64 acc;
        memset(&acc, 0, sizeof(acc));
        for (int y = 0; y < p->ny; ++y) {
            for (int x = 0; x < p->nx; ++x) {
                const int64_t gid = flat(p, x, y, z);
                float world[3];
                cell_world(p, x, y, z, world);
                const int was_solid = mprev[gid] != 0;
                const int is_solid = mcur[gid] != 0;
                float cell_force[3] = {0, 0, 0}, cell_torque[3] = {0, 0, 0};
                float limiter_activation = 0.0f, limiter_restriction = 0.0f;

                if (is_solid) {
                    float w[3] = {wall[4 * gid], wall[4 * gid + 1], wall[4 * gid + 2]};
                    for (int q = 0; q < 19; ++q) pout[q * n + gid] = or_equilibrium(q, 1.0f, w);
                    if (accumulate && !was_solid && include_topo) {
                        float pd = 0.0f, pm[3] = {0, 0, 0};
                        if (sel) {
                            pm[0] = covered[4 * gid];
                            pm[1] = covered[4 * gid + 1];
                            pm[2] = covered[4 * gid + 2];
                            pd = covered[4 * gid + 3];
                        } else {
                            for (int q = 0; q < 19; ++q) {
                                float prev = pin[q * n + gid];
                                pd += prev;
                                pm[0] += prev * (float)C[q][0];
                                pm[1] += prev * (float)C[q][1];
                                pm[2] += prev * (float)C[q][2];
                            }
                        }
                        float imp[3];
                        if (mode == 6) {
                            imp[0] = pm[0];
                            imp[1] = pm[1];
                            imp[2] = pm[2];
                        } else {
                            imp[0] = pm[0] - pd * w[0];
                            imp[1] = pm[1] - pd * w[1];
                            imp[2] = pm[2] - pd * w[2];
                        }
                        cell_force[0] = imp[0] * f2p;
                        cell_force[1] = imp[1] * f2p;
                        cell_force[2] = imp[2] * f2p;
                        float r[3] = {world[0] - body_f[0], world[1] - body_f[1], world[2] - body_f[2]};
                        cross3(r, cell_force, cell_torque);
                        acc_add(&acc, imp, world, body_d, f2p);
                        acc.covered++;
                    }
                    if (p->capture_fields) {
                        density[gid] = 1.0f;
                        velocity[4 * gid] = w[0];
                        velocity[4 * gid + 1] = w[1];
                        velocity[4 * gid + 2] = w[2];
                        velocity[4 * gid + 3] = 0.0f;
                    }
                } else {
                    float f[19];
                    float rho = 0.0f, mom[3] = {0, 0, 0};
                    float fbl[3] = {0, 0, 0}; /* forceOnBodyLattice */

                    if (was_solid) {
                        float rv[3] = {wall[4 * gid], wall[4 * gid + 1], wall[4 * gid + 2]};
                        for (int q = 0; q < 19; ++q) {
                            float v = or_equilibrium(q, 1.0f, rv);
                            f[q] = v;
                            rho += v;
                            mom[0] += v * (float)C[q][0];
                            mom[1] += v * (float)C[q][1];
                            mom[2] += v * (float)C[q][2];
                        }
                        if (accumulate && include_topo && mode == 6) {
                            float topo[3] = {-mom[0], -mom[1], -mom[2]};
                            for (int q = 1; q < 19; ++q) {
                                int bx = x + C[q][0], by = y + C[q][1], bz = z + C[q][2];
                                if (!inside3(p, bx, by, bz)) continue;
                                int64_t nb = flat(p, bx, by, bz);
                                if (!(mprev[nb] == 0 && mcur[nb] == 0)) continue;
                                float old_out = pin[q * n + gid];
                                float sup_in = pin[OPP[q] * n + nb];
                                float s = old_out + sup_in;
                                topo[0] -= s * (float)C[q][0];
                                topo[1] -= s * (float)C[q][1];
                                topo[2] -= s * (float)C[q][2];
                            }
                            fbl[0] += topo[0];
                            fbl[1] += topo[1];
                            fbl[2] += topo[2];
                            float tp[3] = {topo[0] * f2p, topo[1] * f2p, topo[2] * f2p};
                            float r[3] = {world[0] - body_f[0], world[1] - body_f[1], world[2] - body_f[2]};
                            float tq[3];
                            cross3(r, tp, tq);
                            cell_torque[0] += tq[0];
                            cell_torque[1] += tq[1];
                            cell_torque[2] += tq[2];
                            acc_add(&acc, topo, world, body_d, f2p);
                            acc.uncovered++;
                        }
                    } else {
                        float mwd = p->far[3];
                        if (p->local_density) {
                            mwd = 0.0f;
                            for (int q = 0; q < 19; ++q) mwd += pin[q * n + gid];
                        }
                        int interior = x > 0 && y > 0 && z > 0 && x + 1 < p->nx && y + 1 < p->ny && z + 1 < p->nz;
                        for (int q = 0; q < 19; ++q) {
                            int sx = x - C[q][0], sy = y - C[q][1], sz = z - C[q][2];
                            float value;
                            int outside = 0;
                            if (!interior && !inside3(p, sx, sy, sz)) {
                                if (per[0]) sx = sx < 0 ? p->nx - 1 : (sx >= p->nx ? 0 : sx);
                                if (per[1]) sy = sy < 0 ? p->ny - 1 : (sy >= p->ny ? 0 : sy);
                                if (per[2]) sz = sz < 0 ? p->nz - 1 : (sz >= p->nz ? 0 : sz);
                                outside = !inside3(p, sx, sy, sz);
                            }
                            if (outside) {
                                value = outside_value(p, q, x, y, z, sx, sy, sz, pin, mcur);
                            } else {
                                int64_t src = flat(p, sx, sy, sz);
                                uint8_t part = mcur[src];
                                if (part != 0) {
                                    float reflected = pin[OPP[q] * n + gid];
                                    float dir[3] = {(float)C[q][0], (float)C[q][1], (float)C[q][2]};
                                    float qf = 0.5f;
                                    float wv[3] = {wall[4 * src], wall[4 * src + 1], wall[4 * src + 2]};
                                    int64_t farther = 0;
                                    int interp = sel;
                                    if (interp) {
                                        qf = clampf(pin[q * n + src], 1.0e-4f, 1.0f);
                                        for (int k = 0; k < 3; ++k) wv[k] = mixf(wall[4 * gid + k], wall[4 * src + k], qf);
                                        if (qf <= 0.5f) {
                                            int fx = x + C[q][0], fy = y + C[q][1], fz = z + C[q][2];
                                            int fin = inside3(p, fx, fy, fz);
                                            if (fin) farther = flat(p, fx, fy, fz);
                                            if (!fin || mcur[farther] != 0) {
                                                interp = 0;
                                                qf = 0.5f;
                                                wv[0] = wall[4 * src];
                                                wv[1] = wall[4 * src + 1];
                                                wv[2] = wall[4 * src + 2];
                                            }
                                        }
                                    }
                                    float wc = 2.0f * W[q] * mwd * dot3(dir, wv) / CS2;
                                    value = reflected + wc;
                                    if (interp) {
                                        if (qf <= 0.5f) {
                                            float fo = pin[OPP[q] * n + farther];
                                            value = 2.0f * qf * reflected + (1.0f - 2.0f * qf) * fo + wc;
                                        } else {
                                            float pi_ = pin[q * n + gid];
                                            value = (reflected + wc) / (2.0f * qf) + (2.0f * qf - 1.0f) * pi_ / (2.0f * qf);
                                        }
                                    }
                                    if (accumulate && include_link &&
                                        (p->selected_part == 0 || p->selected_part == (int)part)) {
                                        float lf[3];
                                        for (int k = 0; k < 3; ++k) {
                                            switch (mode) {
                                            case 0: lf[k] = -(value * (dir[k] - wv[k]) - reflected * (-dir[k] - wv[k])); break;
                                            case 1:
                                            case 6: lf[k] = -(value + reflected) * dir[k]; break;
                                            case 2: lf[k] = -2.0f * reflected * dir[k]; break;
                                            case 3: lf[k] = -wc * dir[k]; break;
                                            case 4: lf[k] = -(value - reflected - wc) * dir[k]; break;
                                            case 5: lf[k] = (value - reflected) * wv[k]; break;
                                            default: lf[k] = 0.0f; break;
                                            }
                                        }
                                        fbl[0] += lf[0];
                                        fbl[1] += lf[1];
                                        fbl[2] += lf[2];
                                        float lp[3] = {lf[0] * f2p, lf[1] * f2p, lf[2] * f2p};
                                        float bp[3];
                                        for (int k = 0; k < 3; ++k) bp[k] = world[k] - qf * dir[k] * p->dx;
                                        float r[3] = {bp[0] - body_f[0], bp[1] - body_f[1], bp[2] - body_f[2]};
                                        float tq[3];
                                        cross3(r, lp, tq);
                                        cell_torque[0] += tq[0];
                                        cell_torque[1] += tq[1];
                                        cell_torque[2] += tq[2];
                                        acc_add(&acc, lf, bp, body_d, f2p);
                                        acc.links++;
                                    }
                                } else {
                                    value = pin[q * n + src];
                                }
                            }
                            f[q] = value;
                            rho += value;
                            mom[0] += value * (float)C[q][0];
                            mom[1] += value * (float)C[q][1];
                            mom[2] += value * (float)C[q][2];
                        }
                    }

                    rho = fmaxf(rho, 1.0e-8f);
                    float u[3] = {mom[0] / rho, mom[1] / rho, mom[2] / rho};
                    float feq[19];
                    for (int q = 0; q < 19; ++q) feq[q] = or_equilibrium(q, rho, u);
                    float sponge = sponge_factor(p, x, y, z);
                    float cd = 0.0f, cm[3] = {0, 0, 0};
                    float post_all[19];

                    if (regularized) {
                        /* BF.metal:2917-3062, in the pair order of regularized_pairs */
                        regularized_pairs(f, omega_p, rr3, post_all, &limiter_activation, &limiter_restriction);
                    } else if (!limiter) {
                        /* TRT: BF.metal:3063-3093 */
                        for (int q = 0; q < 19; ++q) {
                            int qo = OPP[q];
                            float fp = 0.5f * (f[q] + f[qo]);
                            float fm = 0.5f * (f[q] - f[qo]);
                            float ep = 0.5f * (feq[q] + feq[qo]);
                            float em = 0.5f * (feq[q] - feq[qo]);
                            post_all[q] = f[q] - omega_p * (fp - ep) - omega_m * (fm - em);
                        }
                    } else {
                        /* symmetric positivity limiter: BF.metal:3094-3174 */
                        float si[19], ai[19], sscale = 1.0f;
                        for (int q = 0; q < 19; ++q) {
                            int qo = OPP[q];
                            float fp = 0.5f * (f[q] + f[qo]);
                            float fm = 0.5f * (f[q] - f[qo]);
                            float ep = 0.5f * (feq[q] + feq[qo]);
                            float em = 0.5f * (feq[q] - feq[qo]);
                            float s = -omega_p * (fp - ep);
                            float a = -omega_m * (fm - em);
                            si[q] = s;
                            ai[q] = a;
                            if (s < 0.0f) {
                                float base = f[q] + a;
                                float floor_ = fmaxf(1.0e-12f, 1.0e-6f * fmaxf(feq[q], 0.0f));
                                if (base + s < floor_) {
                                    float cand = clampf((base - floor_) / fmaxf(-s, 1.0e-30f), 0.0f, 1.0f);
                                    sscale = fminf(sscale, cand);
                                }
                            }
                        }
                        if (sscale < 1.0f) {
                            limiter_activation = 1.0f;
                            limiter_restriction = 1.0f - sscale;
                        }
                        for (int q = 0; q < 19; ++q) {
                            if (sscale < 1.0f) {
                                post_all[q] = f[q] + sscale * si[q] + ai[q];
                            } else {
                                int qo = OPP[q];
                                float fp = 0.5f * (f[q] + f[qo]);
                                float fm = 0.5f * (f[q] - f[qo]);
                                float ep = 0.5f * (feq[q] + feq[qo]);
                                float em = 0.5f * (feq[q] - feq[qo]);
                                post_all[q] = f[q] - omega_p * (fp - ep) - omega_m * (fm - em);
                            }
                        }
                    }

                    for (int q = 0; q < 19; ++q) {
                        float post = post_all[q];
                        if (sponge > 0.0f) {
                            float farv = or_equilibrium(q, p->far[3], p->far);
                            post = mixf(post, farv, sponge);
                        }
                        pout[q * n + gid] = post;
                        if (p->capture_fields) {
                            cd += post;
                            cm[0] += post * (float)C[q][0];
                            cm[1] += post * (float)C[q][1];
                            cm[2] += post * (float)C[q][2];
                        }
                    }
                    if (p->capture_fields) {
                        cd = fmaxf(cd, 1.0e-8f);
                        density[gid] = cd;
                        velocity[4 * gid] = cm[0] / cd;
                        velocity[4 * gid + 1] = cm[1] / cd;
                        velocity[4 * gid + 2] = cm[2] / cd;
                        velocity[4 * gid + 3] = 0.0f;
                    }
                    if (accumulate) {
                        cell_force[0] = fbl[0] * f2p;
                        cell_force[1] = fbl[1] * f2p;
                        cell_force[2] = fbl[2] * f2p;
                    }
                    acc.act += (double)limiter_activation;
                    if ((double)limiter_restriction > acc.rmax) acc.rmax = (double)limiter_restriction;
                }
                if (per_cell_loads) {
                    float* o = per_cell_loads + 8 * gid;
                    o[0] = cell_force[0];
                    o[1] = cell_force[1];
                    o[2] = cell_force[2];
                    o[3] = limiter_activation;
                    o[4] = cell_torque[0];
                    o[5] = cell_torque[1];
                    o[6] = cell_torque[2];
                    o[7] = limiter_restriction;
                }
            }
        }
        slab[z] = acc;
    }

    if (loads) {
        memset(loads, 0, sizeof(*loads));
        for (int z = 0; z < nz; ++z) {
            for (int k = 0; k < 3; ++k) {
                loads->f64_force_lattice[k] += slab[z].f[k];
                loads->f64_torque[k] += slab[z].t[k];
            }
            loads->activation += slab[z].act;
            if (slab[z].rmax > loads->max_restriction) loads->max_restriction = slab[z].rmax;
            loads->link_count += slab[z].links;
            loads->covered_count += slab[z].covered;
            loads->uncovered_count += slab[z].uncovered;
        }
        for (int k = 0; k < 3; ++k) loads->f64_force[k] = loads->f64_force_lattice[k] * (double)f2p;
        if (per_cell_loads && accumulate) {
            /* Reference FP32 reduction: lane-0 ascending sum per 256-cell group,
             * then repeated sequential 256-way passes. */
            int64_t groups = (n + 255) / 256;
            float* part = (float*)malloc((size_t)groups * 8 * sizeof(float));
            for (int64_t g = 0; g < groups; ++g) {
                float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (int64_t i = g * 256; i < g * 256 + 256; ++i) {
                    if (i >= n) break; /* padded lanes contribute zero */
                    const float* o = per_cell_loads + 8 * i;
                    s[0] += o[0];
                    s[1] += o[1];
                    s[2] += o[2];
                    s[3] += o[3];
                    s[4] += o[4];
                    s[5] += o[5];
                    s[6] += o[6];
                    s[7] = fmaxf(s[7], o[7]);
                }
                memcpy(part + 8 * g, s, sizeof(s));
            }
            int64_t count = groups;
            while (count > 1) {
                int64_t next = (count + 255) / 256;
                for (int64_t g = 0; g < next; ++g) {
                    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    for (int64_t i = g * 256; i < g * 256 + 256 && i < count; ++i) {
                        const float* o = part + 8 * i;
                        for (int k = 0; k < 7; ++k) s[k] += o[k];
                        s[7] = fmaxf(s[7], o[7]);
                    }
                    memcpy(part + 8 * g, s, sizeof(s));
                }
                count = next;
            }
            for (int k = 0; k < 4; ++k) {
                loads->f32_force[k] = part[k];
                loads->f32_torque[k] = part[4 + k];
            }
            free(part);
        }
    }
    free(slab);
}

void or_fluid_mass_momentum(const or_params* p, const float* pops, const uint8_t* mask, double out[4]) {
    int64_t n = ncells(p);
    double m = 0, mx = 0, my = 0, mz = 0;
#pragma omp parallel for reduction(+ : m, mx, my, mz) schedule(static)
    for (int64_t gid = 0; gid < n; ++gid) {
        if (mask && mask[gid] != 0) continue;
        for (int q = 0; q < 19; ++q) {
            double v = (double)pops[q * n + gid];
            m += v;
            mx += v * C[q][0];
            my += v * C[q][1];
            mz += v * C[q][2];
        }
    }
    out[0] = m;
    out[1] = mx;
    out[2] = my;
    out[3] = mz;
}

/* ------------------------------------------------------------------ */
/* Quaternion helpers: BF.metal:454-475 (normalize by exact division).  */
/* ------------------------------------------------------------------ */
static void quat_normalize(const float q[4], float r[4]) {
    float n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (n2 > 1.0e-20f) {
        float n = sqrtf(n2);
        for (int k = 0; k < 4; ++k) r[k] = q[k] / n;
    } else {
        r[0] = r[1] = r[2] = 0.0f;
        r[3] = 1.0f;
    }
}
static void quat_rotate(const float q[4], const float v[3], float r[3]) {
    float t[3], c2[3];
    cross3(q, v, t);
    t[0] *= 2.0f;
    t[1] *= 2.0f;
    t[2] *= 2.0f;
    cross3(q, t, c2);
    for (int k = 0; k < 3; ++k) r[k] = v[k] + q[3] * t[k] + c2[k];
}
static void quat_unrotate(const float q[4], const float v[3], float r[3]) {
    float c[4] = {-q[0], -q[1], -q[2], q[3]};
    quat_rotate(c, v, r);
}
/* rotateAroundAxis: BF.metal:466-473 */
static void rotate_axis(const float v[3], const float axis[3], float angle, float r[3]) {
    float s = bfx_sinf(angle), c = bfx_cosf(angle);
    float cr[3];
    cross3(axis, v, cr);
    float d = dot3(axis, v);
    for (int k = 0; k < 3; ++k) r[k] = v[k] * c + cr[k] * s + axis[k] * d * (1.0f - c);
}
static void normalize3(const float v[3], float r[3]) {
    float l = lengthf(v);
    r[0] = v[0] / l;
    r[1] = v[1] / l;
    r[2] = v[2] / l;
}

typedef struct {
    float root[3], chord[3], span[3], normal[3], rel_omega[3], tip_twist, tip_twist_rate;
} wing_frame;

/* makeWingFrame: BF.metal:611-684 */
static void make_wing_frame(float side, float stroke, float stroke_rate, float deviation, float deviation_rate,
                            float pitch, float pitch_rate, float tip_twist, float tip_twist_rate,
                            const or_bird* bird, const float pos[3], const float orient[4], wing_frame* fr) {
    float o[4];
    quat_normalize(orient, o);
    float ex[3] = {1, 0, 0}, ey[3] = {0, 1, 0}, ez[3] = {0, 0, 1};
    float bx[3], by[3], bz[3];
    quat_rotate(o, ex, bx);
    quat_rotate(o, ey, by);
    quat_rotate(o, ez, bz);
    float root_local[3] = {bird->wing_geometry1.v[1], side * bird->wing_geometry1.v[2], bird->wing_geometry1.v[3]};
    float rr[3];
    quat_rotate(o, root_local, rr);
    float root[3] = {pos[0] + rr[0], pos[1] + rr[1], pos[2] + rr[2]};
    float signed_stroke = side * stroke;
    float sby[3] = {side * by[0], side * by[1], side * by[2]};
    float sbz[3] = {side * bz[0], side * bz[1], side * bz[2]};
    float span_after[3], normal_after[3], span[3], chord_before[3], chord[3], normal[3];
    rotate_axis(sby, bx, signed_stroke, span_after);
    rotate_axis(sbz, bx, signed_stroke, normal_after);
    rotate_axis(span_after, normal_after, deviation, span);
    rotate_axis(bx, normal_after, deviation, chord_before);
    float signed_pitch = side * pitch;
    rotate_axis(chord_before, span, signed_pitch, chord);
    rotate_axis(normal_after, span, signed_pitch, normal);
    memcpy(fr->root, root, sizeof(root));
    normalize3(chord, fr->chord);
    normalize3(span, fr->span);
    normalize3(normal, fr->normal);
    for (int k = 0; k < 3; ++k)
        fr->rel_omega[k] = bx[k] * (side * stroke_rate) + normal_after[k] * deviation_rate + fr->span[k] * (side * pitch_rate);
    fr->tip_twist = side * tip_twist;
    fr->tip_twist_rate = side * tip_twist_rate;
}

static void set4(or_f4* d, const float v[3], float w) {
    d->v[0] = v[0];
    d->v[1] = v[1];
    d->v[2] = v[2];
    d->v[3] = w;
}

/* prepareBirdGeometry: BF.metal:686-814 (sinusoidal kinematics; the measured
 * keyframe branch is outside this path). */
void or_prepare_bird(const or_bird* bird, const or_body_f32* body, float time, float dx, or_prepared* out) {
    float af = 2.0f * 3.14159265358979323846f * bird->wing_kinematics0.v[0];
    float phase = af * time;
    float stroke = bird->wing_kinematics0.v[2] + bird->wing_kinematics0.v[1] * bfx_sinf(phase);
    float stroke_rate = af * bird->wing_kinematics0.v[1] * bfx_cosf(phase);
    float pitch = bird->wing_kinematics0.v[3] + bird->wing_kinematics1.v[0] * bfx_sinf(phase + bird->wing_kinematics1.v[1]);
    float pitch_rate = af * bird->wing_kinematics1.v[0] * bfx_cosf(phase + bird->wing_kinematics1.v[1]);
    /* Stroke-plane deviation at twice the flapping frequency, amplitude in
     * wing_kinematics1.z (the library's extension: the reference feeds
     * deviation only from measured keyframes). */
    float deviation = bird->wing_kinematics1.v[2] * bfx_sinf(2.0f * phase);
    float deviation_rate = 2.0f * af * bird->wing_kinematics1.v[2] * bfx_cosf(2.0f * phase);
    wing_frame l, r;
    make_wing_frame(1.0f, stroke, stroke_rate, deviation, deviation_rate, pitch, pitch_rate, 0.0f, 0.0f, bird,
                    body->position, body->orientation, &l);
    make_wing_frame(-1.0f, stroke, stroke_rate, deviation, deviation_rate, pitch, pitch_rate, 0.0f, 0.0f, bird,
                    body->position, body->orientation, &r);
    float o[4];
    quat_normalize(body->orientation, o);
    set4(&out->body_position, body->position, 0.0f);
    memcpy(out->orientation.v, o, sizeof(o));
    set4(&out->linear_velocity, body->velocity, 0.0f);
    const float* br = bird->body_radii_mass.v;
    const float* tg = bird->tail_geometry.v;
    const float* wg0 = bird->wing_geometry0.v;
    const float* wg1 = bird->wing_geometry1.v;
    float body_radius = lengthf(br);
    float tv[3] = {br[0] + tg[0], fmaxf(br[1], tg[1]), br[2] + 0.5f * tg[2]};
    float tail_radius = lengthf(tv);
    float rv[3] = {wg1[1], wg1[2], wg1[3]};
    float root_radius = lengthf(rv);
    float wing_radius = root_radius + wg0[0] + fabsf(wg1[0]) + 0.5f * fmaxf(wg0[1], wg0[2]) + 0.5f * wg0[3];
    float geometry_radius = fmaxf(body_radius, fmaxf(tail_radius, wing_radius)) + 2.0f * dx;
    float obw[3];
    quat_rotate(o, body->omega_body, obw);
    set4(&out->omega_body_world, obw, geometry_radius);
    set4(&out->left_root, l.root, 0.0f);
    set4(&out->left_chord, l.chord, l.tip_twist);
    set4(&out->left_span, l.span, 0.0f);
    set4(&out->left_normal, l.normal, 0.0f);
    set4(&out->left_angular_velocity, l.rel_omega, l.tip_twist_rate);
    set4(&out->right_root, r.root, 0.0f);
    set4(&out->right_chord, r.chord, r.tip_twist);
    set4(&out->right_span, r.span, 0.0f);
    set4(&out->right_normal, r.normal, 0.0f);
    set4(&out->right_angular_velocity, r.rel_omega, r.tip_twist_rate);
}

/* sdEllipsoid / sdTaperedWing / sdTail: BF.metal:486-533 */
static float sd_ellipsoid(const float p[3], const float r[3]) {
    float a[3] = {p[0] / r[0], p[1] / r[1], p[2] / r[2]};
    float r2[3] = {r[0] * r[0], r[1] * r[1], r[2] * r[2]};
    float b[3] = {p[0] / r2[0], p[1] / r2[1], p[2] / r2[2]};
    float k0 = lengthf(a);
    float k1 = lengthf(b);
    return k1 > 1.0e-12f ? k0 * (k0 - 1.0f) / k1 : -fminf(r[0], fminf(r[1], r[2]));
}
static float sd_box_tail(float qx, float qy, float qz) {
    float m[3] = {fmaxf(qx, 0.0f), fmaxf(qy, 0.0f), fmaxf(qz, 0.0f)};
    return lengthf(m) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
}
static float sd_tapered_wing(const float l[3], float span, float root_chord, float tip_chord, float thickness,
                             float sweep) {
    float sf = clampf(l[1] / fmaxf(span, 1.0e-6f), 0.0f, 1.0f);
    float chord = mixf(root_chord, tip_chord, sf);
    float cc = -sweep * sf;
    float dx = fabsf(l[0] - cc) - 0.5f * chord;
    float dy = fmaxf(-l[1], l[1] - span);
    float dz = fabsf(l[2]) - 0.5f * thickness;
    return sd_box_tail(dx, dy, dz);
}
static float sd_tail(const float bl[3], const float br[3], const float tg[4]) {
    float len = tg[0], hw = tg[1], th = tg[2];
    float xr = -(bl[0] + br[0]);
    float fr = clampf(xr / fmaxf(len, 1.0e-6f), 0.0f, 1.0f);
    float lhw = mixf(0.35f * hw, hw, fr);
    float dx = fmaxf(-xr, xr - len);
    float dy = fabsf(bl[1]) - lhw;
    float dz = fabsf(bl[2] + 0.15f * br[2]) - 0.5f * th;
    return sd_box_tail(dx, dy, dz);
}

/* buildBirdGeometry: BF.metal:816-938 */
void or_build_bird(const or_params* p, const or_bird* bird, const or_prepared* prep,
                   const uint8_t* mprev, uint8_t* mnext, float* wall) {
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p->nz; ++z) {
        for (int y = 0; y < p->ny; ++y) {
            for (int x = 0; x < p->nx; ++x) {
                int64_t gid = flat(p, x, y, z);
                float world[3];
                cell_world(p, x, y, z, world);
                float rb[3] = {world[0] - prep->body_position.v[0], world[1] - prep->body_position.v[1],
                               world[2] - prep->body_position.v[2]};
                int was_solid = p->has_prev_geom && mprev[gid] != 0;
                float gr = prep->omega_body_world.v[3];
                if (!was_solid && dot3(rb, rb) > gr * gr) {
                    mnext[gid] = 0;
                    wall[4 * gid] = wall[4 * gid + 1] = wall[4 * gid + 2] = wall[4 * gid + 3] = 0.0f;
                    continue;
                }
                float bl[3];
                quat_unrotate(prep->orientation.v, rb, bl);
                float cr[3];
                cross3(prep->omega_body_world.v, rb, cr);
                float base[3] = {prep->linear_velocity.v[0] + cr[0], prep->linear_velocity.v[1] + cr[1],
                                 prep->linear_velocity.v[2] + cr[2]};
                float best = sd_ellipsoid(bl, bird->body_radii_mass.v);
                float bestv[3] = {base[0], base[1], base[2]};
                int part = 1;
                for (int wing = 0; wing < 2; ++wing) {
                    const or_f4* fr = wing == 0 ? &prep->left_root : &prep->right_root;
                    const float* root = fr[0].v;
                    const float* chord = fr[1].v;
                    const float* span = fr[2].v;
                    const float* normal = fr[3].v;
                    const float* rel = fr[4].v;
                    float tip_twist = fr[1].v[3];
                    float tip_rate = fr[4].v[3];
                    float rel_pos[3] = {world[0] - root[0], world[1] - root[1], world[2] - root[2]};
                    float lu[3] = {dot3(rel_pos, chord), dot3(rel_pos, span), dot3(rel_pos, normal)};
                    float sf = clampf(lu[1] / fmaxf(bird->wing_geometry0.v[0], 1.0e-6f), 0.0f, 1.0f);
                    float twist = tip_twist * sf;
                    float tc = bfx_cosf(twist), ts = bfx_sinf(twist);
                    float loc[3] = {tc * lu[0] + ts * lu[2], lu[1], -ts * lu[0] + tc * lu[2]};
                    float d = sd_tapered_wing(loc, bird->wing_geometry0.v[0], bird->wing_geometry0.v[1],
                                              bird->wing_geometry0.v[2], bird->wing_geometry0.v[3],
                                              bird->wing_geometry1.v[0]);
                    if (d < best) {
                        best = d;
                        float c1[3], c2[3];
                        cross3(rel, rel_pos, c1);
                        float sw[3] = {span[0] * (sf * tip_rate), span[1] * (sf * tip_rate), span[2] * (sf * tip_rate)};
                        float arm[3] = {world[0] - (root[0] + span[0] * lu[1]), world[1] - (root[1] + span[1] * lu[1]),
                                        world[2] - (root[2] + span[2] * lu[1])};
                        cross3(sw, arm, c2);
                        for (int k = 0; k < 3; ++k) bestv[k] = base[k] + c1[k] + c2[k];
                        part = wing == 0 ? 2 : 3;
                    }
                }
                float td = sd_tail(bl, bird->body_radii_mass.v, bird->tail_geometry.v);
                if (td < best) {
                    best = td;
                    bestv[0] = base[0];
                    bestv[1] = base[1];
                    bestv[2] = base[2];
                    part = 4;
                }
                int solid = best <= 0.0f;
                mnext[gid] = solid ? (uint8_t)part : 0;
                wall[4 * gid] = bestv[0] * p->v2l;
                wall[4 * gid + 1] = bestv[1] * p->v2l;
                wall[4 * gid + 2] = bestv[2] * p->v2l;
                wall[4 * gid + 3] = 0.0f;
            }
        }
    }
}

/* Ellipsoid body alone (part 1) with the same rigid wall velocity and the
 * same bounding-sphere rule; w stores the implicit value. */
static float ellipsoid_implicit(const or_params* p, const or_bird* bird, const or_prepared* prep, const float w[3]) {
    (void)p;
    float rb[3] = {w[0] - prep->body_position.v[0], w[1] - prep->body_position.v[1], w[2] - prep->body_position.v[2]};
    float bl[3];
    quat_unrotate(prep->orientation.v, rb, bl);
    return sd_ellipsoid(bl, bird->body_radii_mass.v);
}

void or_build_ellipsoid(const or_params* p, const or_bird* bird, const or_prepared* prep,
                        const uint8_t* mprev, uint8_t* mnext, float* wall) {
    float r = fmaxf(bird->body_radii_mass.v[0], fmaxf(bird->body_radii_mass.v[1], bird->body_radii_mass.v[2])) +
              2.0f * p->dx;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p->nz; ++z) {
        for (int y = 0; y < p->ny; ++y) {
            for (int x = 0; x < p->nx; ++x) {
                int64_t gid = flat(p, x, y, z);
                float world[3];
                cell_world(p, x, y, z, world);
                float rb[3] = {world[0] - prep->body_position.v[0], world[1] - prep->body_position.v[1],
                               world[2] - prep->body_position.v[2]};
                int was_solid = p->has_prev_geom && mprev[gid] != 0;
                if (!was_solid && dot3(rb, rb) > r * r) {
                    mnext[gid] = 0;
                    wall[4 * gid] = wall[4 * gid + 1] = wall[4 * gid + 2] = 0.0f;
                    wall[4 * gid + 3] = r;
                    continue;
                }
                float imp = ellipsoid_implicit(p, bird, prep, world);
                float cr[3];
                cross3(prep->omega_body_world.v, rb, cr);
                mnext[gid] = imp <= 0.0f ? 1 : 0;
                wall[4 * gid] = (prep->linear_velocity.v[0] + cr[0]) * p->v2l;
                wall[4 * gid + 1] = (prep->linear_velocity.v[1] + cr[1]) * p->v2l;
                wall[4 * gid + 2] = (prep->linear_velocity.v[2] + cr[2]) * p->v2l;
                wall[4 * gid + 3] = imp;
            }
        }
    }
}

/* Ten-iteration bracketed bisection from the fluid node toward the solid node,
 * the reference's prescribedWingLinkFraction rule (BF.metal:1144-1175)
 * applied to the ellipsoid implicit. */
float or_ellipsoid_link_fraction(const or_params* p, const or_bird* bird, const or_prepared* prep,
                                 int fx, int fy, int fz, int sx, int sy, int sz) {
    float fw[3], sw[3];
    cell_world(p, fx, fy, fz, fw);
    cell_world(p, sx, sy, sz, sw);
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 10; ++it) {
        float mid = 0.5f * (lo + hi);
        float s[3] = {mixf(fw[0], sw[0], mid), mixf(fw[1], sw[1], mid), mixf(fw[2], sw[2], mid)};
        if (ellipsoid_implicit(p, bird, prep, s) > 0.0f) lo = mid;
        else hi = mid;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

/* ------------------------------------------------------------------ */
/* Coupled momentum ledger: measureFluidMassMomentumChange and          */
/* captureExternalFluidSources (BF.metal:4322-4552).  The reference     */
/* forms each cell's terms in FP32 and sums FP32 threadgroup partials;  */
/* the library (and this restatement) forms them in FP64 from the FP32  */
/* populations and sums in FP64.                                        */
/* ------------------------------------------------------------------ */
void or_ledger_sources(const or_params* p, const float* pin, const float* pout, const uint8_t* mprev,
                       const uint8_t* mcur, const float* wall, double out[24]) {
    const int64_t n = ncells(p);
    double acc[24] = {0};
    const int periodic_any = axis_periodic(p, 0) || axis_periodic(p, 1) || axis_periodic(p, 2);
#pragma omp parallel
    {
        double loc[24] = {0};
#pragma omp for schedule(static)
        for (int z = 0; z < p->nz; ++z) {
            for (int y = 0; y < p->ny; ++y) {
                for (int x = 0; x < p->nx; ++x) {
                    int64_t gid = flat(p, x, y, z);
                    int was_solid = mprev[gid] != 0, is_solid = mcur[gid] != 0;
                    /* measureFluidMassMomentumChange: cells that were fluid before, that are fluid after */
                    for (int q = 0; q < 19; ++q) {
                        if (!was_solid) {
                            double v = pin[(int64_t)q * n + gid];
                            loc[0] += v;
                            loc[1] += v * C[q][0];
                            loc[2] += v * C[q][1];
                            loc[3] += v * C[q][2];
                        }
                        if (!is_solid) {
                            double v = pout[(int64_t)q * n + gid];
                            loc[4] += v;
                            loc[5] += v * C[q][0];
                            loc[6] += v * C[q][1];
                            loc[7] += v * C[q][2];
                        }
                    }
                    if (was_solid != is_solid) loc[23] += 1.0;
                    if (is_solid) continue;
                    int persistent_target = !was_solid;
                    double mwd = p->far[3];
                    if (p->local_density) {
                        mwd = 0.0;
                        for (int q = 0; q < 19; ++q) mwd += pin[(int64_t)q * n + gid];
                    }
                    int interior = x > 0 && y > 0 && z > 0 && x + 1 < p->nx && y + 1 < p->ny && z + 1 < p->nz;
                    for (int q = 0; q < 19; ++q) {
                        int sx = x - C[q][0], sy = y - C[q][1], sz = z - C[q][2];
                        int outside = !interior && !inside3(p, sx, sy, sz);
                        if (outside && !periodic_any) {
                            /* open face: the reference's far-field rule; a velocity or outflow face
                               brings in the value the step pulls there, as the library's faces do */
                            double incoming = outside_value(p, q, x, y, z, sx, sy, sz, pin, mcur);
                            double outgoing = pin[(int64_t)OPP[q] * n + gid];
                            loc[8] += incoming - outgoing;
                            loc[9] += (incoming + outgoing) * C[q][0];
                            loc[10] += (incoming + outgoing) * C[q][1];
                            loc[11] += (incoming + outgoing) * C[q][2];
                            loc[20] += 1.0;
                            continue;
                        }
                        if (outside) {
                            sx = sx < 0 ? p->nx - 1 : (sx >= p->nx ? 0 : sx);
                            sy = sy < 0 ? p->ny - 1 : (sy >= p->ny ? 0 : sy);
                            sz = sz < 0 ? p->nz - 1 : (sz >= p->nz ? 0 : sz);
                        }
                        int64_t src = flat(p, sx, sy, sz);
                        if (persistent_target && mcur[src] != 0 && mprev[src] != 0) {
                            /* halfway moving-wall reflection, the reference's ledger rule */
                            double reflected = pin[(int64_t)OPP[q] * n + gid];
                            double cu = C[q][0] * (double)wall[4 * src] + C[q][1] * (double)wall[4 * src + 1] +
                                        C[q][2] * (double)wall[4 * src + 2];
                            double wc = 2.0 * (double)W[q] * mwd * cu / (double)CS2;
                            double incoming = reflected + wc;
                            loc[12] += incoming - reflected;
                            loc[13] += (incoming + reflected) * C[q][0];
                            loc[14] += (incoming + reflected) * C[q][1];
                            loc[15] += (incoming + reflected) * C[q][2];
                            loc[22] += 1.0;
                        }
                    }
                    float sponge = sponge_factor(p, x, y, z);
                    if (sponge > 0.0f) {
                        double inv = 1.0 / fmax(1.0 - (double)sponge, 1.0e-7);
                        for (int q = 0; q < 19; ++q) {
                            double actual = pout[(int64_t)q * n + gid];
                            double far = or_equilibrium(q, p->far[3], p->far);
                            double d = (double)sponge * (far - actual) * inv;
                            loc[16] += d;
                            loc[17] += d * C[q][0];
                            loc[18] += d * C[q][1];
                            loc[19] += d * C[q][2];
                        }
                        loc[21] += 1.0;
                    }
                }
            }
        }
#pragma omp critical
        for (int k = 0; k < 24; ++k) acc[k] += loc[k];
    }
    for (int k = 0; k < 24; ++k) out[k] = acc[k];
}

/* ------------------------------------------------------------------ */
/* Prescribed flapping wing (Li-Nabawy beta planform): the analytic      */
/* geometry of MetalFlappingWingValidation (BF.metal:940-1297).          */
/* ------------------------------------------------------------------ */
/* unitCyclePhase: BF.metal:940-943 */
static float wing_unit_phase(float time, float cycle_steps) {
    float phase = fmodf(time / cycle_steps, 1.0f);
    return phase < 0.0f ? phase + 1.0f : phase;
}

/* prescribedStrokeKinematics: BF.metal:945-1001 (angle, rate per cycle) */
static void wing_stroke(float phase, const or_wing* w, float out[2]) {
    const float pi = 3.14159265358979323846f;
    float amplitude = w->kinematics0.v[1], duration = w->kinematics0.v[2];
    float half = 0.5f * duration, max_rate = w->kinematics1.v[2];
    if (phase < half) {
        float arg = pi * (phase + half) / duration;
        out[0] = amplitude + max_rate * duration / pi * (bfx_sinf(arg) - 1.0f);
        out[1] = max_rate * bfx_cosf(arg);
    } else if (phase < 0.5f - half) {
        float at_end = amplitude - max_rate * duration / pi;
        out[0] = at_end - max_rate * (phase - half);
        out[1] = -max_rate;
    } else if (phase < 0.5f + half) {
        float start = 0.5f - half;
        float at_start = -amplitude + max_rate * duration / pi;
        float arg = pi * (phase - start) / duration;
        out[0] = at_start - max_rate * duration / pi * bfx_sinf(arg);
        out[1] = -max_rate * bfx_cosf(arg);
    } else if (phase < 1.0f - half) {
        float at_end = -amplitude + max_rate * duration / pi;
        out[0] = at_end + max_rate * (phase - (0.5f + half));
        out[1] = max_rate;
    } else {
        float start = 1.0f - half;
        float at_start = amplitude - max_rate * duration / pi;
        float arg = pi * (phase - start) / duration;
        out[0] = at_start + max_rate * duration / pi * bfx_sinf(arg);
        out[1] = max_rate * bfx_cosf(arg);
    }
}

/* prescribedPitchKinematics: BF.metal:1003-1035 */
static void wing_pitch(float phase, const or_wing* w, float out[2]) {
    const float pi = 3.14159265358979323846f;
    float duration = w->kinematics0.v[3], half = 0.5f * duration;
    float low = w->kinematics1.v[0], high = w->kinematics1.v[1], delta = high - low;
    float x, start, change;
    if (phase < half || phase >= 1.0f - half) {
        float wrapped = phase < half ? phase + 1.0f : phase;
        x = (wrapped - (1.0f - half)) / duration;
        start = high;
        change = -delta;
    } else if (phase >= 0.5f - half && phase < 0.5f + half) {
        x = (phase - (0.5f - half)) / duration;
        start = low;
        change = delta;
    } else {
        out[0] = phase < 0.5f ? low : high;
        out[1] = 0.0f;
        return;
    }
    float blend = x - bfx_sinf(2.0f * pi * x) / (2.0f * pi);
    out[1] = change / duration * (1.0f - bfx_cosf(2.0f * pi * x));
    out[0] = start + change * blend;
}

/* preparePrescribedFlappingWing: BF.metal:1038-1078.  time is the absolute
 * step index (the reference passes Float(absoluteStep)). */
void or_prepare_wing(const or_wing* w, float time, or_wing_prepared* out) {
    float cycle_steps = w->kinematics0.v[0];
    float phase = wing_unit_phase(time, cycle_steps);
    float stroke[2], pitch[2];
    wing_stroke(phase, w, stroke);
    wing_pitch(phase, w, pitch);
    const float axis[3] = {0.0f, 0.0f, 1.0f};
    float span[3] = {bfx_cosf(stroke[0]), bfx_sinf(stroke[0]), 0.0f};
    float tangent[3], chord[3], cn[3], normal[3], sn[3];
    cross3(axis, span, tangent);
    rotate_axis(tangent, span, -pitch[0], chord);
    cross3(span, chord, cn);
    normalize3(cn, normal);
    float inv = 1.0f / cycle_steps;
    float omega[3];
    for (int k = 0; k < 3; ++k) omega[k] = axis[k] * (stroke[1] * inv) - span[k] * (pitch[1] * inv);
    out->root = w->root_and_chord;
    normalize3(chord, cn);
    set4(&out->chord, cn, 0.0f);
    normalize3(span, sn);
    set4(&out->span, sn, 0.0f);
    set4(&out->normal, normal, 0.0f);
    set4(&out->angular_velocity, omega, 0.0f);
    out->state.v[0] = stroke[0];
    out->state.v[1] = pitch[0];
    out->state.v[2] = stroke[1] * inv;
    out->state.v[3] = pitch[1] * inv;
}

/* prescribedWingBoundaryCoordinates + prescribedWingMaximumViolation:
 * BF.metal:1091-1142.  Positive outside the wing. */
float or_wing_violation(const or_params* p, const or_wing* w, const or_wing_prepared* pw, const float world[3]) {
    float rel[3] = {world[0] - pw->root.v[0], world[1] - pw->root.v[1], world[2] - pw->root.v[2]};
    float radial = dot3(rel, pw->span.v), normal = dot3(rel, pw->normal.v), chord = dot3(rel, pw->chord.v);
    float radius = w->geometry.v[0], chord_mean = w->root_and_chord.v[3];
    float half = 0.5f * fmaxf(w->geometry.v[1], p->dx);
    float fraction = clampf(radial / radius, 0.0f, 1.0f);
    float beta_base = fmaxf(fraction * (1.0f - fraction), 0.0f);
    float local_chord = chord_mean * w->geometry.v[3] * bfx_powf(beta_base, w->geometry.v[2]);
    float leading = -0.25f * chord_mean;
    float root_v = -radial, tip_v = radial - radius, normal_v = fabsf(normal) - half;
    float lead_v = leading - chord, trail_v = chord - (leading + local_chord);
    return fmaxf(fmaxf(root_v, tip_v), fmaxf(normal_v, fmaxf(lead_v, trail_v)));
}

/* buildPrescribedFlappingWing, classification part: BF.metal:1179-1249.
 * Part id 1; wall = rigid rotation about the root (lattice velocity, the
 * reference's lengths are in cells), w = -1 solid / +1 fluid, (0, 0, 0,
 * radius) outside the bounding sphere. */
void or_build_wing(const or_params* p, const or_wing* w, const or_wing_prepared* pw, const uint8_t* mprev,
                   uint8_t* mnext, float* wall) {
    float chord_mean = w->root_and_chord.v[3];
    float radius = w->geometry.v[0] + 1.5f * chord_mean + 2.0f * p->dx;
    float half = 0.5f * fmaxf(w->geometry.v[1], p->dx);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p->nz; ++z) {
        for (int y = 0; y < p->ny; ++y) {
            for (int x = 0; x < p->nx; ++x) {
                int64_t gid = flat(p, x, y, z);
                float world[3];
                cell_world(p, x, y, z, world);
                float rel[3] = {world[0] - pw->root.v[0], world[1] - pw->root.v[1], world[2] - pw->root.v[2]};
                int was_solid = p->has_prev_geom && mprev[gid] != 0;
                if (!was_solid && dot3(rel, rel) > radius * radius) {
                    mnext[gid] = 0;
                    wall[4 * gid] = wall[4 * gid + 1] = wall[4 * gid + 2] = 0.0f;
                    wall[4 * gid + 3] = radius;
                    continue;
                }
                float cc = dot3(rel, pw->chord.v), rc = dot3(rel, pw->span.v), nc = dot3(rel, pw->normal.v);
                int in_radial = rc >= 0.0f && rc <= w->geometry.v[0];
                int in_normal = fabsf(nc) <= half;
                int is_wing = 0;
                if (in_radial && in_normal) {
                    float fraction = clampf(rc / w->geometry.v[0], 0.0f, 1.0f);
                    float beta_base = fmaxf(fraction * (1.0f - fraction), 0.0f);
                    float local_chord = chord_mean * w->geometry.v[3] * bfx_powf(beta_base, w->geometry.v[2]);
                    float leading = -0.25f * chord_mean;
                    float trailing = leading + local_chord;
                    is_wing = cc >= leading && cc <= trailing;
                }
                mnext[gid] = is_wing ? 1 : 0;
                float u[3];
                cross3(pw->angular_velocity.v, rel, u);
                wall[4 * gid] = u[0] / p->dx;
                wall[4 * gid + 1] = u[1] / p->dx;
                wall[4 * gid + 2] = u[2] / p->dx;
                wall[4 * gid + 3] = is_wing ? -1.0f : 1.0f;
            }
        }
    }
}

/* prescribedWingLinkFraction: BF.metal:1144-1175, with the fluid end placed
 * the way buildPrescribedFlappingWing places it (the solid node's position
 * plus c_q dx, BF.metal:1276-1278). */
float or_wing_link_fraction(const or_params* p, const or_wing* w, const or_wing_prepared* pw, int q, int sx, int sy,
                            int sz) {
    float sw[3], fw[3];
    cell_world(p, sx, sy, sz, sw);
    for (int k = 0; k < 3; ++k) fw[k] = sw[k] + (float)C[q][k] * p->dx;
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 10; ++it) {
        float mid = 0.5f * (lo + hi);
        float smp[3] = {mixf(fw[0], sw[0], mid), mixf(fw[1], sw[1], mid), mixf(fw[2], sw[2], mid)};
        if (or_wing_violation(p, w, pw, smp) > 0.0f) lo = mid;
        else hi = mid;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

/* Link fractions of a list of cut links (fluid cell, direction): the solid
 * source of each is cell - c_q. */
void or_wing_link_fractions(const or_params* p, const or_wing* w, const or_wing_prepared* pw, const uint32_t* cell,
                            const uint8_t* dir, int64_t count, float* out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
        int64_t g = cell[i];
        int x = (int)(g % p->nx), y = (int)((g / p->nx) % p->ny), z = (int)(g / ((int64_t)p->nx * p->ny));
        int q = dir[i];
        out[i] = or_wing_link_fraction(p, w, pw, q, x - C[q][0], y - C[q][1], z - C[q][2]);
    }
}

/* The chord law's power, exposed for the portable-math test. */
float or_powf(float b, float e) { return bfx_powf(b, e); }

/* ------------------------------------------------------------------ */
/* Triangle mesh: closest point BF.metal:1529-1583; raster 1638-1686;  */
/* resolve 1697-1738/1978-2039; links 2044-2076.                        */
/* ------------------------------------------------------------------ */
static void closest_point(const float p[3], const float a[3], const float b[3], const float c[3], float out[3],
                          float bary[3]) {
    float ab[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    float ac[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    float ap[3] = {p[0] - a[0], p[1] - a[1], p[2] - a[2]};
    float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0.0f && d2 <= 0.0f) {
        memcpy(out, a, 12);
        bary[0] = 1; bary[1] = 0; bary[2] = 0;
        return;
    }
    float bp[3] = {p[0] - b[0], p[1] - b[1], p[2] - b[2]};
    float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
        memcpy(out, b, 12);
        bary[0] = 0; bary[1] = 1; bary[2] = 0;
        return;
    }
    float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float v = d1 / (d1 - d3);
        for (int k = 0; k < 3; ++k) out[k] = a[k] + v * ab[k];
        bary[0] = 1.0f - v; bary[1] = v; bary[2] = 0;
        return;
    }
    float cp[3] = {p[0] - c[0], p[1] - c[1], p[2] - c[2]};
    float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0.0f && d5 <= d6) {
        memcpy(out, c, 12);
        bary[0] = 0; bary[1] = 0; bary[2] = 1;
        return;
    }
    float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
        float w = d2 / (d2 - d6);
        for (int k = 0; k < 3; ++k) out[k] = a[k] + w * ac[k];
        bary[0] = 1.0f - w; bary[1] = 0; bary[2] = w;
        return;
    }
    float va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
        float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int k = 0; k < 3; ++k) out[k] = b[k] + w * (c[k] - b[k]);
        bary[0] = 0; bary[1] = 1.0f - w; bary[2] = w;
        return;
    }
    float inv = 1.0f / fmaxf(va + vb + vc, 1.0e-20f);
    float v = vb * inv, w = vc * inv;
    for (int k = 0; k < 3; ++k) out[k] = a[k] + ab[k] * v + ac[k] * w;
    bary[0] = 1.0f - v - w; bary[1] = v; bary[2] = w;
}

/* Keyframe replay (BF.metal:1585-1622; the reference's host picks the
 * interval once): the interval [first, first + 1] holds `time` -- an exact
 * interior keyframe opens the following interval, times past the last
 * keyframe stay on the last interval and times before the first on the first
 * -- the offset is a + (b - a) * blend with the blend clamped to [0, 1], its
 * rate (b - a) / duration; both are rotated into the world and added to the
 * body's rigid motion. */
void or_mesh_prepare_keyframes(const or_prepared* prep, const float* times, uint32_t nframes, const float* points,
                               uint32_t nverts, float time, float v2l, float* pos, float* vel) {
    uint32_t lo = 0, hi = nframes; /* first index with times[j] > time */
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (times[mid] > time) hi = mid;
        else lo = mid + 1;
    }
    uint32_t first = lo == 0 ? 0 : lo - 1;
    if (first > nframes - 2) first = nframes - 2;
    const float duration = times[first + 1] - times[first];
    float blend = (time - times[first]) / duration;
    blend = blend < 0.0f ? 0.0f : (blend > 1.0f ? 1.0f : blend);
    for (uint32_t i = 0; i < nverts; ++i) {
        const float* pa = points + 3 * ((size_t)first * nverts + i);
        const float* pb = pa + 3 * (size_t)nverts;
        float d[3], l[3], dl[3], r[3], rd[3], cr[3], w[3], v[3];
        for (int k = 0; k < 3; ++k) {
            d[k] = pb[k] - pa[k];
            l[k] = pa[k] + d[k] * blend;
            dl[k] = d[k] / duration;
        }
        quat_rotate(prep->orientation.v, l, r);
        quat_rotate(prep->orientation.v, dl, rd);
        for (int k = 0; k < 3; ++k) w[k] = prep->body_position.v[k] + r[k];
        cross3(prep->omega_body_world.v, r, cr);
        for (int k = 0; k < 3; ++k) v[k] = prep->linear_velocity.v[k] + cr[k] + rd[k];
        pos[4 * i] = w[0]; pos[4 * i + 1] = w[1]; pos[4 * i + 2] = w[2]; pos[4 * i + 3] = 0.0f;
        vel[4 * i] = v[0] * v2l; vel[4 * i + 1] = v[1] * v2l; vel[4 * i + 2] = v[2] * v2l; vel[4 * i + 3] = 0.0f;
    }
}

void or_mesh_prepare_articulated(const or_prepared* prep, const float* local, const uint8_t* segment,
                                 uint32_t nverts, float v2l, float* pos, float* vel) {
    for (uint32_t i = 0; i < nverts; ++i) {
        const float* l = local + 3 * i;
        float w[3], v[3];
        if (segment[i] == 0) {
            float r[3];
            quat_rotate(prep->orientation.v, l, r);
            for (int k = 0; k < 3; ++k) w[k] = prep->body_position.v[k] + r[k];
            float rb[3] = {r[0], r[1], r[2]}, cr[3];
            cross3(prep->omega_body_world.v, rb, cr);
            for (int k = 0; k < 3; ++k) v[k] = prep->linear_velocity.v[k] + cr[k];
        } else {
            const or_f4* fr = segment[i] == 1 ? &prep->left_root : &prep->right_root;
            for (int k = 0; k < 3; ++k) w[k] = fr[0].v[k] + fr[1].v[k] * l[0] + fr[2].v[k] * l[1] + fr[3].v[k] * l[2];
            float rb[3] = {w[0] - prep->body_position.v[0], w[1] - prep->body_position.v[1], w[2] - prep->body_position.v[2]};
            float cr[3], cw[3];
            cross3(prep->omega_body_world.v, rb, cr);
            float rr[3] = {w[0] - fr[0].v[0], w[1] - fr[0].v[1], w[2] - fr[0].v[2]};
            cross3(fr[4].v, rr, cw);
            for (int k = 0; k < 3; ++k) v[k] = prep->linear_velocity.v[k] + cr[k] + cw[k];
        }
        pos[4 * i] = w[0]; pos[4 * i + 1] = w[1]; pos[4 * i + 2] = w[2]; pos[4 * i + 3] = 0.0f;
        vel[4 * i] = v[0] * v2l; vel[4 * i + 1] = v[1] * v2l; vel[4 * i + 2] = v[2] * v2l; vel[4 * i + 3] = 0.0f;
    }
}

void or_prepare_segments(const or_bird* bird, const or_prepared* prep, const or_joint* joints, int njoints,
                         float time, or_segment* out) {
    float af = 2.0f * 3.14159265358979323846f * bird->wing_kinematics0.v[0];
    float phase = af * time;
    for (int side = 0; side < 2 && njoints > 0; ++side) {
        const or_f4* fr = side == 0 ? &prep->left_root : &prep->right_root;
        float sgn = side == 0 ? 1.0f : -1.0f;
        float po[3], pc[3], ps[3], pn[3], pw[3], pu[3] = {0.0f, 0.0f, 0.0f};
        for (int k = 0; k < 3; ++k) {
            po[k] = fr[0].v[k];
            pc[k] = fr[1].v[k];
            ps[k] = fr[2].v[k];
            pn[k] = fr[3].v[k];
            pw[k] = fr[4].v[k];
        }
        for (int j = 0; j < njoints; ++j) {
            const or_joint* jt = &joints[j];
            float o[3], ax[3], cc[3], cs[3], cn[3], om[3], d[3], cr[3], uu[3];
            /* the right frame's normal is the mirror of the left's negated: negate
             * the axis's normal component there (with the angle) to keep the mirror */
            float a2 = sgn * jt->axis[2];
            for (int k = 0; k < 3; ++k) {
                o[k] = po[k] + pc[k] * jt->origin[0] + ps[k] * jt->origin[1] + pn[k] * jt->origin[2];
                ax[k] = pc[k] * jt->axis[0] + ps[k] * jt->axis[1] + pn[k] * a2;
            }
            float ang = sgn * (jt->bias + jt->amplitude * bfx_sinf(phase + jt->phase));
            float rate = sgn * (af * jt->amplitude * bfx_cosf(phase + jt->phase));
            rotate_axis(pc, ax, ang, cc);
            rotate_axis(ps, ax, ang, cs);
            rotate_axis(pn, ax, ang, cn);
            for (int k = 0; k < 3; ++k) {
                om[k] = pw[k] + ax[k] * rate;
                d[k] = o[k] - po[k];
            }
            cross3(pw, d, cr);
            for (int k = 0; k < 3; ++k) uu[k] = pu[k] + cr[k];
            or_segment* f = &out[2 * j + side];
            for (int k = 0; k < 3; ++k) {
                f->origin[k] = o[k];
                f->chord[k] = cc[k];
                f->span[k] = cs[k];
                f->normal[k] = cn[k];
                f->omega[k] = om[k];
                f->uvel[k] = uu[k];
            }
            f->origin[3] = f->chord[3] = f->span[3] = f->normal[3] = f->omega[3] = f->uvel[3] = 0.0f;
            memcpy(po, o, sizeof(o));
            memcpy(pc, cc, sizeof(cc));
            memcpy(ps, cs, sizeof(cs));
            memcpy(pn, cn, sizeof(cn));
            memcpy(pw, om, sizeof(om));
            memcpy(pu, uu, sizeof(uu));
        }
    }
}

void or_mesh_prepare_segments(const or_prepared* prep, const or_segment* segs, const float* local,
                              const uint8_t* segment, uint32_t nverts, float v2l, float* pos, float* vel) {
    or_mesh_prepare_articulated(prep, local, segment, nverts, v2l, pos, vel);
    for (uint32_t i = 0; i < nverts; ++i) {
        if (segment[i] < 3) continue;
        const or_segment* f = &segs[segment[i] - 3];
        const float* l = local + 3 * i;
        float w[3], rb[3], rr[3], cr[3], cw[3];
        for (int k = 0; k < 3; ++k) w[k] = f->origin[k] + f->chord[k] * l[0] + f->span[k] * l[1] + f->normal[k] * l[2];
        for (int k = 0; k < 3; ++k) {
            rb[k] = w[k] - prep->body_position.v[k];
            rr[k] = w[k] - f->origin[k];
        }
        cross3(prep->omega_body_world.v, rb, cr);
        cross3(f->omega, rr, cw);
        for (int k = 0; k < 3; ++k) {
            pos[4 * i + k] = w[k];
            vel[4 * i + k] = (prep->linear_velocity.v[k] + cr[k] + cw[k] + f->uvel[k]) * v2l;
        }
        pos[4 * i + 3] = 0.0f;
        vel[4 * i + 3] = 0.0f;
    }
}

static void tri_vertices(const float* pos, const uint32_t* tris, uint32_t t, float a[3], float b[3], float c[3]) {
    uint32_t ia = tris[3 * t], ib = tris[3 * t + 1], ic = tris[3 * t + 2];
    memcpy(a, pos + 4 * ia, 12);
    memcpy(b, pos + 4 * ib, 12);
    memcpy(c, pos + 4 * ic, 12);
}

/* 64-bit key = quantized distance (1/65536 cell, 32 bits) << 32 | triangle id;
 * the reference packs 20 + 12 bits and caps the mesh at 4,096 triangles. */
void or_mesh_rasterize(const or_params* p, const float* pos, const uint32_t* tris, uint32_t ntris,
                       float half_thickness, uint64_t* keys) {
    float cs = p->dx;
    for (uint32_t t = 0; t < ntris; ++t) {
        float a[3], b[3], c[3];
        tri_vertices(pos, tris, t, a, b, c);
        float guard = half_thickness + 2.0f * cs;
        int lo[3], hi[3];
        int dims[3] = {p->nx, p->ny, p->nz};
        for (int k = 0; k < 3; ++k) {
            float mn = fminf(a[k], fminf(b[k], c[k])) - guard;
            float mx = fmaxf(a[k], fmaxf(b[k], c[k])) + guard;
            lo[k] = (int)floorf((mn - p->origin[k]) / cs - 0.5f);
            hi[k] = (int)ceilf((mx - p->origin[k]) / cs - 0.5f);
            lo[k] = lo[k] < 0 ? 0 : (lo[k] > dims[k] - 1 ? dims[k] - 1 : lo[k]);
            hi[k] = hi[k] < 0 ? 0 : (hi[k] > dims[k] - 1 ? dims[k] - 1 : hi[k]);
        }
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int x = lo[0]; x <= hi[0]; ++x) {
                    float w[3], cp[3], bary[3];
                    cell_world(p, x, y, z, w);
                    closest_point(w, a, b, c, cp, bary);
                    float d[3] = {w[0] - cp[0], w[1] - cp[1], w[2] - cp[2]};
                    float dc = lengthf(d) / cs;
                    float bin = roundf(dc * 65536.0f);
                    uint64_t ub = bin >= 4294967295.0f ? 0xFFFFFFFFull : (uint64_t)bin;
                    uint64_t key = (ub << 32) | (uint64_t)t;
                    int64_t gid = flat(p, x, y, z);
                    if (key < keys[gid]) keys[gid] = key;
                }
    }
}

void or_mesh_resolve(const or_params* p, const float* pos, const float* vel, const uint32_t* tris,
                     const uint8_t* tri_part, uint32_t ntris, float half_thickness, const uint64_t* keys,
                     uint8_t* mask, float* wall) {
    int64_t n = ncells(p);
#pragma omp parallel for schedule(static)
    for (int64_t gid = 0; gid < n; ++gid) {
        uint64_t key = keys[gid];
        if (key == UINT64_MAX) continue;
        uint32_t t = (uint32_t)(key & 0xFFFFFFFFu);
        if (t >= ntris) continue;
        int64_t xy = (int64_t)p->nx * p->ny;
        int z = (int)(gid / xy);
        int64_t rem = gid - (int64_t)z * xy;
        int y = (int)(rem / p->nx);
        int x = (int)(rem - (int64_t)y * p->nx);
        float w[3], a[3], b[3], c[3], cp[3], bary[3];
        cell_world(p, x, y, z, w);
        tri_vertices(pos, tris, t, a, b, c);
        closest_point(w, a, b, c, cp, bary);
        uint32_t ia = tris[3 * t], ib = tris[3 * t + 1], ic = tris[3 * t + 2];
        float v[3];
        for (int k = 0; k < 3; ++k) v[k] = bary[0] * vel[4 * ia + k] + bary[1] * vel[4 * ib + k] + bary[2] * vel[4 * ic + k];
        float d[3] = {w[0] - cp[0], w[1] - cp[1], w[2] - cp[2]};
        float sd = lengthf(d) - half_thickness;
        int solid = sd <= 0.0f;
        mask[gid] = solid ? tri_part[t] : 0;
        wall[4 * gid] = v[0];
        wall[4 * gid + 1] = v[1];
        wall[4 * gid + 2] = v[2];
        wall[4 * gid + 3] = sd / p->dx;
    }
}

static float tri_distance(const float* pos, const uint32_t* tris, uint32_t t, const float w[3]) {
    float a[3], b[3], c[3], cp[3], bary[3];
    tri_vertices(pos, tris, t, a, b, c);
    closest_point(w, a, b, c, cp, bary);
    float d[3] = {w[0] - cp[0], w[1] - cp[1], w[2] - cp[2]};
    return lengthf(d);
}

/* Exact wall position along the link: root of min(d_A, d_B) - h, where A and B
 * are the winning triangles of the fluid and solid cells, bracketed by an
 * 8-way scan from the fluid end and refined by 24 bisections (the procedure
 * of Scripts/audit-dove-moving-wall-link-ray-root.py:161-197, restricted to
 * the two candidate triangles). q is measured from the fluid node. */
float or_mesh_ray_root(const or_params* p, const float* pos, const uint32_t* tris, uint32_t ntris,
                       float half_thickness, const uint64_t* keys, int fx, int fy, int fz, int sx, int sy, int sz) {
    float fw[3], sw[3];
    cell_world(p, fx, fy, fz, fw);
    cell_world(p, sx, sy, sz, sw);
    uint64_t kf = keys[flat(p, fx, fy, fz)], ks = keys[flat(p, sx, sy, sz)];
    uint32_t ta = (uint32_t)(ks & 0xFFFFFFFFu);
    uint32_t tb = kf == UINT64_MAX ? ta : (uint32_t)(kf & 0xFFFFFFFFu);
    if (ta >= ntris) return 0.5f;
    if (tb >= ntris) tb = ta;
    float lo = 0.0f, hi = 1.0f;
    int found = 0;
    for (int i = 1; i <= 8; ++i) {
        float t = (float)i * 0.125f;
        float s[3] = {mixf(fw[0], sw[0], t), mixf(fw[1], sw[1], t), mixf(fw[2], sw[2], t)};
        float g = fminf(tri_distance(pos, tris, ta, s), tri_distance(pos, tris, tb, s)) - half_thickness;
        if (g <= 0.0f) {
            hi = t;
            found = 1;
            break;
        }
        lo = t;
    }
    if (!found) return 1.0f;
    for (int it = 0; it < 24; ++it) {
        float mid = 0.5f * (lo + hi);
        float s[3] = {mixf(fw[0], sw[0], mid), mixf(fw[1], sw[1], mid), mixf(fw[2], sw[2], mid)};
        float g = fminf(tri_distance(pos, tris, ta, s), tri_distance(pos, tris, tb, s)) - half_thickness;
        if (g <= 0.0f) hi = mid;
        else lo = mid;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

int64_t or_write_links(const or_params* p, int kind, const or_bird* bird, const or_prepared* prep,
                       const float* mesh_pos, const uint32_t* tris, uint32_t ntris, float half_thickness,
                       const uint64_t* keys, float* pops, const uint8_t* mprev, const uint8_t* mcur,
                       const float* wall, float* covered) {
    int64_t n = ncells(p);
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
    for (int z = 0; z < p->nz; ++z) {
        for (int y = 0; y < p->ny; ++y) {
            for (int x = 0; x < p->nx; ++x) {
                int64_t s = flat(p, x, y, z);
                if (mcur[s] == 0) continue;
                if (p->has_prev_geom && mprev[s] == 0 && covered) {
                    /* preserve the just-covered fluid state before the slots are reused */
                    float pd = 0.0f, pm[3] = {0, 0, 0};
                    for (int q = 0; q < 19; ++q) {
                        float prev = pops[q * n + s];
                        pd += prev;
                        pm[0] += prev * (float)C[q][0];
                        pm[1] += prev * (float)C[q][1];
                        pm[2] += prev * (float)C[q][2];
                    }
                    covered[4 * s] = pm[0];
                    covered[4 * s + 1] = pm[1];
                    covered[4 * s + 2] = pm[2];
                    covered[4 * s + 3] = pd;
                }
                for (int q = 1; q < 19; ++q) {
                    int bx = x + C[q][0], by = y + C[q][1], bz = z + C[q][2];
                    if (!inside3(p, bx, by, bz)) continue;
                    int64_t nb = flat(p, bx, by, bz);
                    if (mcur[nb] != 0) continue;
                    float qf;
                    if (kind == 0) {
                        qf = or_ellipsoid_link_fraction(p, bird, prep, bx, by, bz, x, y, z);
                    } else if (kind == 1) {
                        float sd = fminf(wall[4 * s + 3], 0.0f);
                        float fd = fmaxf(wall[4 * nb + 3], 0.0f);
                        qf = clampf(fd / fmaxf(fd - sd, 1.0e-6f), 1.0e-4f, 1.0f);
                    } else if (kind == 2) {
                        qf = or_mesh_ray_root(p, mesh_pos, tris, ntris, half_thickness, keys, bx, by, bz, x, y, z);
                    } else {
                        qf = or_wing_link_fraction(p, (const or_wing*)(const void*)bird,
                                                   (const or_wing_prepared*)(const void*)prep, q, x, y, z);
                    }
                    pops[q * n + s] = qf;
                    total++;
                }
            }
        }
    }
    return total;
}

int64_t or_enumerate_links(const or_params* p, const uint8_t* mprev, const uint8_t* mcur, uint32_t* cell,
                           uint8_t* dir, int64_t capacity) {
    int64_t count = 0;
    const int per[3] = {axis_periodic(p, 0), axis_periodic(p, 1), axis_periodic(p, 2)};
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                int64_t g = flat(p, x, y, z);
                if (mcur[g] != 0 || mprev[g] != 0) continue;
                for (int q = 1; q < 19; ++q) {
                    int sx = x - C[q][0], sy = y - C[q][1], sz = z - C[q][2];
                    if (!inside3(p, sx, sy, sz)) {
                        if (per[0]) sx = sx < 0 ? p->nx - 1 : (sx >= p->nx ? 0 : sx);
                        if (per[1]) sy = sy < 0 ? p->ny - 1 : (sy >= p->ny ? 0 : sy);
                        if (per[2]) sz = sz < 0 ? p->nz - 1 : (sz >= p->nz ? 0 : sz);
                        if (!inside3(p, sx, sy, sz)) continue;
                    }
                    if (mcur[flat(p, sx, sy, sz)] == 0) continue;
                    if (cell && count < capacity) {
                        cell[count] = (uint32_t)g;
                        dir[count] = (uint8_t)q;
                    }
                    count++;
                }
            }
    return count;
}

/* ------------------------------------------------------------------ */
/* Rigid body: integrateBirdBody BF.metal:6574-6627 (FP32 and the FP64  */
/* form used on the GPU); RigidBodyIntegrator RigidBody.swift:88-126.   */
/* ------------------------------------------------------------------ */
void or_integrate_body_f32(or_body_f32* body, const or_bird* bird, const float force[3], const float torque[3],
                           const float gravity[3], float dt_total, int substeps) {
    int n = substeps < 1 ? 1 : substeps;
    float dt = dt_total / (float)n;
    float mass = bird->body_radii_mass.v[3];
    const float* inertia = bird->inertia.v;
    float v[3], x[3], o[4], w[3];
    memcpy(v, body->velocity, 12);
    memcpy(x, body->position, 12);
    quat_normalize(body->orientation, o);
    memcpy(w, body->omega_body, 12);
    for (int s = 0; s < n; ++s) {
        for (int k = 0; k < 3; ++k) v[k] += (force[k] / mass + gravity[k]) * dt;
        for (int k = 0; k < 3; ++k) x[k] += v[k] * dt;
        float tb[3];
        quat_unrotate(o, torque, tb);
        float am[3] = {inertia[0] * w[0], inertia[1] * w[1], inertia[2] * w[2]};
        float g[3];
        cross3(w, am, g);
        float aa[3] = {(tb[0] - g[0]) / inertia[0], (tb[1] - g[1]) / inertia[1], (tb[2] - g[2]) / inertia[2]};
        for (int k = 0; k < 3; ++k) w[k] += aa[k] * dt;
        /* quaternionMultiply(orientation, (omega, 0)) */
        float d[4], cr[3];
        cross3(o, w, cr);
        for (int k = 0; k < 3; ++k) d[k] = o[3] * w[k] + 0.0f * o[k] + cr[k];
        d[3] = o[3] * 0.0f - dot3(o, w);
        float nq[4];
        for (int k = 0; k < 4; ++k) nq[k] = o[k] + 0.5f * dt * d[k];
        quat_normalize(nq, o);
    }
    memcpy(body->position, x, 12);
    memcpy(body->velocity, v, 12);
    memcpy(body->orientation, o, 16);
    memcpy(body->omega_body, w, 12);
}

static void cross3d(const double a[3], const double b[3], double r[3]) {
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static void quat_normalize_d(const double q[4], double r[4]) {
    double n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (n2 > 1.0e-40) {
        double n = sqrt(n2);
        for (int k = 0; k < 4; ++k) r[k] = q[k] / n;
    } else {
        r[0] = r[1] = r[2] = 0.0;
        r[3] = 1.0;
    }
}
static void quat_rotate_d(const double q[4], const double v[3], double r[3]) {
    double t[3], c2[3];
    cross3d(q, v, t);
    t[0] *= 2.0;
    t[1] *= 2.0;
    t[2] *= 2.0;
    cross3d(q, t, c2);
    for (int k = 0; k < 3; ++k) r[k] = v[k] + q[3] * t[k] + c2[k];
}

void or_integrate_body_f64(or_body_f64* body, const or_bird* bird, const double force[3], const double torque[3],
                           const double gravity[3], double dt_total, int substeps) {
    int n = substeps < 1 ? 1 : substeps;
    double dt = dt_total / (double)n;
    double mass = (double)bird->body_radii_mass.v[3];
    double inertia[3] = {(double)bird->inertia.v[0], (double)bird->inertia.v[1], (double)bird->inertia.v[2]};
    double v[3], x[3], o[4], w[3];
    memcpy(v, body->velocity, 24);
    memcpy(x, body->position, 24);
    quat_normalize_d(body->orientation, o);
    memcpy(w, body->omega_body, 24);
    for (int s = 0; s < n; ++s) {
        for (int k = 0; k < 3; ++k) v[k] += (force[k] / mass + gravity[k]) * dt;
        for (int k = 0; k < 3; ++k) x[k] += v[k] * dt;
        double conj[4] = {-o[0], -o[1], -o[2], o[3]}, tb[3];
        quat_rotate_d(conj, torque, tb);
        double am[3] = {inertia[0] * w[0], inertia[1] * w[1], inertia[2] * w[2]};
        double g[3];
        cross3d(w, am, g);
        for (int k = 0; k < 3; ++k) w[k] += ((tb[k] - g[k]) / inertia[k]) * dt;
        double d[4], cr[3];
        cross3d(o, w, cr);
        for (int k = 0; k < 3; ++k) d[k] = o[3] * w[k] + cr[k];
        d[3] = -(o[0] * w[0] + o[1] * w[1] + o[2] * w[2]);
        double nq[4];
        for (int k = 0; k < 4; ++k) nq[k] = o[k] + 0.5 * dt * d[k];
        quat_normalize_d(nq, o);
    }
    memcpy(body->position, x, 24);
    memcpy(body->velocity, v, 24);
    memcpy(body->orientation, o, 32);
    memcpy(body->omega_body, w, 24);
}

/* RigidBodyIntegrator.integrate (RigidBody.swift:88-126), FP32, with the
 * Swift Quaternion semantics (normalized by division, VectorMath.swift). */
void or_rigid_body_swift_f32(or_body_f32* body, float mass, const float inertia[3], const float force[3],
                             const float torque[3], const float gravity[3], float dt, int substeps) {
    float st = dt / (float)substeps;
    for (int s = 0; s < substeps; ++s) {
        float acc[3] = {force[0] / mass + gravity[0], force[1] / mass + gravity[1], force[2] / mass + gravity[2]};
        for (int k = 0; k < 3; ++k) body->velocity[k] += acc[k] * st;
        for (int k = 0; k < 3; ++k) body->position[k] += body->velocity[k] * st;
        float q[4];
        float mag = sqrtf(body->orientation[0] * body->orientation[0] + body->orientation[1] * body->orientation[1] +
                          body->orientation[2] * body->orientation[2] + body->orientation[3] * body->orientation[3]);
        if (mag > 1e-12f) {
            for (int k = 0; k < 4; ++k) q[k] = body->orientation[k] / mag;
        } else {
            q[0] = q[1] = q[2] = 0.0f;
            q[3] = 1.0f;
        }
        float tb[3];
        quat_unrotate(q, torque, tb);
        float* om = body->omega_body;
        float am[3] = {inertia[0] * om[0], inertia[1] * om[1], inertia[2] * om[2]};
        float gy[3];
        cross3(om, am, gy);
        float on[3];
        for (int k = 0; k < 3; ++k) on[k] = om[k] + ((tb[k] - gy[k]) / inertia[k]) * st;
        float d[4], cr[3];
        cross3(q, on, cr);
        for (int k = 0; k < 3; ++k) d[k] = q[3] * on[k] + 0.0f * q[k] + cr[k];
        d[3] = q[3] * 0.0f - dot3(q, on);
        float nq[4];
        for (int k = 0; k < 3; ++k) nq[k] = q[k] + d[k] * (0.5f * st);
        nq[3] = q[3] + d[3] * (0.5f * st);
        float m2 = sqrtf(nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3]);
        if (m2 > 1e-12f) {
            for (int k = 0; k < 4; ++k) body->orientation[k] = nq[k] / m2;
        } else {
            body->orientation[0] = body->orientation[1] = body->orientation[2] = 0.0f;
            body->orientation[3] = 1.0f;
        }
        memcpy(om, on, 12);
    }
}

/* prescribedWingMomentum + updateWingInertialReaction: BF.metal:6461-6572 */
static void wing_momentum(const float root[3], const float chord[3], const float span[3], const float normal[3],
                          const float rel[3], const float mc[4], const float inertia[3], const float body_pos[3],
                          float lin[3], float ang[3]) {
    float co[3];
    for (int k = 0; k < 3; ++k) co[k] = chord[k] * mc[1] + span[k] * mc[2] + normal[k] * mc[3];
    float cv[3];
    cross3(rel, co, cv);
    for (int k = 0; k < 3; ++k) lin[k] = mc[0] * cv[k];
    float a = inertia[0] * dot3(rel, chord), b = inertia[1] * dot3(rel, span), c = inertia[2] * dot3(rel, normal);
    float spin[3];
    for (int k = 0; k < 3; ++k) spin[k] = chord[k] * a + span[k] * b + normal[k] * c;
    float arm[3] = {root[0] + co[0] - body_pos[0], root[1] + co[1] - body_pos[1], root[2] + co[2] - body_pos[2]};
    float cr[3];
    cross3(arm, lin, cr);
    for (int k = 0; k < 3; ++k) ang[k] = cr[k] + spin[k];
}

void or_wing_reaction(const or_prepared* prep, const or_bird* bird, float dt, int initialize_only, float* previous,
                      float* reaction) {
    if (bird->left_wing_inertia.v[3] < 0.5f || bird->right_wing_inertia.v[3] < 0.5f) {
        memset(previous, 0, 16 * sizeof(float));
        memset(reaction, 0, 16 * sizeof(float));
        return;
    }
    float ll[3], la[3], rl[3], ra[3];
    wing_momentum(prep->left_root.v, prep->left_chord.v, prep->left_span.v, prep->left_normal.v,
                  prep->left_angular_velocity.v, bird->left_wing_mass_com.v, bird->left_wing_inertia.v,
                  prep->body_position.v, ll, la);
    wing_momentum(prep->right_root.v, prep->right_chord.v, prep->right_span.v, prep->right_normal.v,
                  prep->right_angular_velocity.v, bird->right_wing_mass_com.v, bird->right_wing_inertia.v,
                  prep->body_position.v, rl, ra);
    float inv = 1.0f / dt;
    if (initialize_only) {
        memset(reaction, 0, 16 * sizeof(float));
    } else {
        const float* cur[4] = {ll, la, rl, ra};
        for (int j = 0; j < 4; ++j) {
            for (int k = 0; k < 3; ++k) reaction[4 * j + k] = -(cur[j][k] - previous[4 * j + k]) * inv;
            reaction[4 * j + 3] = 0.0f;
        }
    }
    const float* cur[4] = {ll, la, rl, ra};
    for (int j = 0; j < 4; ++j) {
        for (int k = 0; k < 3; ++k) previous[4 * j + k] = cur[j][k];
        previous[4 * j + 3] = 0.0f;
    }
}

/* monitorBirdRuntimeSafety: BF.metal:6629-6707 */
void or_safety(const or_body_f32* body, const or_bird* bird, const or_params* p, uint32_t step_lo, uint32_t step_hi,
               float* metrics, uint32_t* event) {
    float o[4];
    quat_normalize(body->orientation, o);
    const float* le = bird->safety_geometry.v;
    float ex[3] = {le[0], 0, 0}, ey[3] = {0, le[1], 0}, ez[3] = {0, 0, le[2]};
    float a[3], b[3], c[3];
    quat_rotate(o, ex, a);
    quat_rotate(o, ey, b);
    quat_rotate(o, ez, c);
    float we[3];
    for (int k = 0; k < 3; ++k) we[k] = fabsf(a[k]) + fabsf(b[k]) + fabsf(c[k]);
    float dx = p->dx;
    float margin = (p->sponge_width + 3.0f) * dx;
    int dims[3] = {p->nx, p->ny, p->nz};
    float clearance = INFINITY;
    for (int k = 0; k < 3; ++k) {
        float mn = p->origin[k] + margin;
        float mx = p->origin[k] + (float)dims[k] * dx - margin;
        float lc = body->position[k] - we[k] - mn;
        float uc = mx - body->position[k] - we[k];
        clearance = fminf(clearance, fminf(lc, uc));
    }
    float v2l = p->v2l;
    float ffp[3] = {p->far[0] / v2l, p->far[1] / v2l, p->far[2] / v2l};
    float rv[3] = {body->velocity[0] - ffp[0], body->velocity[1] - ffp[1], body->velocity[2] - ffp[2]};
    float rel = lengthf(rv);
    float rot = lengthf(body->omega_body) * bird->safety_geometry.v[3];
    float surface = rel + rot + bird->safety_limits.v[0];
    float mach = surface * v2l / sqrtf(CS2);
    int finite = isfinite(mach) && isfinite(clearance);
    for (int k = 0; k < 3; ++k)
        finite = finite && isfinite(body->position[k]) && isfinite(body->velocity[k]) && isfinite(body->omega_body[k]);
    for (int k = 0; k < 4; ++k) finite = finite && isfinite(body->orientation[k]);
    if (isfinite(mach)) metrics[0] = fmaxf(metrics[0], mach);
    if (isfinite(clearance)) metrics[1] = fminf(metrics[1], clearance);
    uint32_t flags = 0;
    if (!finite) flags |= 4u;
    if (isfinite(mach) && mach > bird->safety_limits.v[1]) flags |= 1u;
    if (isfinite(clearance) && clearance < 0.0f) flags |= 2u;
    if (flags != 0 && event[2] == 0) {
        event[0] = step_lo;
        event[1] = step_hi;
        event[2] = flags;
        event[3] = 0;
        metrics[2] = mach;
        metrics[3] = clearance;
    }
}

/* InterpolatedBounceBackReference.linkFraction / population /
 * conservativeUncoveredBodyImpulse (InterpolatedBounceBackReference.swift:12-61). */
double or_link_fraction(double fluid_implicit, double solid_implicit) {
    double q = fluid_implicit / (fluid_implicit - solid_implicit);
    q = q < 1.0e-4 ? 1.0e-4 : q;
    return q > 1.0 ? 1.0 : q;
}

double or_interpolated_population(double q, double reflected, double farther_outgoing, double previous_incoming,
                                  double moving_wall_correction) {
    if (q <= 0.5) return 2.0 * q * reflected + (1.0 - 2.0 * q) * farther_outgoing + moving_wall_correction;
    return (reflected + moving_wall_correction) / (2.0 * q) + (2.0 * q - 1.0) * previous_incoming / (2.0 * q);
}

void or_uncovered_impulse(const double refill_momentum[3], const double* directions, const double* old_outgoing,
                          const double* suppressed_incoming, int count, double out[3]) {
    for (int k = 0; k < 3; ++k) out[k] = -refill_momentum[k];
    for (int i = 0; i < count; ++i) {
        double s = old_outgoing[i] + suppressed_incoming[i];
        for (int k = 0; k < 3; ++k) out[k] = out[k] - s * directions[3 * i + k];
    }
}
