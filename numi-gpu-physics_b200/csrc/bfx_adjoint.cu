// Discrete adjoint of the moving-boundary D3Q19 step: the gradient of a
// time-averaged load objective (force component, aerodynamic power) with
// respect to the four prescribed wing-kinematic parameters
//   theta = (stroke amplitude, pitch amplitude, pitch phase, deviation amplitude).
//
// Scope: TRT collision, FP32 or FP64 populations, triangle-mesh geometry moved
// by the prescribed wing frames (no free flight), far-field / velocity /
// periodic faces, momentum-exchange estimator 6.  The reference has no adjoint;
// the forward step it differentiates is the one bfx_fluid.cu and
// bfx_geometry.cu restate from stepFluidTRT (BirdFlow.metal:2507-3236).
//
// Each reverse step undoes one forward step in the reverse kernel order:
//   k_adj_rare      solid / newly uncovered cells of the box: their values are
//                   wall equilibria, so their adjoint feeds dJ/dtheta through the
//                   wall velocity; their slots get zero.
//   k_adj_bulk      every fluid cell: transposed TRT Jacobian at the taped
//                   pre-collision velocity, sponge factor, reverse streaming
//                   (the adjoint is written into the slots the forward pulled
//                   from: the AA layout makes this an in-place permutation).
//   k_adj_links1/2  bounce-back links: the adjoint of the reconstructed value
//                   flows to the reflected / interpolation populations, to q
//                   and to the wall velocity; the load objective enters here.
//   k_adj_halo      halo values: periodic images receive their adjoint, face
//                   constants drop it.
//   k_adj_topology  cover / uncover momentum impulses of the load.
//   k_adj_reduce    fixed-order FP64 sum of the block partials of dJ/dtheta.
// Topology (which cells are solid, which links exist, which bounce-back case
// applies) is held fixed inside a step: the objective is piecewise smooth in
// theta and the adjoint is the derivative of the smooth piece.
//
// The geometry tangents (dq/dtheta, du_wall/dtheta) are forward-mode duals of
// the same float computations the forward step performs: wing frames
// (k_prepare), vertex placement (k_mesh_prepare), the triangle closest point
// (k_mesh_resolve) and the link fraction (linear rule, or the implicit-function
// derivative of the ray root).
#include <algorithm>

#include "bfx_bulk.cuh"
#include "bfx_geom_common.cuh"

namespace bfx {
namespace {

constexpr int NP = kKinematicParams;

// ---------------------------------------------------------------------------
// Forward-mode duals over the kinematic parameters.  The value part repeats
// the forward step's float operations in the same order, so branch decisions
// (closest-point region, clamps) follow the forward step.
// ---------------------------------------------------------------------------
struct Du {
    float v;
    float d[NP];
};
__device__ __forceinline__ Du dc(float v) {
    Du r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = 0.0f;
    return r;
}
__device__ __forceinline__ Du operator+(const Du& a, const Du& b) {
    Du r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
__device__ __forceinline__ Du operator-(const Du& a, const Du& b) {
    Du r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
__device__ __forceinline__ Du operator*(const Du& a, const Du& b) {
    Du r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
__device__ __forceinline__ Du operator*(const Du& a, float b) {
    Du r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = a.d[k] * b;
    return r;
}
__device__ __forceinline__ Du operator*(float a, const Du& b) {
    Du r;
    r.v = a * b.v;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = a * b.d[k];
    return r;
}
__device__ __forceinline__ Du operator/(const Du& a, const Du& b) {
    Du r;
    r.v = a.v / b.v;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
    return r;
}
__device__ __forceinline__ Du dsqrt(const Du& a) {
    Du r;
    r.v = sqrtf(a.v);
    const float s = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = a.d[k] * s;
    return r;
}
__device__ __forceinline__ Du dsin(const Du& a) {
    Du r;
    r.v = bfx_sinf(a.v);
    const float c = bfx_cosf(a.v);
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = c * a.d[k];
    return r;
}
__device__ __forceinline__ Du dcos(const Du& a) {
    Du r;
    r.v = bfx_cosf(a.v);
    const float s = bfx_sinf(a.v);
#pragma unroll
    for (int k = 0; k < NP; ++k) r.d[k] = -s * a.d[k];
    return r;
}

struct DV {
    Du x, y, z;
};
__device__ __forceinline__ DV dv(V3 a) { return DV{dc(a.x), dc(a.y), dc(a.z)}; }
__device__ __forceinline__ DV operator-(const DV& a, const DV& b) { return DV{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Du ddot(const DV& a, const DV& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ DV dcross(const DV& a, const DV& b) {
    return DV{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ DV dcross(V3 a, const DV& b) {
    return DV{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// rotateAroundAxis (BF.metal:466-473) on duals
__device__ DV drotate(const DV& v, const DV& axis, const Du& angle) {
    const Du s = dsin(angle), c = dcos(angle);
    const DV cr = dcross(axis, v);
    const Du d = ddot(axis, v);
    const Du omc = dc(1.0f) - c;
    return DV{v.x * c + cr.x * s + axis.x * d * omc, v.y * c + cr.y * s + axis.y * d * omc,
              v.z * c + cr.z * s + axis.z * d * omc};
}
__device__ DV dnormalize(const DV& v) {
    const Du l = dsqrt(ddot(v, v));
    return DV{v.x / l, v.y / l, v.z / l};
}

// ---------------------------------------------------------------------------
// Wing-frame tangent: k_prepare's kinematics and makeWingFrame on duals.
// ---------------------------------------------------------------------------
__global__ void k_frame_tangent(const bfx_bird* birdp, const DeviceState* st, float dt, int init, FrameTangent* out) {
    const bfx_bird& bird = *birdp;
    const uint64_t absolute = init ? 0 : st->step + 1;
    const float time = (float)((double)absolute * (double)dt);
    const V3 pos = v3((float)st->body[0], (float)st->body[1], (float)st->body[2]);
    const float4 orient = make_float4((float)st->body[3], (float)st->body[4], (float)st->body[5], (float)st->body[6]);
    const float af = 2.0f * 3.14159265358979323846f * bird.wing_kinematics0.v[0];
    const float phase = af * time;
    Du th[NP];
    const float tv[NP] = {bird.wing_kinematics0.v[1], bird.wing_kinematics1.v[0], bird.wing_kinematics1.v[1],
                          bird.wing_kinematics1.v[2]};
    for (int k = 0; k < NP; ++k) {
        th[k] = dc(tv[k]);
        th[k].d[k] = 1.0f;
    }
    const Du stroke = dc(bird.wing_kinematics0.v[2]) + th[0] * bfx_sinf(phase);
    const Du stroke_rate = (af * th[0]) * bfx_cosf(phase);
    const Du pitch_arg = dc(phase) + th[2];
    const Du pitch = dc(bird.wing_kinematics0.v[3]) + th[1] * dsin(pitch_arg);
    const Du pitch_rate = (af * th[1]) * dcos(pitch_arg);
    const Du deviation = th[3] * bfx_sinf(2.0f * phase);
    const Du deviation_rate = ((2.0f * af) * th[3]) * bfx_cosf(2.0f * phase);
    const float4 o = qnormalize(orient);
    const V3 bx = qrotate(o, v3(1, 0, 0)), by = qrotate(o, v3(0, 1, 0)), bz = qrotate(o, v3(0, 0, 1));
    (void)pos;
    for (int sidx = 0; sidx < 2; ++sidx) {
        const float side = sidx == 0 ? 1.0f : -1.0f;
        const Du signed_stroke = side * stroke;
        const DV span_after = drotate(dv(v3(side * by.x, side * by.y, side * by.z)), dv(bx), signed_stroke);
        const DV normal_after = drotate(dv(v3(side * bz.x, side * bz.y, side * bz.z)), dv(bx), signed_stroke);
        const DV span = drotate(span_after, normal_after, deviation);
        const DV chord_before = drotate(dv(bx), normal_after, deviation);
        const Du signed_pitch = side * pitch;
        const DV chord = drotate(chord_before, span, signed_pitch);
        const DV normal = drotate(normal_after, span, signed_pitch);
        const DV cn = dnormalize(chord), sn = dnormalize(span), nn = dnormalize(normal);
        const Du sr = side * stroke_rate, pr = side * pitch_rate;
        const DV rel = DV{bx.x * sr + normal_after.x * deviation_rate + sn.x * pr,
                          bx.y * sr + normal_after.y * deviation_rate + sn.y * pr,
                          bx.z * sr + normal_after.z * deviation_rate + sn.z * pr};
        const DV* vecs[4] = {&cn, &sn, &nn, &rel};
        for (int j = 0; j < 4; ++j) {
            const Du* comp[3] = {&vecs[j]->x, &vecs[j]->y, &vecs[j]->z};
            for (int c = 0; c < 3; ++c) {
                out->v[sidx][j][c] = comp[c]->v;
                for (int k = 0; k < NP; ++k) out->d[sidx][j][c][k] = comp[c]->d[k];
            }
        }
    }
}

__device__ __forceinline__ DV frame_vec(const FrameTangent& ft, int side, int j) {
    DV r;
    Du* comp[3] = {&r.x, &r.y, &r.z};
    for (int c = 0; c < 3; ++c) {
        comp[c]->v = ft.v[side][j][c];
#pragma unroll
        for (int k = 0; k < NP; ++k) comp[c]->d[k] = ft.d[side][j][c][k];
    }
    return r;
}

// Vertex position and lattice velocity (k_mesh_prepare) on duals.
__device__ void vertex_dual(const GeomArgs& a, const FrameTangent& ft, uint32_t i, DV& pos, DV& vel) {
    const Prepared& p = a.b.state->prep;
    const V3 l = v3(a.b.mesh_local[3 * i], a.b.mesh_local[3 * i + 1], a.b.mesh_local[3 * i + 2]);
    const uint8_t seg = a.b.mesh_segment[i];
    const float v2l = a.fp.v2l;
    if (seg == 0) {
        const V3 r = qrotate(p.orientation, l);
        const V3 w = v3(p.body_position.x + r.x, p.body_position.y + r.y, p.body_position.z + r.z);
        const V3 cr = cross(v3(p.omega_body_world), r);
        const V3 v = v3(p.linear_velocity.x + cr.x, p.linear_velocity.y + cr.y, p.linear_velocity.z + cr.z);
        pos = dv(w);
        vel = dv(v3(v.x * v2l, v.y * v2l, v.z * v2l));
        return;
    }
    const int side = seg == 1 ? 0 : 1;
    const V3 root = v3(side == 0 ? p.left_root : p.right_root);
    const DV chord = frame_vec(ft, side, 0), span = frame_vec(ft, side, 1), normal = frame_vec(ft, side, 2);
    const DV rel = frame_vec(ft, side, 3);
    pos = DV{dc(root.x) + chord.x * l.x + span.x * l.y + normal.x * l.z,
             dc(root.y) + chord.y * l.x + span.y * l.y + normal.y * l.z,
             dc(root.z) + chord.z * l.x + span.z * l.y + normal.z * l.z};
    const DV rb = pos - dv(v3(p.body_position));
    const DV cr = dcross(v3(p.omega_body_world), rb);
    const DV rr = pos - dv(root);
    const DV cw = dcross(rel, rr);
    const DV v = DV{dc(p.linear_velocity.x) + cr.x + cw.x, dc(p.linear_velocity.y) + cr.y + cw.y,
                    dc(p.linear_velocity.z) + cr.z + cw.z};
    vel = DV{v.x * v2l, v.y * v2l, v.z * v2l};
}

// Triangle closest point (the forward closest_point) with dual vertices.
__device__ DV closest_point_dual(V3 p, const DV& a, const DV& b, const DV& c, Du (&bary)[3]) {
    const DV P = dv(p);
    const DV ab = b - a, ac = c - a, ap = P - a;
    const Du d1 = ddot(ab, ap), d2 = ddot(ac, ap);
    if (d1.v <= 0.0f && d2.v <= 0.0f) {
        bary[0] = dc(1.0f);
        bary[1] = dc(0.0f);
        bary[2] = dc(0.0f);
        return a;
    }
    const DV bp = P - b;
    const Du d3 = ddot(ab, bp), d4 = ddot(ac, bp);
    if (d3.v >= 0.0f && d4.v <= d3.v) {
        bary[0] = dc(0.0f);
        bary[1] = dc(1.0f);
        bary[2] = dc(0.0f);
        return b;
    }
    const Du vc = d1 * d4 - d3 * d2;
    if (vc.v <= 0.0f && d1.v >= 0.0f && d3.v <= 0.0f) {
        const Du v = d1 / (d1 - d3);
        bary[0] = dc(1.0f) - v;
        bary[1] = v;
        bary[2] = dc(0.0f);
        return DV{a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z};
    }
    const DV cp = P - c;
    const Du d5 = ddot(ab, cp), d6 = ddot(ac, cp);
    if (d6.v >= 0.0f && d5.v <= d6.v) {
        bary[0] = dc(0.0f);
        bary[1] = dc(0.0f);
        bary[2] = dc(1.0f);
        return c;
    }
    const Du vb = d5 * d2 - d1 * d6;
    if (vb.v <= 0.0f && d2.v >= 0.0f && d6.v <= 0.0f) {
        const Du w = d2 / (d2 - d6);
        bary[0] = dc(1.0f) - w;
        bary[1] = dc(0.0f);
        bary[2] = w;
        return DV{a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z};
    }
    const Du va = d3 * d6 - d5 * d4;
    const Du e1 = d4 - d3, e2 = d5 - d6;
    if (va.v <= 0.0f && e1.v >= 0.0f && e2.v >= 0.0f) {
        const Du w = e1 / (e1 + e2);
        bary[0] = dc(0.0f);
        bary[1] = dc(1.0f) - w;
        bary[2] = w;
        const DV cb = c - b;
        return DV{b.x + w * cb.x, b.y + w * cb.y, b.z + w * cb.z};
    }
    Du sum = va + vb + vc;
    if (sum.v < 1.0e-20f) sum = dc(1.0e-20f);
    const Du inv = dc(1.0f) / sum;
    const Du v = vb * inv, w = vc * inv;
    bary[0] = dc(1.0f) - v - w;
    bary[1] = v;
    bary[2] = w;
    return DV{a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w};
}

struct CellDual {
    DV u;      // wall velocity (lattice)
    Du sd;     // signed distance (cells)
    bool valid;
};

// k_mesh_resolve's wall velocity and signed distance of a cell whose winning
// triangle is t, on duals.
__device__ CellDual cell_dual(const GeomArgs& a, const FrameTangent& ft, uint32_t t, V3 world) {
    CellDual r;
    r.valid = t < a.b.ntris;
    if (!r.valid) {
        r.u = dv(v3(0.0f, 0.0f, 0.0f));
        r.sd = dc(16.0f);
        return r;
    }
    DV P[3], U[3];
    for (int j = 0; j < 3; ++j) vertex_dual(a, ft, a.b.mesh_tris[3 * t + j], P[j], U[j]);
    Du bary[3];
    const DV cp = closest_point_dual(world, P[0], P[1], P[2], bary);
    r.u = DV{bary[0] * U[0].x + bary[1] * U[1].x + bary[2] * U[2].x,
             bary[0] * U[0].y + bary[1] * U[1].y + bary[2] * U[2].y,
             bary[0] * U[0].z + bary[1] * U[1].z + bary[2] * U[2].z};
    const DV diff = dv(world) - cp;
    const Du sd = dsqrt(ddot(diff, diff)) - dc(a.b.half_thickness);
    r.sd.v = sd.v / a.fp.dx;
#pragma unroll
    for (int k = 0; k < NP; ++k) r.sd.d[k] = sd.d[k] / a.fp.dx;
    return r;
}

__device__ __forceinline__ uint32_t key_triangle(unsigned long long key) {
    return key == 0xFFFFFFFFFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)(key & 0xFFFFFFFFull);
}

// ---------------------------------------------------------------------------
// Per-link tangents (taped forward step, after k_links_emit).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_link_tangent(const GeomArgs a, int link_rule, int interpolated, float* out) {
    const FrameTangent& ft = *a.b.frames;
    const Grid& g = a.g;
    int64_t count = a.b.state->link_count;
    if (count > (int64_t)a.b.link_capacity) count = a.b.link_capacity;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        float* o = out + (size_t)kLinkTangentWords * i;
        const uint32_t gid = a.b.link_cell[i];
        const int q = (int)(a.b.link_meta[i] & 0xFF);
        int x, y, z;
        unflat(g, gid, x, y, z);
        int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
        if (!wrap(g, sx, sy, sz)) {
            for (int k = 0; k < kLinkTangentWords; ++k) o[k] = 0.0f;
            continue;
        }
        const V3 fw = cell_world(a.fp, x, y, z), sw = cell_world(a.fp, sx, sy, sz);
        const unsigned long long kf = box_key(a, x, y, z), ks = box_key(a, sx, sy, sz);
        const CellDual cf = cell_dual(a, ft, key_triangle(kf), fw);
        const CellDual cs = cell_dual(a, ft, key_triangle(ks), sw);
        Du qd = dc(0.0f);
        if (interpolated) {
            if (link_rule == BFX_LINK_LINEAR) {
                const Du fd = cf.sd.v > 0.0f ? cf.sd : dc(0.0f);
                const Du sd = cs.sd.v < 0.0f ? cs.sd : dc(0.0f);
                Du den = fd - sd;
                if (den.v < 1.0e-6f) den = dc(1.0e-6f);
                const Du qq = fd / den;
                if (qq.v >= 1.0e-4f && qq.v <= 1.0f) qd = qq;
            } else {
                // ray root: the forward bisection, then dq = -g_theta / g_s at the root
                const uint32_t ta = key_triangle(ks);
                uint32_t tb = kf == 0xFFFFFFFFFFFFFFFFull ? ta : key_triangle(kf);
                if (tb >= a.b.ntris) tb = ta;
                if (ta < a.b.ntris) {
                    const float h = a.b.half_thickness;
                    float lo = 0.0f, hi = 1.0f;
                    bool found = false;
                    for (int k = 1; k <= 8; ++k) {
                        const float t = (float)k * 0.125f;
                        const V3 s = v3(mixf(fw.x, sw.x, t), mixf(fw.y, sw.y, t), mixf(fw.z, sw.z, t));
                        if (fminf(tri_distance(a, ta, s), tri_distance(a, tb, s)) - h <= 0.0f) {
                            hi = t;
                            found = true;
                            break;
                        }
                        lo = t;
                    }
                    if (found) {
                        for (int it = 0; it < 24; ++it) {
                            const float mid = 0.5f * (lo + hi);
                            const V3 s = v3(mixf(fw.x, sw.x, mid), mixf(fw.y, sw.y, mid), mixf(fw.z, sw.z, mid));
                            if (fminf(tri_distance(a, ta, s), tri_distance(a, tb, s)) - h <= 0.0f) hi = mid;
                            else lo = mid;
                        }
                        const float sq = 0.5f * (lo + hi);
                        if (sq >= 1.0e-4f && sq <= 1.0f) {
                            const V3 ps = v3(mixf(fw.x, sw.x, sq), mixf(fw.y, sw.y, sq), mixf(fw.z, sw.z, sq));
                            const float da = tri_distance(a, ta, ps), db = tri_distance(a, tb, ps);
                            const uint32_t tw = da <= db ? ta : tb;
                            DV P[3], U[3];
                            for (int j = 0; j < 3; ++j) vertex_dual(a, ft, a.b.mesh_tris[3 * tw + j], P[j], U[j]);
                            Du bary[3];
                            const DV cp = closest_point_dual(ps, P[0], P[1], P[2], bary);
                            const DV diff = dv(ps) - cp;
                            const Du dist = dsqrt(ddot(diff, diff));
                            if (dist.v > 1.0e-12f) {
                                const V3 n = v3(diff.x.v / dist.v, diff.y.v / dist.v, diff.z.v / dist.v);
                                const float gs = dot(n, sw - fw);
                                if (fabsf(gs) > 1.0e-9f * a.fp.dx) {
                                    qd.v = sq;
                                    for (int k = 0; k < NP; ++k) qd.d[k] = -dist.d[k] / gs;
                                }
                            }
                        }
                    }
                }
            }
        }
        for (int k = 0; k < NP; ++k) {
            o[k] = qd.d[k];
            o[4 + 3 * k + 0] = cf.u.x.d[k];
            o[4 + 3 * k + 1] = cf.u.y.d[k];
            o[4 + 3 * k + 2] = cf.u.z.d[k];
            o[16 + 3 * k + 0] = cs.u.x.d[k];
            o[16 + 3 * k + 1] = cs.u.y.d[k];
            o[16 + 3 * k + 2] = cs.u.z.d[k];
        }
    }
}

// ---------------------------------------------------------------------------
// Transposed TRT collision.  post_i = f_i - w+ (f+_i - e+_i) - w- (f-_i - e-_i)
// with e = equilibrium(rho(f), u(f)).  For an adjoint lambda of post, with
// Lam_i = w+ lambda+_i + w- lambda-_i:
//   mu_j = lambda_j - Lam_j + A + B . (c_j - u),
//   A   = sum_i Lam_i e_i / rho,
//   B_a = sum_i Lam_i w_i (3 c_ia + 9 (c_i.u) c_ia - 3 u_a)
// (the density cancels, so only the velocity is taped).
// ---------------------------------------------------------------------------
template <class R>
__device__ __forceinline__ void trt_adjoint(const R (&lam)[19], R ux, R uy, R uz, R wp, R wm, R (&mu)[19]) {
    const R u2 = ux * ux + uy * uy + uz * uz;
    R L[19];
    L[0] = wp * lam[0];
    R A = L[0] * Lat<R>::w0 * (R(1) - R(1.5) * u2);
    R Bx = L[0] * Lat<R>::w0 * (R(-3) * ux), By = L[0] * Lat<R>::w0 * (R(-3) * uy),
      Bz = L[0] * Lat<R>::w0 * (R(-3) * uz);
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const R lp = R(0.5) * (lam[q] + lam[q + 1]);
        const R lm = R(0.5) * (lam[q] - lam[q + 1]);
        const R Lq = wp * lp + wm * lm, Lo = wp * lp - wm * lm;
        L[q] = Lq;
        L[q + 1] = Lo;
        const R w = wq<R>(q);
        const R cu = cdotq<R>(q, ux, uy, uz);
        const R even = R(1) + R(4.5) * cu * cu - R(1.5) * u2;
        const R S = Lq + Lo, D = Lq - Lo;
        A += w * (S * even + D * (R(3) * cu));
        const R k1 = R(3) * D + R(9) * cu * S;
        if (cx(q)) Bx += w * (R(cx(q)) * k1);
        if (cy(q)) By += w * (R(cy(q)) * k1);
        if (cz(q)) Bz += w * (R(cz(q)) * k1);
        Bx -= w * (R(3) * ux * S);
        By -= w * (R(3) * uy * S);
        Bz -= w * (R(3) * uz * S);
    }
    const R base = A - (Bx * ux + By * uy + Bz * uz);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        R m = lam[q] - L[q] + base;
        if (cx(q)) m += R(cx(q)) * Bx;
        if (cy(q)) m += R(cy(q)) * By;
        if (cz(q)) m += R(cz(q)) * Bz;
        mu[q] = m;
    }
}

// G_b = sum_q lam_q d equilibrium_q(1, u) / du_b
template <class R>
__device__ __forceinline__ void feq_velocity_adjoint(const R (&lam)[19], R ux, R uy, R uz, R (&G)[3]) {
    G[0] = G[1] = G[2] = R(0);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const R w = wq<R>(q);
        const R cu = cdotq<R>(q, ux, uy, uz);
        G[0] += lam[q] * w * (R(3 * cx(q)) + R(9) * cu * R(cx(q)) - R(3) * ux);
        G[1] += lam[q] * w * (R(3 * cy(q)) + R(9) * cu * R(cy(q)) - R(3) * uy);
        G[2] += lam[q] * w * (R(3 * cz(q)) + R(9) * cu * R(cz(q)) - R(3) * uz);
    }
}

// ---------------------------------------------------------------------------
// Adjoint kernels.
// ---------------------------------------------------------------------------
struct AdjArgs {
    GeomArgs ga;                // taped geometry (state, masks, keys), mesh, grid, parameters
    void* lam;
    void* plane[19];
    int32_t doff[19];
    const void* moments;
    const void* links;
    void* nu;
    double* part_rare;
    double* part_links;
    Objective* obj;
    double weight;              // objective weight of this step
};

// Slot a real cell reads as its incoming direction q (see incoming_slot).
template <class T>
__device__ __forceinline__ T* incoming_slot_raw(T* A, const Grid& g, int rep_s, int q, int x, int y, int z) {
    if (rep_s) return A + (int64_t)q * g.pn + pflat(g, x, y, z);
    return A + (int64_t)opp(q) * g.pn + pflat(g, x - cx(q), y - cy(q), z - cz(q));
}

// Slot holding f*_q(x) in representation rep_s (see canon_load).
template <class T>
__device__ __forceinline__ T* canon_slot(T* A, const Grid& g, int rep_s, int q, int x, int y, int z) {
    if (!rep_s) return A + (int64_t)opp(q) * g.pn + pflat(g, x, y, z);
    return A + (int64_t)q * g.pn + pflat(g, x + cx(q), y + cy(q), z + cz(q));
}

// Fluid cells: reverse streaming through the transposed collision.
template <class R, int REP_S>
__global__ void __launch_bounds__(256) k_adj_bulk(const AdjArgs a) {
    const Grid& g = a.ga.g;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= g.nx || y >= g.ny) return;
    const uint32_t gid = (uint32_t)x + (uint32_t)g.nx * ((uint32_t)y + (uint32_t)g.ny * (uint32_t)z);
    if (a.ga.b.mask_next[gid]) return;
    const uint32_t pid = (uint32_t)(x + 1) + (uint32_t)g.px * ((uint32_t)(y + 1) + (uint32_t)g.py * (uint32_t)(z + 1));
    R lam[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (REP_S) lam[q] = ((const R*)a.plane[opp(q)])[pid];
        else lam[q] = ((const R*)a.plane[q])[(uint32_t)(pid + (uint32_t)a.doff[q])];
    }
    const R* m = (const R*)a.moments + 4 * (size_t)gid;
    const R ux = m[1], uy = m[2], uz = m[3];
    const FluidParams& fp = a.ga.fp;
    if (fp.has_sponge) {
        const float sp = sponge_factor(g, fp, x, y, z);
        if (sp > 0.0f) {
            const R keep = R(1) - (R)sp;
#pragma unroll
            for (int q = 0; q < 19; ++q) lam[q] *= keep;
        }
    }
    R mu[19];
    trt_adjoint<R>(lam, ux, uy, uz, (R)fp.omega_p, (R)fp.omega_m, mu);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        if (REP_S) ((R*)a.plane[q])[pid] = mu[q];
        else ((R*)a.plane[opp(q)])[(uint32_t)(pid - (uint32_t)a.doff[q])] = mu[q];
    }
}

template <int K>
__device__ __forceinline__ void write_partials(double (&v)[K], double* out) {
    __shared__ double sh[K][256];
    // most blocks contribute nothing: skip their tree (a sum of zeros is 0)
    bool nonzero = false;
    for (int k = 0; k < K; ++k) nonzero = nonzero || v[k] != 0.0;
    if (__syncthreads_or(nonzero)) block_sum<K>(v, sh);
    const int block = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (linear_tid() == 0)
        for (int k = 0; k < K; ++k) out[K * block + k] = v[k];
}

// Solid and newly uncovered cells of the box.
template <class R, int REP_S>
__global__ void __launch_bounds__(256) k_adj_rare(const AdjArgs a) {
    const GeomArgs& ga = a.ga;
    const Grid& g = ga.g;
    const FluidParams& fp = ga.fp;
    double grad[NP] = {0.0, 0.0, 0.0, 0.0};
    int x, y, z;
    int64_t bidx;
    if (block_inactive(ga)) {
        // flagged cells lie within the active bounds
        const int block = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        if (linear_tid() == 0)
            for (int k = 0; k < NP; ++k) a.part_rare[NP * block + k] = 0.0;
        return;
    }
    if (box_cell(ga, x, y, z, bidx) && cell_active(ga, x, y, z)) {
        const int64_t gid = flat(g, x, y, z);
        const uint8_t mk = ga.b.mask_next[gid];
        if (mk) {
            const uint32_t pid = (uint32_t)pflat(g, x, y, z);
            R lam[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                R* slot = REP_S ? (R*)a.plane[opp(q)] + pid : (R*)a.plane[q] + (uint32_t)(pid + (uint32_t)a.doff[q]);
                lam[q] = *slot;
                *slot = R(0);
            }
            const V3 world = cell_world(fp, x, y, z);
            const CellDual cd = cell_dual(ga, *ga.b.frames, key_triangle(ga.b.keys[bidx]), world);
            const R ux = (R)cd.u.x.v, uy = (R)cd.u.y.v, uz = (R)cd.u.z.v;
            R G[3];
            if (mk & kPartMask) {
                feq_velocity_adjoint<R>(lam, ux, uy, uz, G);
            } else {
                // newly uncovered: equilibrium refill, collision, sponge
                const R u2 = ux * ux + uy * uy + uz * uz;
                R f[19];
#pragma unroll
                for (int q = 0; q < 19; ++q) f[q] = feqq<R>(q, R(1), ux, uy, uz, u2);
                R rho = 0, mx = 0, my = 0, mz = 0;
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    rho += f[q];
                    mx += f[q] * (R)cx(q);
                    my += f[q] * (R)cy(q);
                    mz += f[q] * (R)cz(q);
                }
                rho = rho > R(1.0e-8) ? rho : R(1.0e-8);
                if (fp.has_sponge) {
                    const float sp = sponge_factor(g, fp, x, y, z);
                    if (sp > 0.0f)
                        for (int q = 0; q < 19; ++q) lam[q] *= R(1) - (R)sp;
                }
                R mu[19];
                trt_adjoint<R>(lam, mx / rho, my / rho, mz / rho, (R)fp.omega_p, (R)fp.omega_m, mu);
                feq_velocity_adjoint<R>(mu, ux, uy, uz, G);
                // refill momentum of the uncover impulse: d(sum_q feq_q(1,u) c_q)/du = identity
                if (a.weight != 0.0 && fp.accumulate && fp.force_mode == 6 && (!fp.interpolated || fp.load_component != 1)) {
                    for (int c = 0; c < 3; ++c) G[c] -= (R)(a.weight * (double)fp.f2p * a.obj->force_weight[c]);
                }
            }
            const Du* du[3] = {&cd.u.x, &cd.u.y, &cd.u.z};
            for (int k = 0; k < NP; ++k)
                for (int c = 0; c < 3; ++c) grad[k] += (double)G[c] * (double)du[c]->d[k];
        }
    }
    write_partials<NP>(grad, a.part_rare);
}

// Links, pass 1: consume the adjoint of the bounce-back value.
template <class R>
__global__ void __launch_bounds__(256) k_adj_links1(const AdjArgs a, int rep_s) {
    const GeomArgs& ga = a.ga;
    const Grid& g = ga.g;
    const FluidParams& fp = ga.fp;
    const LinkTape<R>* links = (const LinkTape<R>*)a.links;
    R* lamA = (R*)a.lam;
    double grad[NP] = {0.0, 0.0, 0.0, 0.0};
    int64_t count = ga.b.state->link_count;
    if (count > (int64_t)ga.b.link_capacity) count = ga.b.link_capacity;
    const double W = a.weight;
    const double wF[3] = {a.obj->force_weight[0], a.obj->force_weight[1], a.obj->force_weight[2]};
    const double wP = a.obj->power_weight;
    const double f2p = (double)fp.f2p, v2l = (double)fp.v2l;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const LinkTape<R>& t = links[i];
        const int q = (int)t.dir;
        int x, y, z;
        unflat(g, t.cell, x, y, z);
        R* in = incoming_slot_raw(lamA, g, rep_s, q, x, y, z);
        const R mu = *in;
        *in = R(0);
        const double c[3] = {(double)cx(q), (double)cy(q), (double)cz(q)};
        const double cwv = c[0] * (double)t.wv[0] + c[1] * (double)t.wv[1] + c[2] * (double)t.wv[2];
        // J contribution of the link: W f2p (value + reflected) (-wF.c + wP (c.wv) / v2l)
        const double kappa = W * f2p * (-(wF[0] * c[0] + wF[1] * c[1] + wF[2] * c[2]) + wP * cwv / v2l);
        const R nu = mu + (R)kappa;
        const R qf = t.q;
        const R mwd = (R)fp.far[3];
        const R wqv = q <= 6 ? Lat<R>::w1 : Lat<R>::w2;
        const R wc = R(2) * wqv * mwd * (R)cwv / Lat<R>::cs2;
        R dvdr = R(1), dvdq = R(0), dvdwc = R(1);
        if (t.kase == 1) {
            dvdr = R(2) * qf;
            dvdq = R(2) * t.reflected - R(2) * t.other;
        } else if (t.kase == 2) {
            const R tq = R(2) * qf;
            dvdr = R(1) / tq;
            dvdwc = R(1) / tq;
            dvdq = (t.other - t.reflected - wc) / (tq * qf);
        }
        *canon_slot(lamA, g, rep_s, opp(q), x, y, z) += nu * dvdr + (R)kappa;
        if (t.kase == 1) *canon_slot(lamA, g, rep_s, opp(q), x + cx(q), y + cy(q), z + cz(q)) += nu * (R(1) - R(2) * qf);
        if (t.kase == 2) ((R*)a.nu)[i] = nu;
        const double gwc = (double)(nu * dvdwc) * (2.0 * (double)wqv * (double)mwd / (double)Lat<R>::cs2);
        const double gval = W * f2p * wP * ((double)t.value + (double)t.reflected) / v2l;
        double gwv[3];
        for (int k = 0; k < 3; ++k) gwv[k] = (gwc + gval) * c[k];
        for (int k = 0; k < NP; ++k)
            grad[k] += (double)(nu * dvdq) * (double)t.dq[k] + gwv[0] * (double)t.dwv[k][0] +
                       gwv[1] * (double)t.dwv[k][1] + gwv[2] * (double)t.dwv[k][2];
    }
    write_partials<NP>(grad, a.part_links);
}

// Links, pass 2: the interpolation partner f*_q(x) of the q > 1/2 case.
template <class R>
__global__ void __launch_bounds__(256) k_adj_links2(const AdjArgs a, int rep_s) {
    const GeomArgs& ga = a.ga;
    const Grid& g = ga.g;
    const LinkTape<R>* links = (const LinkTape<R>*)a.links;
    int64_t count = ga.b.state->link_count;
    if (count > (int64_t)ga.b.link_capacity) count = ga.b.link_capacity;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const LinkTape<R>& t = links[i];
        if (t.kase != 2) continue;
        int x, y, z;
        unflat(g, t.cell, x, y, z);
        const R tq = R(2) * t.q;
        *canon_slot((R*)a.lam, g, rep_s, (int)t.dir, x, y, z) += ((const R*)a.nu)[i] * ((tq - R(1)) / tq);
    }
}

// Halo: the adjoint of a periodic copy goes to its image; face constants drop it.
template <class R>
__global__ void __launch_bounds__(128) k_adj_halo(const AdjArgs a, int rep_s, int64_t halo_cells) {
    const Grid& g = a.ga.g;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= halo_cells) return;
    int hx, hy, hz;
    if (!padded_shell_cell(g, t, hx, hy, hz)) return;
    hx -= 1;
    hy -= 1;
    hz -= 1;
    R* A = (R*)a.lam;
    // two passes, as in k_halo: the loads read halo-facing slots (rep E:
    // A[opp q][h]; rep S: A[q][h + c_q]) and the image stores write
    // A[opp q][w] / A[q][w + c_q] of a real cell w, which no load reads
    R v[19];
    uint32_t live = 0;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const int bx = hx + cx(q), by = hy + cy(q), bz = hz + cz(q);
        if (!inside(g, bx, by, bz)) continue;
        live |= 1u << q;
        const R* slot = rep_s ? A + (int64_t)q * g.pn + pflat(g, bx, by, bz) : A + (int64_t)opp(q) * g.pn + pflat(g, hx, hy, hz);
        v[q] = *slot;
    }
    int wx = hx, wy = hy, wz = hz;
    const bool image = wrap(g, wx, wy, wz);
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        if (!(live & (1u << q))) continue;
        const int bx = hx + cx(q), by = hy + cy(q), bz = hz + cz(q);
        R* slot = rep_s ? A + (int64_t)q * g.pn + pflat(g, bx, by, bz) : A + (int64_t)opp(q) * g.pn + pflat(g, hx, hy, hz);
        *slot = R(0);
        if (image) *canon_slot(A, g, rep_s, q, wx, wy, wz) = v[q];
    }
}

// Cover / uncover impulses (the forward k_topology): pass 0 covered, pass 1 uncovered.
template <class R>
__global__ void __launch_bounds__(256) k_adj_topology(const AdjArgs a, int rep_s, int pass) {
    const GeomArgs& ga = a.ga;
    const Grid& g = ga.g;
    const FluidParams& fp = ga.fp;
    int x, y, z;
    int64_t bidx;
    if (block_inactive(ga)) return;
    if (!box_cell(ga, x, y, z, bidx) || !cell_active(ga, x, y, z)) return;
    if (!fp.accumulate || (fp.interpolated && fp.load_component == 1)) return;
    const int64_t gid = flat(g, x, y, z);
    const uint8_t mk = ga.b.mask_next[gid];
    const double s = a.weight * (double)fp.f2p;
    const double* wF = a.obj->force_weight;
    R* A = (R*)a.lam;
    if (pass == 0 && (mk & kCovered)) {
        for (int q = 0; q < 19; ++q) {
            const double c = wF[0] * cx(q) + wF[1] * cy(q) + wF[2] * cz(q);
            if (c != 0.0) *canon_slot(A, g, rep_s, q, x, y, z) += (R)(s * c);
        }
    } else if (pass == 1 && (mk & kUncovered) && fp.force_mode == 6) {
        for (int q = 1; q < 19; ++q) {
            const int nx_ = x + cx(q), ny_ = y + cy(q), nz_ = z + cz(q);
            if (!inside(g, nx_, ny_, nz_)) continue;
            const int64_t nb = flat(g, nx_, ny_, nz_);
            if (!((ga.b.mask_prev[nb] & kPartMask) == 0 && (ga.b.mask_next[nb] & kPartMask) == 0)) continue;
            const double c = wF[0] * cx(q) + wF[1] * cy(q) + wF[2] * cz(q);
            if (c == 0.0) continue;
            *canon_slot(A, g, rep_s, q, x, y, z) -= (R)(s * c);
            *canon_slot(A, g, rep_s, opp(q), nx_, ny_, nz_) -= (R)(s * c);
        }
    }
}

// Initial state: k_init writes equilibrium(1, u_wall(t = 0)) into the cells
// that are solid at t = 0, so lambda^0 of those cells feeds dJ/dtheta through
// the initial wall velocity.
template <class R>
__global__ void __launch_bounds__(256) k_adj_init(const AdjArgs a, int rep_s) {
    const GeomArgs& ga = a.ga;
    const Grid& g = ga.g;
    double grad[NP] = {0.0, 0.0, 0.0, 0.0};
    int x, y, z;
    int64_t bidx;
    if (box_cell(ga, x, y, z, bidx)) {
        const int64_t gid = flat(g, x, y, z);
        if (ga.b.mask_next[gid] & kPartMask) {
            R lam[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) lam[q] = *canon_slot((const R*)a.lam, g, rep_s, q, x, y, z);
            const V3 world = cell_world(ga.fp, x, y, z);
            const CellDual cd = cell_dual(ga, *ga.b.frames, key_triangle(ga.b.keys[bidx]), world);
            R G[3];
            feq_velocity_adjoint<R>(lam, (R)cd.u.x.v, (R)cd.u.y.v, (R)cd.u.z.v, G);
            const Du* du[3] = {&cd.u.x, &cd.u.y, &cd.u.z};
            for (int k = 0; k < NP; ++k)
                for (int c = 0; c < 3; ++c) grad[k] += (double)G[c] * (double)du[c]->d[k];
        }
    }
    write_partials<NP>(grad, a.part_rare);
}

__global__ void k_adj_reduce(const double* rare, int nrare, const double* links, int nlinks, Objective* obj) {
    __shared__ double sh[NP][256];
    double acc[NP] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < nrare; i += blockDim.x)
        for (int k = 0; k < NP; ++k) acc[k] += rare[NP * i + k];
    for (int i = threadIdx.x; i < nlinks; i += blockDim.x)
        for (int k = 0; k < NP; ++k) acc[k] += links[NP * i + k];
    block_sum<NP>(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < NP; ++k) obj->grad[k] += acc[k];
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
void launch_frame_tangent(const GeomBuffers& gb, float dt, int init, FrameTangent* out, cudaStream_t s) {
    k_frame_tangent<<<1, 1, 0, s>>>(gb.bird, gb.state, dt, init, out);
}

void launch_link_tangent(int link_rule, int interpolated, const GridDesc& g, const FluidParams& fp,
                         const BoxDesc& box, const GeomBuffers& gb, float* out, cudaStream_t s) {
    GeomArgs a = make_geom(g, fp, box, gb, nullptr);
    const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(4096, ((int64_t)gb.link_capacity + 127) / 128));
    k_link_tangent<<<blocks, 128, 0, s>>>(a, link_rule, interpolated, out);
}

template <class R>
static void adjoint_step_t(int rep_s, const GridDesc& gd, const BoxDesc& box, AdjArgs& a, int apply_blocks,
                           cudaStream_t s) {
    dim3 bgrid, bblock;
    box_shape(box, bgrid, bblock);
    dim3 cgrid, cblock;
    cell_launch_shape(gd, cgrid, cblock);
    if (rep_s) {
        k_adj_rare<R, 1><<<bgrid, bblock, 0, s>>>(a);
        k_adj_bulk<R, 1><<<cgrid, cblock, 0, s>>>(a);
    } else {
        k_adj_rare<R, 0><<<bgrid, bblock, 0, s>>>(a);
        k_adj_bulk<R, 0><<<cgrid, cblock, 0, s>>>(a);
    }
    k_adj_links1<R><<<apply_blocks, 256, 0, s>>>(a, rep_s);
    k_adj_links2<R><<<apply_blocks, 256, 0, s>>>(a, rep_s);
    const int64_t halo = a.ga.g.pn - a.ga.g.n;
    k_adj_halo<R><<<(unsigned)((halo + 127) / 128), 128, 0, s>>>(a, rep_s, halo);
    k_adj_topology<R><<<bgrid, bblock, 0, s>>>(a, rep_s, 0);
    k_adj_topology<R><<<bgrid, bblock, 0, s>>>(a, rep_s, 1);
    k_adj_reduce<<<1, 256, 0, s>>>(a.part_rare, (int)(bgrid.x * bgrid.y * bgrid.z), a.part_links, apply_blocks, a.obj);
}

static AdjArgs adjoint_args(int storage, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                            const GeomBuffers& gb, const StepTape& tape, const AdjointWork& w, double weight) {
    GeomBuffers tb = gb;
    tb.mask_next = (uint8_t*)tape.mask_next;
    tb.mask_prev = (uint8_t*)tape.mask_prev;
    tb.keys = (unsigned long long*)tape.keys;
    tb.state = (DeviceState*)tape.state;
    tb.frames = tape.frames;
    AdjArgs a;
    a.ga = make_geom(g, fp, box, tb, nullptr);
    a.lam = w.lam;
    const size_t elem = storage == BFX_STORAGE_F64 ? 8 : 4;
    for (int q = 0; q < 19; ++q) {
        a.plane[q] = (char*)w.lam + (size_t)q * (size_t)a.ga.g.pn * elem;
        a.doff[q] = (int32_t)((int64_t)cx(q) + (int64_t)a.ga.g.px * cy(q) + a.ga.g.pxy * cz(q));
    }
    a.moments = tape.moments;
    a.links = tape.links;
    a.nu = w.nu;
    a.part_rare = w.partials_rare;
    a.part_links = w.partials_links;
    a.obj = w.objective;
    a.weight = weight;
    return a;
}

void launch_adjoint_step(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                         const GeomBuffers& gb, const StepTape& tape, const AdjointWork& w, double weight,
                         cudaStream_t s) {
    AdjArgs a = adjoint_args(storage, g, fp, box, gb, tape, w, weight);
    if (storage == BFX_STORAGE_F64) adjoint_step_t<double>(rep_s, g, box, a, gb.apply_blocks, s);
    else adjoint_step_t<float>(rep_s, g, box, a, gb.apply_blocks, s);
}

void launch_adjoint_init(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                         const GeomBuffers& gb, const StepTape& init, const AdjointWork& w, cudaStream_t s) {
    AdjArgs a = adjoint_args(storage, g, fp, box, gb, init, w, 0.0);
    dim3 bgrid, bblock;
    box_shape(box, bgrid, bblock);
    if (storage == BFX_STORAGE_F64) k_adj_init<double><<<bgrid, bblock, 0, s>>>(a, rep_s);
    else k_adj_init<float><<<bgrid, bblock, 0, s>>>(a, rep_s);
    k_adj_reduce<<<1, 256, 0, s>>>(a.part_rare, (int)(bgrid.x * bgrid.y * bgrid.z), a.part_links, 0, a.obj);
}

}  // namespace bfx
