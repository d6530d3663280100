// Moving-boundary kernels of the D3Q19 step: pose preparation, cell
// classification (analytic bird, ellipsoid, articulated triangle mesh), cut-link
// compaction, interpolated moving-wall bounce-back with momentum exchange,
// cover/uncover topology impulses, FP64 load reduction and the FP64 6-DOF
// update.  Each kernel cites the reference kernel it restates
// (Sources/BirdFlowMetal/Metal/BirdFlow.metal, "BF.metal").
//
// Geometry work is confined to a box that follows the body (its extent is
// fixed at creation from the conservative body radius plus a 4-cell margin,
// its origin is recomputed on the device every step), so a step costs
// O(box) here and O(lattice) only in the fused fluid kernel.
#include <algorithm>

#include "bfx_geom_common.cuh"

namespace bfx {


struct WingFrame {
    V3 root, chord, span, normal, rel;
    float tip_twist, tip_rate;
};

// Sine and cosine of one rotation angle.
struct SinCos {
    float s, c;
};

// makeWingFrame: BF.metal:611-684, with the sines and cosines of the signed
// stroke, the deviation and the signed pitch given.
__device__ void make_wing_frame(float side, SinCos stroke, float stroke_rate, SinCos deviation, float deviation_rate,
                                SinCos pitch, float pitch_rate, const bfx_bird& bird, V3 pos, float4 orient,
                                WingFrame& fr) {
    float4 o = qnormalize(orient);
    V3 bx = qrotate(o, v3(1, 0, 0)), by = qrotate(o, v3(0, 1, 0)), bz = qrotate(o, v3(0, 0, 1));
    V3 root_local = v3(bird.wing_geometry1.v[1], side * bird.wing_geometry1.v[2], bird.wing_geometry1.v[3]);
    V3 rr = qrotate(o, root_local);
    V3 root = pos + rr;
    V3 span_after = rotate_axis_sc(v3(side * by.x, side * by.y, side * by.z), bx, stroke.s, stroke.c);
    V3 normal_after = rotate_axis_sc(v3(side * bz.x, side * bz.y, side * bz.z), bx, stroke.s, stroke.c);
    V3 span = rotate_axis_sc(span_after, normal_after, deviation.s, deviation.c);
    V3 chord_before = rotate_axis_sc(bx, normal_after, deviation.s, deviation.c);
    V3 chord = rotate_axis_sc(chord_before, span, pitch.s, pitch.c);
    V3 normal = rotate_axis_sc(normal_after, span, pitch.s, pitch.c);
    fr.root = root;
    fr.chord = normalize3(chord);
    fr.span = normalize3(span);
    fr.normal = normalize3(normal);
    float sr = side * stroke_rate, pr = side * pitch_rate;
    fr.rel = v3(bx.x * sr + normal_after.x * deviation_rate + fr.span.x * pr,
                bx.y * sr + normal_after.y * deviation_rate + fr.span.y * pr,
                bx.z * sr + normal_after.z * deviation_rate + fr.span.z * pr);
    fr.tip_twist = side * 0.0f;
    fr.tip_rate = side * 0.0f;
}

// ---------------------------------------------------------------------------
// prepareBirdGeometry (BF.metal:686-814) + updateWingInertialReaction
// (BF.metal:6493-6572) + the geometry box origin.  One thread.
// ---------------------------------------------------------------------------
__device__ void wing_momentum(V3 root, V3 chord, V3 span, V3 normal, V3 rel, const float* mc, const float* inertia,
                              V3 body_pos, V3& lin, V3& ang) {
    V3 co = v3(chord.x * mc[1] + span.x * mc[2] + normal.x * mc[3], chord.y * mc[1] + span.y * mc[2] + normal.y * mc[3],
               chord.z * mc[1] + span.z * mc[2] + normal.z * mc[3]);
    V3 cv = cross(rel, co);
    lin = v3(mc[0] * cv.x, mc[0] * cv.y, mc[0] * cv.z);
    float a = inertia[0] * dot(rel, chord), b = inertia[1] * dot(rel, span), c = inertia[2] * dot(rel, normal);
    V3 spin = v3(chord.x * a + span.x * b + normal.x * c, chord.y * a + span.y * b + normal.y * c,
                 chord.z * a + span.z * b + normal.z * c);
    V3 arm = v3(root.x + co.x - body_pos.x, root.y + co.y - body_pos.y, root.z + co.z - body_pos.z);
    V3 cr = cross(arm, lin);
    ang = cr + spin;
}

__global__ void k_prepare(const GeomArgs a, int init, float dt, float box_radius) {
    // One warp stages what the single-thread update reads (bird parameters,
    // joints, step, body state, previous wing momentum) into shared memory
    // with parallel loads.  The update then reads no global memory: its
    // stores into the device state may alias global loads, which would
    // otherwise wait one load latency after another.
    __shared__ bfx_bird sbird;
    __shared__ bfx_joint sjoint[2];
    __shared__ double sbody[13];
    __shared__ float sprev[16];
    __shared__ uint64_t sstep;
    DeviceState* st = a.b.state;
    {
        const int t = threadIdx.x;
        const uint32_t* bsrc = (const uint32_t*)a.b.bird;
        for (int i = t; i < (int)(sizeof(bfx_bird) / 4); i += blockDim.x) ((uint32_t*)&sbird)[i] = bsrc[i];
        const int nj = a.b.joint_count < 2 ? a.b.joint_count : 2;
        const uint32_t* jsrc = (const uint32_t*)a.b.joints;
        for (int i = t; i < nj * (int)(sizeof(bfx_joint) / 4); i += blockDim.x) ((uint32_t*)sjoint)[i] = jsrc[i];
        if (t < 13) sbody[t] = st->body[t];
        if (t < 16) sprev[t] = st->wing_prev[t];
        if (t == 0) sstep = st->step;
        __syncthreads();
    }
    const bfx_bird& bird = sbird;
    uint64_t absolute = init ? 0 : sstep + 1;
    float time = (float)((double)absolute * (double)dt);
    float af = 2.0f * 3.14159265358979323846f * bird.wing_kinematics0.v[0];
    float phase = af * time;
    // The step's sines and cosines (portable FP64 series, bit-identical to the
    // host) are independent of one another: the lanes evaluate them in two
    // passes, the phase angles and then the rotation angles built from them.
    //   pass 1: phase, phase + pitch phase, 2 phase, phase + joint phase (2)
    //   pass 2: +/- stroke, deviation, +/- pitch, +/- each joint angle
    const int njoints = a.b.joint_count < 2 ? a.b.joint_count : 2;
    __shared__ SinCos sc1[5], sc2[9];
    {
        const int t = threadIdx.x;
        if (t < 10) {
            const int k = t >> 1;
            const float ang = k == 0 ? phase
                              : k == 1 ? phase + bird.wing_kinematics1.v[1]
                              : k == 2 ? 2.0f * phase
                              : phase + (k - 3 < njoints ? sjoint[k - 3].phase : 0.0f);
            if (t & 1) sc1[k].c = bfx_cosf(ang);
            else sc1[k].s = bfx_sinf(ang);
        }
        __syncthreads();
        if (t < 18) {
            const int k = t >> 1;
            const float stroke = bird.wing_kinematics0.v[2] + bird.wing_kinematics0.v[1] * sc1[0].s;
            const float pitch = bird.wing_kinematics0.v[3] + bird.wing_kinematics1.v[0] * sc1[1].s;
            float ang;
            if (k < 2) ang = (k == 0 ? 1.0f : -1.0f) * stroke;
            else if (k == 2) ang = bird.wing_kinematics1.v[2] * sc1[2].s;
            else if (k < 5) ang = (k == 3 ? 1.0f : -1.0f) * pitch;
            else {
                const int j = (k - 5) >> 1;
                const float sgn = ((k - 5) & 1) ? -1.0f : 1.0f;
                ang = j < njoints ? sgn * (sjoint[j].bias + sjoint[j].amplitude * sc1[3 + j].s) : 0.0f;
            }
            if (t & 1) sc2[k].c = bfx_cosf(ang);
            else sc2[k].s = bfx_sinf(ang);
        }
        __syncthreads();
        if (t != 0) return;
    }
    V3 pos = v3((float)sbody[0], (float)sbody[1], (float)sbody[2]);
    float4 orient = make_float4((float)sbody[3], (float)sbody[4], (float)sbody[5], (float)sbody[6]);
    V3 vel = v3((float)sbody[7], (float)sbody[8], (float)sbody[9]);
    V3 omb = v3((float)sbody[10], (float)sbody[11], (float)sbody[12]);
    float stroke_rate = af * bird.wing_kinematics0.v[1] * sc1[0].c;
    float pitch_rate = af * bird.wing_kinematics1.v[0] * sc1[1].c;
    // stroke-plane deviation at twice the flapping frequency (figure-of-eight
    // tip path); the reference feeds deviation only from measured keyframes
    float deviation_rate = 2.0f * af * bird.wing_kinematics1.v[2] * sc1[2].c;
    WingFrame l, r;
    make_wing_frame(1.0f, sc2[0], stroke_rate, sc2[2], deviation_rate, sc2[3], pitch_rate, bird, pos, orient, l);
    make_wing_frame(-1.0f, sc2[1], stroke_rate, sc2[2], deviation_rate, sc2[4], pitch_rate, bird, pos, orient, r);
    // articulated segments: each joint rotates its parent's frame about the
    // hinge axis and moves it to the joint (angles mirrored on the right wing)
    for (int side = 0; side < 2 && njoints > 0; ++side) {
        const WingFrame& wf = side == 0 ? l : r;
        const float sgn = side == 0 ? 1.0f : -1.0f;
        V3 po = wf.root, pc = wf.chord, ps = wf.span, pn = wf.normal, pw = wf.rel, pu = v3(0.0f, 0.0f, 0.0f);
        for (int j = 0; j < njoints; ++j) {
            const bfx_joint& jt = sjoint[j];
            const V3 o = v3(po.x + pc.x * jt.origin[0] + ps.x * jt.origin[1] + pn.x * jt.origin[2],
                            po.y + pc.y * jt.origin[0] + ps.y * jt.origin[1] + pn.y * jt.origin[2],
                            po.z + pc.z * jt.origin[0] + ps.z * jt.origin[1] + pn.z * jt.origin[2]);
            // the right frame's normal is the mirror image of the left's negated: its
            // hinge takes the axis with the normal component negated (and the angle
            // negated) so the two wings stay mirror images
            const float a2 = sgn * jt.axis[2];
            const V3 ax = v3(pc.x * jt.axis[0] + ps.x * jt.axis[1] + pn.x * a2,
                             pc.y * jt.axis[0] + ps.y * jt.axis[1] + pn.y * a2,
                             pc.z * jt.axis[0] + ps.z * jt.axis[1] + pn.z * a2);
            const SinCos rot = sc2[5 + 2 * j + side];
            const float rate = sgn * (af * jt.amplitude * sc1[3 + j].c);
            const V3 cc = rotate_axis_sc(pc, ax, rot.s, rot.c), cs = rotate_axis_sc(ps, ax, rot.s, rot.c),
                     cn = rotate_axis_sc(pn, ax, rot.s, rot.c);
            const V3 om = v3(pw.x + ax.x * rate, pw.y + ax.y * rate, pw.z + ax.z * rate);
            const V3 uu = pu + cross(pw, o - po);
            SegmentFrame& f = st->seg[2 * j + side];
            f.origin = f4(o, 0.0f);
            f.chord = f4(cc, 0.0f);
            f.span = f4(cs, 0.0f);
            f.normal = f4(cn, 0.0f);
            f.omega = f4(om, 0.0f);
            f.uvel = f4(uu, 0.0f);
            po = o;
            pc = cc;
            ps = cs;
            pn = cn;
            pw = om;
            pu = uu;
        }
    }
    st->geom_time = time;
    float4 o = qnormalize(orient);
    Prepared& p = st->prep;
    p.body_position = f4(pos, 0.0f);
    p.orientation = o;
    p.linear_velocity = f4(vel, 0.0f);
    const float* br = bird.body_radii_mass.v;
    const float* tg = bird.tail_geometry.v;
    const float* wg0 = bird.wing_geometry0.v;
    const float* wg1 = bird.wing_geometry1.v;
    float body_radius = length(v3(br[0], br[1], br[2]));
    float tail_radius = length(v3(br[0] + tg[0], fmaxf(br[1], tg[1]), br[2] + 0.5f * tg[2]));
    float root_radius = length(v3(wg1[1], wg1[2], wg1[3]));
    float wing_radius = root_radius + wg0[0] + fabsf(wg1[0]) + 0.5f * fmaxf(wg0[1], wg0[2]) + 0.5f * wg0[3];
    float geometry_radius = fmaxf(body_radius, fmaxf(tail_radius, wing_radius)) + 2.0f * a.fp.dx;
    p.omega_body_world = f4(qrotate(o, omb), geometry_radius);
    p.left_root = f4(l.root, 0.0f);
    p.left_chord = f4(l.chord, l.tip_twist);
    p.left_span = f4(l.span, 0.0f);
    p.left_normal = f4(l.normal, 0.0f);
    p.left_angular_velocity = f4(l.rel, l.tip_rate);
    p.right_root = f4(r.root, 0.0f);
    p.right_chord = f4(r.chord, r.tip_twist);
    p.right_span = f4(r.span, 0.0f);
    p.right_normal = f4(r.normal, 0.0f);
    p.right_angular_velocity = f4(r.rel, r.tip_rate);

    // wing inertial reaction
    if (bird.left_wing_inertia.v[3] < 0.5f || bird.right_wing_inertia.v[3] < 0.5f) {
        for (int k = 0; k < 16; ++k) {
            st->wing_prev[k] = 0.0f;
            st->wing_reaction[k] = 0.0f;
        }
    } else {
        V3 cur[4];
        wing_momentum(l.root, l.chord, l.span, l.normal, l.rel, bird.left_wing_mass_com.v, bird.left_wing_inertia.v,
                      pos, cur[0], cur[1]);
        wing_momentum(r.root, r.chord, r.span, r.normal, r.rel, bird.right_wing_mass_com.v, bird.right_wing_inertia.v,
                      pos, cur[2], cur[3]);
        float inv = 1.0f / dt;
        for (int j = 0; j < 4; ++j) {
            if (init) {
                st->wing_reaction[4 * j] = st->wing_reaction[4 * j + 1] = st->wing_reaction[4 * j + 2] = 0.0f;
            } else {
                st->wing_reaction[4 * j] = -(cur[j].x - sprev[4 * j]) * inv;
                st->wing_reaction[4 * j + 1] = -(cur[j].y - sprev[4 * j + 1]) * inv;
                st->wing_reaction[4 * j + 2] = -(cur[j].z - sprev[4 * j + 2]) * inv;
            }
            st->wing_reaction[4 * j + 3] = 0.0f;
            st->wing_prev[4 * j] = cur[j].x;
            st->wing_prev[4 * j + 1] = cur[j].y;
            st->wing_prev[4 * j + 2] = cur[j].z;
            st->wing_prev[4 * j + 3] = 0.0f;
        }
    }

    // geometry box: centred on the body origin, clamped into the lattice
    int ext[3] = {a.bx, a.by, a.bz};
    int dims[3] = {a.g.nx, a.g.ny, a.g.nz};
    float c[3] = {pos.x, pos.y, pos.z};
    for (int k = 0; k < 3; ++k) {
        float cc = (c[k] - a.fp.origin[k]) / a.fp.dx - 0.5f;
        int lo = (int)floorf(cc) - ext[k] / 2;
        lo = lo < 0 ? 0 : lo;
        lo = lo > dims[k] - ext[k] ? dims[k] - ext[k] : lo;
        st->box_origin[k] = lo < 0 ? 0 : lo;
        // active bounds: open for the analytic shapes; for a mesh, empty until
        // k_mesh_prepare places the vertices
        const bool mesh = a.b.mesh_local != nullptr;
        st->act_lo[k] = mesh ? (1 << 30) : -(1 << 30);
        st->act_hi[k] = mesh ? -(1 << 30) : (1 << 30);
    }
    (void)box_radius;
}

// ---------------------------------------------------------------------------
// Signed distances: sdEllipsoid / sdTaperedWing / sdTail (BF.metal:486-533).
// ---------------------------------------------------------------------------
__device__ __forceinline__ float sd_ellipsoid(V3 p, V3 r) {
    V3 a = v3(p.x / r.x, p.y / r.y, p.z / r.z);
    V3 r2 = v3(r.x * r.x, r.y * r.y, r.z * r.z);
    V3 b = v3(p.x / r2.x, p.y / r2.y, p.z / r2.z);
    float k0 = length(a);
    float k1 = length(b);
    return k1 > 1.0e-12f ? k0 * (k0 - 1.0f) / k1 : -fminf(r.x, fminf(r.y, r.z));
}
__device__ __forceinline__ float sd_box_tail(float qx, float qy, float qz) {
    return length(v3(fmaxf(qx, 0.0f), fmaxf(qy, 0.0f), fmaxf(qz, 0.0f))) + fminf(fmaxf(qx, fmaxf(qy, qz)), 0.0f);
}
__device__ __forceinline__ float sd_tapered_wing(V3 l, float span, float root_chord, float tip_chord, float thickness,
                                                 float sweep) {
    float sf = clampf(l.y / fmaxf(span, 1.0e-6f), 0.0f, 1.0f);
    float chord = mixf(root_chord, tip_chord, sf);
    float cc = -sweep * sf;
    float dx = fabsf(l.x - cc) - 0.5f * chord;
    float dy = fmaxf(-l.y, l.y - span);
    float dz = fabsf(l.z) - 0.5f * thickness;
    return sd_box_tail(dx, dy, dz);
}
__device__ __forceinline__ float sd_tail(V3 bl, V3 br, const float* tg) {
    float len = tg[0], hw = tg[1], th = tg[2];
    float xr = -(bl.x + br.x);
    float fr = clampf(xr / fmaxf(len, 1.0e-6f), 0.0f, 1.0f);
    float lhw = mixf(0.35f * hw, hw, fr);
    float dx = fmaxf(-xr, xr - len);
    float dy = fabsf(bl.y) - lhw;
    float dz = fabsf(bl.z + 0.15f * br.z) - 0.5f * th;
    return sd_box_tail(dx, dy, dz);
}

// buildBirdGeometry: BF.metal:816-938
__global__ void k_classify_bird(const GeomArgs a, int has_prev) {
    int x, y, z;
    int64_t bidx;
    if (!box_cell(a, x, y, z, bidx)) return;
    const Prepared& p = a.b.state->prep;
    const bfx_bird& bird = *a.b.bird;
    const int64_t gid = flat(a.g, x, y, z);
    V3 world = cell_world(a.fp, x, y, z);
    V3 rb = world - v3(p.body_position);
    uint8_t prev_part = a.b.mask_prev[gid] & kPartMask;
    bool was_solid = has_prev && prev_part != 0;
    float gr = p.omega_body_world.w;
    if (!was_solid && dot(rb, rb) > gr * gr) {
        a.b.mask_next[gid] = topo_flags(0, prev_part, has_prev);
        a.b.wall[gid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    V3 bl = qunrotate(p.orientation, rb);
    V3 base = v3(p.linear_velocity) + cross(v3(p.omega_body_world), rb);
    float best = sd_ellipsoid(bl, v3(bird.body_radii_mass.v[0], bird.body_radii_mass.v[1], bird.body_radii_mass.v[2]));
    V3 bestv = base;
    uint8_t part = 1;
    for (int wing = 0; wing < 2; ++wing) {
        const float4* fr = wing == 0 ? &p.left_root : &p.right_root;
        V3 root = v3(fr[0]), chord = v3(fr[1]), span = v3(fr[2]), normal = v3(fr[3]), rel = v3(fr[4]);
        float tip_twist = fr[1].w, tip_rate = fr[4].w;
        V3 rp = world - root;
        V3 lu = v3(dot(rp, chord), dot(rp, span), dot(rp, normal));
        float sf = clampf(lu.y / fmaxf(bird.wing_geometry0.v[0], 1.0e-6f), 0.0f, 1.0f);
        float twist = tip_twist * sf;
        float tc = bfx_cosf(twist), ts = bfx_sinf(twist);
        V3 loc = v3(tc * lu.x + ts * lu.z, lu.y, -ts * lu.x + tc * lu.z);
        float d = sd_tapered_wing(loc, bird.wing_geometry0.v[0], bird.wing_geometry0.v[1], bird.wing_geometry0.v[2],
                                  bird.wing_geometry0.v[3], bird.wing_geometry1.v[0]);
        if (d < best) {
            best = d;
            V3 c1 = cross(rel, rp);
            float k = sf * tip_rate;
            V3 sw = v3(span.x * k, span.y * k, span.z * k);
            V3 arm = v3(world.x - (root.x + span.x * lu.y), world.y - (root.y + span.y * lu.y),
                        world.z - (root.z + span.z * lu.y));
            V3 c2 = cross(sw, arm);
            bestv = v3(base.x + c1.x + c2.x, base.y + c1.y + c2.y, base.z + c1.z + c2.z);
            part = wing == 0 ? 2 : 3;
        }
    }
    float td = sd_tail(bl, v3(bird.body_radii_mass.v[0], bird.body_radii_mass.v[1], bird.body_radii_mass.v[2]),
                       bird.tail_geometry.v);
    if (td < best) {
        best = td;
        bestv = base;
        part = 4;
    }
    uint8_t solid_part = best <= 0.0f ? part : (uint8_t)0;
    a.b.mask_next[gid] = topo_flags(solid_part, prev_part, has_prev);
    a.b.wall[gid] = make_float4(bestv.x * a.fp.v2l, bestv.y * a.fp.v2l, bestv.z * a.fp.v2l, 0.0f);
}

// Body ellipsoid alone (part 1); w holds the implicit value.
__device__ __forceinline__ float ellipsoid_implicit(const Prepared& p, const bfx_bird& bird, V3 w) {
    V3 rb = w - v3(p.body_position);
    V3 bl = qunrotate(p.orientation, rb);
    return sd_ellipsoid(bl, v3(bird.body_radii_mass.v[0], bird.body_radii_mass.v[1], bird.body_radii_mass.v[2]));
}

__global__ void k_classify_ellipsoid(const GeomArgs a, int has_prev) {
    int x, y, z;
    int64_t bidx;
    if (!box_cell(a, x, y, z, bidx)) return;
    const Prepared& p = a.b.state->prep;
    const bfx_bird& bird = *a.b.bird;
    const int64_t gid = flat(a.g, x, y, z);
    float r = fmaxf(bird.body_radii_mass.v[0], fmaxf(bird.body_radii_mass.v[1], bird.body_radii_mass.v[2])) +
              2.0f * a.fp.dx;
    V3 world = cell_world(a.fp, x, y, z);
    V3 rb = world - v3(p.body_position);
    uint8_t prev_part = a.b.mask_prev[gid] & kPartMask;
    bool was_solid = has_prev && prev_part != 0;
    if (!was_solid && dot(rb, rb) > r * r) {
        a.b.mask_next[gid] = topo_flags(0, prev_part, has_prev);
        a.b.wall[gid] = make_float4(0.0f, 0.0f, 0.0f, r);
        return;
    }
    float imp = ellipsoid_implicit(p, bird, world);
    V3 cr = cross(v3(p.omega_body_world), rb);
    a.b.mask_next[gid] = topo_flags(imp <= 0.0f ? 1 : 0, prev_part, has_prev);
    a.b.wall[gid] = make_float4((p.linear_velocity.x + cr.x) * a.fp.v2l, (p.linear_velocity.y + cr.y) * a.fp.v2l,
                                (p.linear_velocity.z + cr.z) * a.fp.v2l, imp);
}

// ---------------------------------------------------------------------------
// Prescribed flapping wing: the analytic Li-Nabawy beta-planform wing of
// MetalFlappingWingValidation (BF.metal:940-1297).  The runtime packs the
// bfx_flapping_wing record into the device bird record: root_and_chord in
// wing_geometry0, geometry in wing_geometry1, kinematics0 / kinematics1 in
// wing_kinematics0 / wing_kinematics1.  Its lengths are in cells (the
// reference runs it in lattice units); the prepared frame sits in the left
// wing slots of Prepared, the kinematic state (stroke, pitch and their rates
// per step) in right_root.
// ---------------------------------------------------------------------------
struct WingRec {
    const float* root_and_chord;
    const float* geometry;
    const float* k0;
    const float* k1;
};
__device__ __forceinline__ WingRec wing_rec(const bfx_bird& b) {
    return WingRec{b.wing_geometry0.v, b.wing_geometry1.v, b.wing_kinematics0.v, b.wing_kinematics1.v};
}

// prescribedStrokeKinematics: BF.metal:945-1001 (angle, rate per cycle)
__device__ void wing_stroke(float phase, const WingRec& w, float& angle, float& rate) {
    const float pi = 3.14159265358979323846f;
    const float amplitude = w.k0[1], duration = w.k0[2], half = 0.5f * duration, max_rate = w.k1[2];
    if (phase < half) {
        const float arg = pi * (phase + half) / duration;
        angle = amplitude + max_rate * duration / pi * (bfx_sinf(arg) - 1.0f);
        rate = max_rate * bfx_cosf(arg);
    } else if (phase < 0.5f - half) {
        const float at_end = amplitude - max_rate * duration / pi;
        angle = at_end - max_rate * (phase - half);
        rate = -max_rate;
    } else if (phase < 0.5f + half) {
        const float start = 0.5f - half;
        const float at_start = -amplitude + max_rate * duration / pi;
        const float arg = pi * (phase - start) / duration;
        angle = at_start - max_rate * duration / pi * bfx_sinf(arg);
        rate = -max_rate * bfx_cosf(arg);
    } else if (phase < 1.0f - half) {
        const float at_end = -amplitude + max_rate * duration / pi;
        angle = at_end + max_rate * (phase - (0.5f + half));
        rate = max_rate;
    } else {
        const float start = 1.0f - half;
        const float at_start = amplitude - max_rate * duration / pi;
        const float arg = pi * (phase - start) / duration;
        angle = at_start + max_rate * duration / pi * bfx_sinf(arg);
        rate = max_rate * bfx_cosf(arg);
    }
}

// prescribedPitchKinematics: BF.metal:1003-1035
__device__ void wing_pitch(float phase, const WingRec& w, float& angle, float& rate) {
    const float pi = 3.14159265358979323846f;
    const float duration = w.k0[3], half = 0.5f * duration;
    const float low = w.k1[0], high = w.k1[1], delta = high - low;
    float x, start, change;
    if (phase < half || phase >= 1.0f - half) {
        const float wrapped = phase < half ? phase + 1.0f : phase;
        x = (wrapped - (1.0f - half)) / duration;
        start = high;
        change = -delta;
    } else if (phase >= 0.5f - half && phase < 0.5f + half) {
        x = (phase - (0.5f - half)) / duration;
        start = low;
        change = delta;
    } else {
        angle = phase < 0.5f ? low : high;
        rate = 0.0f;
        return;
    }
    const float blend = x - bfx_sinf(2.0f * pi * x) / (2.0f * pi);
    rate = change / duration * (1.0f - bfx_cosf(2.0f * pi * x));
    angle = start + change * blend;
}

// preparePrescribedFlappingWing (BF.metal:1038-1078) and the geometry box,
// one thread.  The phase runs on the absolute step index, as the reference's
// validator passes Float(absoluteStep) as the time.
__global__ void k_prepare_wing(const GeomArgs a, int init, float dt) {
    if (threadIdx.x != 0) return;
    DeviceState* st = a.b.state;
    const WingRec w = wing_rec(*a.b.bird);
    const uint64_t absolute = init ? 0 : st->step + 1;
    const float time = (float)absolute;
    const float cycle_steps = w.k0[0];
    float phase = fmodf(time / cycle_steps, 1.0f);
    phase = phase < 0.0f ? phase + 1.0f : phase;
    float stroke, stroke_rate, pitch, pitch_rate;
    wing_stroke(phase, w, stroke, stroke_rate);
    wing_pitch(phase, w, pitch, pitch_rate);
    const V3 axis = v3(0.0f, 0.0f, 1.0f);
    const V3 span = v3(bfx_cosf(stroke), bfx_sinf(stroke), 0.0f);
    const V3 tangent = cross(axis, span);
    const float ps = bfx_sinf(-pitch), pc = bfx_cosf(-pitch);
    const V3 chord = rotate_axis_sc(tangent, span, ps, pc);
    const V3 normal = normalize3(cross(span, chord));
    const float inv = 1.0f / cycle_steps;
    const V3 omega = v3(axis.x * (stroke_rate * inv) - span.x * (pitch_rate * inv),
                        axis.y * (stroke_rate * inv) - span.y * (pitch_rate * inv),
                        axis.z * (stroke_rate * inv) - span.z * (pitch_rate * inv));
    Prepared& p = st->prep;
    const V3 pos = v3((float)st->body[0], (float)st->body[1], (float)st->body[2]);
    p.body_position = f4(pos, 0.0f);
    p.orientation = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    p.linear_velocity = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const float radius = w.geometry[0] + 1.5f * w.root_and_chord[3] + 2.0f * a.fp.dx;
    p.omega_body_world = make_float4(0.0f, 0.0f, 0.0f, radius);
    p.left_root = make_float4(w.root_and_chord[0], w.root_and_chord[1], w.root_and_chord[2], w.root_and_chord[3]);
    p.left_chord = f4(normalize3(chord), 0.0f);
    p.left_span = f4(normalize3(span), 0.0f);
    p.left_normal = f4(normal, 0.0f);
    p.left_angular_velocity = f4(omega, 0.0f);
    p.right_root = make_float4(stroke, pitch, stroke_rate * inv, pitch_rate * inv);
    p.right_chord = p.right_span = p.right_normal = p.right_angular_velocity = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int k = 0; k < 16; ++k) {
        st->wing_prev[k] = 0.0f;
        st->wing_reaction[k] = 0.0f;
    }
    st->geom_time = (float)((double)absolute * (double)dt);
    // geometry box centred on the wing root, clamped into the lattice
    const int ext[3] = {a.bx, a.by, a.bz};
    const int dims[3] = {a.g.nx, a.g.ny, a.g.nz};
    const float c[3] = {w.root_and_chord[0], w.root_and_chord[1], w.root_and_chord[2]};
    for (int k = 0; k < 3; ++k) {
        const float cc = (c[k] - a.fp.origin[k]) / a.fp.dx - 0.5f;
        int lo = (int)floorf(cc) - ext[k] / 2;
        lo = lo < 0 ? 0 : lo;
        lo = lo > dims[k] - ext[k] ? dims[k] - ext[k] : lo;
        st->box_origin[k] = lo < 0 ? 0 : lo;
        st->act_lo[k] = -(1 << 30);
        st->act_hi[k] = 1 << 30;
    }
}

// prescribedWingBoundaryCoordinates + prescribedWingMaximumViolation
// (BF.metal:1091-1142): positive outside the wing.
__device__ float wing_violation(const WingRec& w, const Prepared& p, float dx, V3 world) {
    const V3 rel = world - v3(p.left_root);
    const float radial = dot(rel, v3(p.left_span)), normal = dot(rel, v3(p.left_normal)),
                chord = dot(rel, v3(p.left_chord));
    const float radius = w.geometry[0], chord_mean = w.root_and_chord[3];
    const float half = 0.5f * fmaxf(w.geometry[1], dx);
    const float fraction = clampf(radial / radius, 0.0f, 1.0f);
    const float beta_base = fmaxf(fraction * (1.0f - fraction), 0.0f);
    const float local_chord = chord_mean * w.geometry[3] * bfx_powf(beta_base, w.geometry[2]);
    const float leading = -0.25f * chord_mean;
    const float root_v = -radial, tip_v = radial - radius, normal_v = fabsf(normal) - half;
    const float lead_v = leading - chord, trail_v = chord - (leading + local_chord);
    return fmaxf(fmaxf(root_v, tip_v), fmaxf(normal_v, fmaxf(lead_v, trail_v)));
}

// buildPrescribedFlappingWing, classification (BF.metal:1179-1249): part 1;
// wall = rigid rotation about the root in lattice velocity, w = -1 solid /
// +1 fluid, (0, 0, 0, radius) outside the bounding sphere.
__global__ void k_classify_wing(const GeomArgs a, int has_prev) {
    int x, y, z;
    int64_t bidx;
    if (!box_cell(a, x, y, z, bidx)) return;
    const Prepared& p = a.b.state->prep;
    const WingRec w = wing_rec(*a.b.bird);
    const int64_t gid = flat(a.g, x, y, z);
    const float chord_mean = w.root_and_chord[3];
    const float radius = w.geometry[0] + 1.5f * chord_mean + 2.0f * a.fp.dx;
    const V3 world = cell_world(a.fp, x, y, z);
    const V3 rel = world - v3(p.left_root);
    const uint8_t prev_part = a.b.mask_prev[gid] & kPartMask;
    const bool was_solid = has_prev && prev_part != 0;
    if (!was_solid && dot(rel, rel) > radius * radius) {
        a.b.mask_next[gid] = topo_flags(0, prev_part, has_prev);
        a.b.wall[gid] = make_float4(0.0f, 0.0f, 0.0f, radius);
        return;
    }
    const float cc = dot(rel, v3(p.left_chord)), rc = dot(rel, v3(p.left_span)), nc = dot(rel, v3(p.left_normal));
    const float half = 0.5f * fmaxf(w.geometry[1], a.fp.dx);
    const bool in_radial = rc >= 0.0f && rc <= w.geometry[0];
    const bool in_normal = fabsf(nc) <= half;
    bool is_wing = false;
    if (in_radial && in_normal) {
        const float fraction = clampf(rc / w.geometry[0], 0.0f, 1.0f);
        const float beta_base = fmaxf(fraction * (1.0f - fraction), 0.0f);
        const float local_chord = chord_mean * w.geometry[3] * bfx_powf(beta_base, w.geometry[2]);
        const float leading = -0.25f * chord_mean;
        const float trailing = leading + local_chord;
        is_wing = cc >= leading && cc <= trailing;
    }
    const V3 u = cross(v3(p.left_angular_velocity), rel);
    a.b.mask_next[gid] = topo_flags(is_wing ? 1 : 0, prev_part, has_prev);
    a.b.wall[gid] = make_float4(u.x / a.fp.dx, u.y / a.fp.dx, u.z / a.fp.dx, is_wing ? -1.0f : 1.0f);
}

// prescribedWingLinkFraction (BF.metal:1144-1175) of the link from solid s
// toward s + c_q, the fluid end placed at s's position plus c_q dx as
// buildPrescribedFlappingWing places it (BF.metal:1276-1278).
__device__ float wing_link_fraction(const GeomArgs& a, int q, int sx, int sy, int sz) {
    const Prepared& p = a.b.state->prep;
    const WingRec w = wing_rec(*a.b.bird);
    const V3 sw = cell_world(a.fp, sx, sy, sz);
    const V3 fw = v3(sw.x + (float)cx(q) * a.fp.dx, sw.y + (float)cy(q) * a.fp.dx, sw.z + (float)cz(q) * a.fp.dx);
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 10; ++it) {
        const float mid = 0.5f * (lo + hi);
        const V3 smp = v3(mixf(fw.x, sw.x, mid), mixf(fw.y, sw.y, mid), mixf(fw.z, sw.z, mid));
        if (wing_violation(w, p, a.fp.dx, smp) > 0.0f) lo = mid;
        else hi = mid;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

// driven by the rigid frames instead of keyframes).
__device__ void mesh_vertex(const GeomArgs& a, uint32_t i, V3& w, V3& v);

// Vertex positions and velocities, and the bounding box of the vertices in
// cells (warp min / max, then one atomic per warp and bound: order-free).
__global__ void k_mesh_prepare(const GeomArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < a.b.nverts;
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    if (valid) {
        V3 w, v;
        mesh_vertex(a, i, w, v);
        a.b.mesh_pos[i] = f4(w, 0.0f);
        a.b.mesh_vel[i] = make_float4(v.x * a.fp.v2l, v.y * a.fp.v2l, v.z * a.fp.v2l, 0.0f);
        const float c[3] = {(w.x - a.fp.origin[0]) / a.fp.dx - 0.5f, (w.y - a.fp.origin[1]) / a.fp.dx - 0.5f,
                            (w.z - a.fp.origin[2]) / a.fp.dx - 0.5f};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            // clamp before the conversion (a non-finite position opens the bounds)
            const float ck = c[k] == c[k] ? fminf(fmaxf(c[k], -1.0e9f), 1.0e9f) : 0.0f;
            lo[k] = c[k] == c[k] ? (int)floorf(ck) : -(1 << 30);
            hi[k] = c[k] == c[k] ? (int)ceilf(ck) : (1 << 30);
            lo[k] = lo[k] < -(1 << 30) ? -(1 << 30) : lo[k];
            hi[k] = hi[k] > (1 << 30) ? (1 << 30) : hi[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            const int l = __shfl_down_sync(0xffffffffu, lo[k], o), h = __shfl_down_sync(0xffffffffu, hi[k], o);
            lo[k] = l < lo[k] ? l : lo[k];
            hi[k] = h > hi[k] ? h : hi[k];
        }
    }
    if ((threadIdx.x & 31) == 0 && lo[0] <= hi[0]) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(&a.b.state->act_lo[k], lo[k]);
            atomicMax(&a.b.state->act_hi[k], hi[k]);
        }
    }
}

// Keyframe replay of a body-frame offset (prepareIndexedBirdSurface,
// BF.metal:1585-1622): the interval [first, first + 1] holds the geometry time
// (an exact interior keyframe opens the following interval, times past the
// last keyframe stay on the last one, before the first on the first), the
// offset is mix(a, b, blend) = a + (b - a) blend with the blend clamped to
// [0, 1], and its rate is (b - a) / duration.
__device__ void keyframe_offset(const GeomArgs& a, uint32_t i, V3& l, V3& dl) {
    const float t = a.b.state->geom_time;
    const float* T = a.b.kf_times;
    const int nf = a.b.kf_count;
    int lo = 0, hi = nf;  // first index with T[j] > t
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (T[mid] > t) hi = mid;
        else lo = mid + 1;
    }
    int first = lo - 1;
    first = first < 0 ? 0 : (first > nf - 2 ? nf - 2 : first);
    const float duration = T[first + 1] - T[first];
    float blend = (t - T[first]) / duration;
    blend = blend < 0.0f ? 0.0f : (blend > 1.0f ? 1.0f : blend);
    const float* pa = a.b.kf_points + 3 * ((size_t)first * a.b.nverts + i);
    const float* pb = pa + 3 * (size_t)a.b.nverts;
    const V3 d = v3(pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]);
    l = v3(pa[0] + d.x * blend, pa[1] + d.y * blend, pa[2] + d.z * blend);
    dl = v3(d.x / duration, d.y / duration, d.z / duration);
}

__device__ void mesh_vertex(const GeomArgs& a, uint32_t i, V3& w, V3& v) {
    const Prepared& p = a.b.state->prep;
    if (a.b.kf_count >= 2) {
        // body-frame keyframe offset on top of the body's rigid motion
        V3 l, dl;
        keyframe_offset(a, i, l, dl);
        const V3 r = qrotate(p.orientation, l), rd = qrotate(p.orientation, dl);
        w = v3(p.body_position.x + r.x, p.body_position.y + r.y, p.body_position.z + r.z);
        const V3 cr = cross(v3(p.omega_body_world), r);
        v = v3(p.linear_velocity.x + cr.x + rd.x, p.linear_velocity.y + cr.y + rd.y,
               p.linear_velocity.z + cr.z + rd.z);
        return;
    }
    V3 l = v3(a.b.mesh_local[3 * i], a.b.mesh_local[3 * i + 1], a.b.mesh_local[3 * i + 2]);
    uint8_t seg = a.b.mesh_segment[i];
    if (seg == 0) {
        V3 r = qrotate(p.orientation, l);
        w = v3(p.body_position.x + r.x, p.body_position.y + r.y, p.body_position.z + r.z);
        V3 cr = cross(v3(p.omega_body_world), r);
        v = v3(p.linear_velocity.x + cr.x, p.linear_velocity.y + cr.y, p.linear_velocity.z + cr.z);
    } else if (seg >= 3) {
        // articulated segment: rigid motion of its own frame on top of the chain
        const SegmentFrame& f = a.b.state->seg[seg - 3];
        w = v3(f.origin.x + f.chord.x * l.x + f.span.x * l.y + f.normal.x * l.z,
               f.origin.y + f.chord.y * l.x + f.span.y * l.y + f.normal.y * l.z,
               f.origin.z + f.chord.z * l.x + f.span.z * l.y + f.normal.z * l.z);
        V3 rb = v3(w.x - p.body_position.x, w.y - p.body_position.y, w.z - p.body_position.z);
        V3 cr = cross(v3(p.omega_body_world), rb);
        V3 rr = v3(w.x - f.origin.x, w.y - f.origin.y, w.z - f.origin.z);
        V3 cw = cross(v3(f.omega), rr);
        v = v3(p.linear_velocity.x + cr.x + cw.x + f.uvel.x, p.linear_velocity.y + cr.y + cw.y + f.uvel.y,
               p.linear_velocity.z + cr.z + cw.z + f.uvel.z);
    } else {
        const float4* fr = seg == 1 ? &p.left_root : &p.right_root;
        w = v3(fr[0].x + fr[1].x * l.x + fr[2].x * l.y + fr[3].x * l.z,
               fr[0].y + fr[1].y * l.x + fr[2].y * l.y + fr[3].y * l.z,
               fr[0].z + fr[1].z * l.x + fr[2].z * l.y + fr[3].z * l.z);
        V3 rb = v3(w.x - p.body_position.x, w.y - p.body_position.y, w.z - p.body_position.z);
        V3 cr = cross(v3(p.omega_body_world), rb);
        V3 rr = v3(w.x - fr[0].x, w.y - fr[0].y, w.z - fr[0].z);
        V3 cw = cross(v3(fr[4]), rr);
        v = v3(p.linear_velocity.x + cr.x + cw.x, p.linear_velocity.y + cr.y + cw.y,
               p.linear_velocity.z + cr.z + cw.z);
    }
}

// Clears the keys of the active cells (only those are read this step); slab launch.
__global__ void k_mesh_clear(const GeomArgs a) {
    if (slab_inactive(a)) return;
    int lo[3], hi[3];
    active_bounds(a, lo, hi);
#pragma unroll
    for (int k = 0; k < kSlabZ; ++k) {
        int x, y, z;
        int64_t bidx;
        if (slab_cell(a, k, x, y, z, bidx) && in_bounds(lo, hi, x, y, z)) a.b.keys[bidx] = 0xFFFFFFFFFFFFFFFFull;
    }
}

// One warp per triangle: the lanes share the triangle's voxel box (its AABB
// grown by the half thickness plus two cells, clamped to the lattice and the
// geometry box) and each keeps the atomic minimum of (quantised distance,
// triangle id) per voxel.  LEAN caps a thread at 40 registers (a few bytes
// spill): the pipelined build runs the raster beside the persistent TRT fluid
// kernel, whose CTA leaves about 22 K registers of an SM free, room for four
// lean blocks against two of the unconstrained (64-register) kernel.
template <int LEAN>
__global__ void __launch_bounds__(128, LEAN ? 12 : 1) k_mesh_raster(const GeomArgs a) {
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= a.b.ntris) return;
    V3 A, B, C;
    tri_vertices(a, t, A, B, C);
    const float cs = a.fp.dx;
    const float guard = a.b.half_thickness + 2.0f * cs;
    int lo[3], hi[3];
    const int dims[3] = {a.g.nx, a.g.ny, a.g.nz};
    const int ext[3] = {a.bx, a.by, a.bz};
    const int32_t* o = a.b.state->box_origin;
    float mn[3] = {fminf(A.x, fminf(B.x, C.x)), fminf(A.y, fminf(B.y, C.y)), fminf(A.z, fminf(B.z, C.z))};
    float mx[3] = {fmaxf(A.x, fmaxf(B.x, C.x)), fmaxf(A.y, fmaxf(B.y, C.y)), fmaxf(A.z, fmaxf(B.z, C.z))};
    for (int k = 0; k < 3; ++k) {
        lo[k] = (int)floorf(((mn[k] - guard) - a.fp.origin[k]) / cs - 0.5f);
        hi[k] = (int)ceilf(((mx[k] + guard) - a.fp.origin[k]) / cs - 0.5f);
        lo[k] = lo[k] < 0 ? 0 : (lo[k] > dims[k] - 1 ? dims[k] - 1 : lo[k]);
        hi[k] = hi[k] < 0 ? 0 : (hi[k] > dims[k] - 1 ? dims[k] - 1 : hi[k]);
        // confine to the geometry box (the key array is box-local)
        lo[k] = lo[k] < o[k] ? o[k] : lo[k];
        hi[k] = hi[k] > o[k] + ext[k] - 1 ? o[k] + ext[k] - 1 : hi[k];
    }
    const int ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
    if (ex <= 0 || ey <= 0 || ez <= 0) return;
    const int total = ex * ey * ez;
    // Voxels farther than the guard from the triangle decide nothing (a cell
    // next to a solid one lies within h + sqrt(3) dx of its triangle, inside
    // the guard), so only voxels within the guard of the triangle's bounding
    // sphere compute their distance: a superset, with a relative slack that
    // covers the rounding of the squared distances.
    const V3 cen = v3((A.x + B.x + C.x) * (1.0f / 3.0f), (A.y + B.y + C.y) * (1.0f / 3.0f),
                      (A.z + B.z + C.z) * (1.0f / 3.0f));
    const float r2 = fmaxf(dot(A - cen, A - cen), fmaxf(dot(B - cen, B - cen), dot(C - cen, C - cen)));
    const float reach = sqrtf(r2) + guard;
    const float reach2 = reach * reach * 1.0001f;
    // voxel index -> (x, y, z) by reciprocal multiplication (exact for these small extents)
    const float inv_ex = 1.0f / (float)ex, inv_ey = 1.0f / (float)ey;
    auto voxel = [&](int i, int& x, int& y, int& z) {
        const int r = (int)(((float)i + 0.5f) * inv_ex);
        const int zi = (int)(((float)r + 0.5f) * inv_ey);
        x = lo[0] + (i - r * ex);
        y = lo[1] + (r - zi * ey);
        z = lo[2] + zi;
    };
    auto key_voxel = [&](int i) {
        int x, y, z;
        voxel(i, x, y, z);
        V3 w = cell_world(a.fp, x, y, z), bary;
        V3 cp = closest_point(w, A, B, C, bary);
        float dc = length(w - cp) / cs;
        float bin = roundf(dc * 65536.0f);
        unsigned long long ub = bin >= 4294967295.0f ? 0xFFFFFFFFull : (unsigned long long)bin;
        unsigned long long key = (ub << 32) | (unsigned long long)t;
        int64_t bi = (int64_t)(x - o[0]) + (int64_t)a.bx * ((int64_t)(y - o[1]) + (int64_t)a.by * (z - o[2]));
        atomicMin(&a.b.keys[bi], key);
    };
    // The sphere test rejects a good share of the box: queue the voxels that
    // pass (warp ballot into a per-warp list) and run the closest-point search
    // 32 at a time, so that its lanes are all busy.  Keys are minima, so the
    // order of the atomics does not matter.
    __shared__ int queue[4][64];
    int* qw = queue[(threadIdx.x >> 5) & 3];
    const unsigned below = (1u << lane) - 1u;
    int qn = 0;  // warp-uniform queue length (< 32 between rounds)
    for (int base = 0; base < total; base += 32) {
        const int i = base + lane;
        bool pass = false;
        if (i < total) {
            int x, y, z;
            voxel(i, x, y, z);
            const V3 dcen = cell_world(a.fp, x, y, z) - cen;
            pass = dot(dcen, dcen) <= reach2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, pass);
        if (pass) qw[qn + __popc(m & below)] = i;
        qn += __popc(m);
        __syncwarp();
        if (qn >= 32) {
            const int mine = qw[lane];
            __syncwarp();
            if (lane < qn - 32) qw[lane] = qw[lane + 32];
            __syncwarp();
            qn -= 32;
            key_voxel(mine);
        }
    }
    if (lane < qn) key_voxel(qw[lane]);
}

__device__ bool resolve_cell(const GeomArgs& a, int has_prev, int x, int y, int z, int64_t bidx);

// Mask byte and wall value of every active cell (cells outside the active
// bounds keep mask 0; their wall value is never read); slab launch.  With a
// live list, every slab also appends each of its kSlabZ slices (one block of
// the link count's box launch) in which a cell holds a key or a changed
// occupancy: only such blocks can hold a cut link (its fluid cell is keyed)
// or a topology event, so the link count and emission visit those alone.  The
// list's order is not fixed, and nothing depends on it: the counts are stored
// by block index and the emission writes at offsets scanned in block order.
__global__ void k_mesh_resolve(const GeomArgs a, int has_prev) {
    const bool inactive = slab_inactive(a);
    int lo[3], hi[3];
    active_bounds(a, lo, hi);
#pragma unroll
    for (int k = 0; k < kSlabZ; ++k) {
        int x, y, z;
        int64_t bidx;
        bool live = false;
        if (!inactive && slab_cell(a, k, x, y, z, bidx) && in_bounds(lo, hi, x, y, z))
            live = resolve_cell(a, has_prev, x, y, z, bidx);
        if (a.b.live_list) {
            const int any = __syncthreads_or(live);
            const int lz = (int)blockIdx.z * kSlabZ + k;
            if (any && linear_tid() == 0 && lz < a.bz)
                a.b.live_list[atomicAdd(a.b.live_count, 1u)] = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * lz);
        }
    }
}

// Resolves one cell; true when it holds a key or its occupancy changed.
__device__ bool resolve_cell(const GeomArgs& a, int has_prev, int x, int y, int z, int64_t bidx) {
    const int64_t gid = flat(a.g, x, y, z);
    uint8_t prev_part = a.b.mask_prev[gid] & kPartMask;
    unsigned long long key = a.b.keys[bidx];
    uint32_t t = (uint32_t)(key & 0xFFFFFFFFull);
    if (key == 0xFFFFFFFFFFFFFFFFull || t >= a.b.ntris) {
        const uint8_t m = topo_flags(0, prev_part, has_prev);
        a.b.mask_next[gid] = m;
        a.b.wall[gid] = make_float4(0.0f, 0.0f, 0.0f, 16.0f);
        return m != 0;
    }
    V3 w = cell_world(a.fp, x, y, z);
    V3 A, B, C, bary;
    tri_vertices(a, t, A, B, C);
    V3 cp = closest_point(w, A, B, C, bary);
    float4 va = a.b.mesh_vel[a.b.mesh_tris[3 * t]], vb = a.b.mesh_vel[a.b.mesh_tris[3 * t + 1]],
           vc = a.b.mesh_vel[a.b.mesh_tris[3 * t + 2]];
    V3 v = v3(bary.x * va.x + bary.y * vb.x + bary.z * vc.x, bary.x * va.y + bary.y * vb.y + bary.z * vc.y,
              bary.x * va.z + bary.y * vb.z + bary.z * vc.z);
    float sd = length(w - cp) - a.b.half_thickness;
    uint8_t part = sd <= 0.0f ? a.b.mesh_tri_part[t] : (uint8_t)0;
    a.b.mask_next[gid] = topo_flags(part, prev_part, has_prev);
    a.b.wall[gid] = make_float4(v.x, v.y, v.z, sd / a.fp.dx);
    return true;
}

__global__ void k_fill_wall_w(float4* wall, int64_t n, float w) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wall[i] = make_float4(0.0f, 0.0f, 0.0f, w);
}

// ellipsoid implicit (the prescribedWingLinkFraction rule, BF.metal:1144-1175).
__device__ float ellipsoid_link_fraction(const GeomArgs& a, int fx, int fy, int fz, int sx, int sy, int sz) {
    const Prepared& p = a.b.state->prep;
    const bfx_bird& bird = *a.b.bird;
    V3 fw = cell_world(a.fp, fx, fy, fz), sw = cell_world(a.fp, sx, sy, sz);
    float lo = 0.0f, hi = 1.0f;
    for (int it = 0; it < 10; ++it) {
        float mid = 0.5f * (lo + hi);
        V3 s = v3(mixf(fw.x, sw.x, mid), mixf(fw.y, sw.y, mid), mixf(fw.z, sw.z, mid));
        if (ellipsoid_implicit(p, bird, s) > 0.0f) lo = mid;
        else hi = mid;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

// min(d_A, d_B) - h, A and B the winning triangles of the two end cells.
__device__ float mesh_ray_root(const GeomArgs& a, int fx, int fy, int fz, int sx, int sy, int sz) {
    V3 fw = cell_world(a.fp, fx, fy, fz), sw = cell_world(a.fp, sx, sy, sz);
    unsigned long long kf = box_key(a, fx, fy, fz), ks = box_key(a, sx, sy, sz);
    uint32_t ta = (uint32_t)(ks & 0xFFFFFFFFull);
    uint32_t tb = kf == 0xFFFFFFFFFFFFFFFFull ? ta : (uint32_t)(kf & 0xFFFFFFFFull);
    if (ta >= a.b.ntris) return 0.5f;
    if (tb >= a.b.ntris) tb = ta;
    const float h = a.b.half_thickness;
    float lo = 0.0f, hi = 1.0f;
    bool found = false;
    for (int i = 1; i <= 8; ++i) {
        float t = (float)i * 0.125f;
        V3 s = v3(mixf(fw.x, sw.x, t), mixf(fw.y, sw.y, t), mixf(fw.z, sw.z, t));
        float gv = fminf(tri_distance(a, ta, s), tri_distance(a, tb, s)) - h;
        if (gv <= 0.0f) {
            hi = t;
            found = true;
            break;
        }
        lo = t;
    }
    if (!found) return 1.0f;
    for (int it = 0; it < 24; ++it) {
        float mid = 0.5f * (lo + hi);
        V3 s = v3(mixf(fw.x, sw.x, mid), mixf(fw.y, sw.y, mid), mixf(fw.z, sw.z, mid));
        float gv = fminf(tri_distance(a, ta, s), tri_distance(a, tb, s)) - h;
        if (gv <= 0.0f) hi = mid;
        else lo = mid;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

// mesh_ray_root on the 16 lanes of a group (gl: lane in the group, gmask: the
// group's lanes in the warp).  The 8 march points, and in each of 8 rounds the
// 7 midpoints of three bisection levels, are evaluated at once on separate
// lanes -- two lanes per point, one per candidate triangle -- and the
// decisions are then taken in the one-thread order.  Every evaluated point and
// the returned fraction equal mesh_ray_root's; the search's dependent chain
// shrinks from up to 32 distance evaluations to 9.
__device__ float mesh_ray_root_group(const GeomArgs& a, int fx, int fy, int fz, int sx, int sy, int sz, int gl,
                                     unsigned gmask, int gshift) {
    V3 fw = cell_world(a.fp, fx, fy, fz), sw = cell_world(a.fp, sx, sy, sz);
    unsigned long long kf = box_key(a, fx, fy, fz), ks = box_key(a, sx, sy, sz);
    uint32_t ta = (uint32_t)(ks & 0xFFFFFFFFull);
    uint32_t tb = kf == 0xFFFFFFFFFFFFFFFFull ? ta : (uint32_t)(kf & 0xFFFFFFFFull);
    if (ta >= a.b.ntris) return 0.5f;
    if (tb >= a.b.ntris) tb = ta;
    const float h = a.b.half_thickness;
    const uint32_t tri = (gl & 1) ? tb : ta;
    // inside (gv <= 0) at the point of parameter t, for the pair of lanes of one point
    auto inside = [&](float t) {
        V3 s = v3(mixf(fw.x, sw.x, t), mixf(fw.y, sw.y, t), mixf(fw.z, sw.z, t));
        const float d = tri_distance(a, tri, s);
        const float gv = fminf(d, __shfl_xor_sync(gmask, d, 1)) - h;
        return (__ballot_sync(gmask, gv <= 0.0f) >> gshift) & 0x5555u;  // one bit per point: bit 2 * point
    };
    // march: point p at t = (p + 1) / 8
    const unsigned march = inside((float)((gl >> 1) + 1) * 0.125f);
    if (march == 0) return 1.0f;
    const int p = (__ffs(march) - 1) >> 1;
    float lo = (float)p * 0.125f, hi = (float)(p + 1) * 0.125f;
    for (int round = 0; round < 8; ++round) {
        // the three-level bisection tree of (lo, hi): node 0; nodes 1, 2; nodes 3..6
        const float m0 = 0.5f * (lo + hi);
        const float m1 = 0.5f * (lo + m0), m2 = 0.5f * (m0 + hi);
        const int node = (gl >> 1) < 7 ? (gl >> 1) : 0;
        float t;
        switch (node) {
        case 0: t = m0; break;
        case 1: t = m1; break;
        case 2: t = m2; break;
        case 3: t = 0.5f * (lo + m1); break;
        case 4: t = 0.5f * (m1 + m0); break;
        case 5: t = 0.5f * (m0 + m2); break;
        default: t = 0.5f * (m2 + hi); break;
        }
        const unsigned in = inside(t);
        auto hit = [&](int n) { return (in >> (2 * n)) & 1u; };
        int k;
        if (hit(0)) { hi = m0; k = 1; } else { lo = m0; k = 2; }
        const float mk = k == 1 ? m1 : m2;
        int k3;
        if (hit(k)) { hi = mk; k3 = k == 1 ? 3 : 5; } else { lo = mk; k3 = k == 1 ? 4 : 6; }
        const float m3 = 0.5f * (lo + hi);
        if (hit(k3)) hi = m3;
        else lo = m3;
    }
    return clampf(0.5f * (lo + hi), 1.0e-4f, 1.0f);
}

// Persistent fluid cell that may border a solid one.  With a mesh, a cell
// next to a solid cell lies within h + sqrt(3) dx of its triangle, inside the
// raster's h + 2 dx guard, so it owns a key: keyless cells are skipped without
// reading their 18 neighbours.  Link counting and emission use this same test.
__device__ __forceinline__ bool may_have_links(const GeomArgs& a, int64_t bidx, uint8_t m_next, uint8_t m_prev) {
    // the key is loaded unconditionally, so its load overlaps the mask loads
    const bool keyed = a.b.keys == nullptr || a.b.keys[bidx] != 0xFFFFFFFFFFFFFFFFull;
    return persistent_fluid(m_next, m_prev) && keyed;
}

// ---------------------------------------------------------------------------
// Topology events and impulses (BF.metal:2557-2609 covered, 2616-2666
// uncovered).  A cell is an event when its occupancy changed this step and its
// impulse enters the loads.  Which cells are events depends on the geometry
// alone, so the event list is built with the cut-link list (k_link_count,
// the offset scan, k_links_emit); the impulses read the pre-step populations
// and run in k_topology, after the previous step's fluid kernel and before
// the link kernel overwrites any slot they read.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool topology_event(const FluidParams& fp, uint8_t m_next) {
    const int sel = fp.interpolated;
    const int mode = sel ? fp.force_mode : 6;
    const bool include_topo = !sel || fp.load_component != 1;
    if (!fp.accumulate || !include_topo) return false;
    return (m_next & kCovered) != 0 || ((m_next & kUncovered) != 0 && mode == 6);
}

// Impulse of one event cell into acc (force 0-2, torque 3-5, covered and
// uncovered counts 6-7), one warp per event: lane q loads direction q, then
// every lane forms the sums in the reference's direction order from the
// shuffled values (the same operations, in the same order, as one thread
// summing q = 0..18), so the lanes' loads overlap instead of one thread's
// long dependent chain.  Lane 0 adds the impulse to its acc.
template <class S>
__device__ __forceinline__ void topology_impulse_warp(const GeomArgs& a, int rep_s, int64_t gid, int lane,
                                                      double (&acc)[8]) {
    using R = typename S::R;
    const FluidParams& fp = a.fp;
    const int mode = fp.interpolated ? fp.force_mode : 6;
    const Grid& g = a.g;
    int x, y, z;
    unflat(g, gid, x, y, z);
    const uint8_t m1 = a.b.mask_next[gid];
    const typename S::T* A = (const typename S::T*)a.pops;
    const float4 w = a.b.wall[gid];
    const int q = lane < 19 ? lane : 0;
    R tx, ty, tz;
    if (m1 & kCovered) {
        // newly covered: previous fluid momentum (minus the wall-moving density for estimators 0-5)
        const R mine = lane < 19 ? canon_load<S>(A, g, rep_s, q, x, y, z) : R(0);
        R pd = 0, pmx = 0, pmy = 0, pmz = 0;
#pragma unroll
        for (int k = 0; k < 19; ++k) {
            const R prev = __shfl_sync(0xffffffffu, mine, k);
            pd += prev;
            pmx += prev * (R)cx(k);
            pmy += prev * (R)cy(k);
            pmz += prev * (R)cz(k);
        }
        tx = pmx;
        ty = pmy;
        tz = pmz;
        if (mode != 6) {
            tx = pmx - pd * (R)w.x;
            ty = pmy - pd * (R)w.y;
            tz = pmz - pd * (R)w.z;
        }
    } else {
        // newly uncovered: refill momentum plus the moving-domain stencil over
        // the neighbours that are fluid before and after the step
        const R feq_mine = lane < 19 ? feq_rt<R>(q, R(1), (R)w.x, (R)w.y, (R)w.z) : R(0);
        R sum_mine = R(0);
        bool live = false;
        if (lane >= 1 && lane < 19) {
            const int bx = x + cx(q), by = y + cy(q), bz = z + cz(q);
            if (inside(g, bx, by, bz)) {
                const int64_t nb = flat(g, bx, by, bz);
                const R old_out = canon_load<S>(A, g, rep_s, q, x, y, z);
                const R sup_in = canon_load<S>(A, g, rep_s, opp(q), bx, by, bz);
                live = (a.b.mask_prev[nb] & kPartMask) == 0 && (a.b.mask_next[nb] & kPartMask) == 0;
                sum_mine = old_out + sup_in;
            }
        }
        const uint32_t live_bits = __ballot_sync(0xffffffffu, live);
        R mx = 0, my = 0, mz = 0;
#pragma unroll
        for (int k = 0; k < 19; ++k) {
            const R v = __shfl_sync(0xffffffffu, feq_mine, k);
            mx += v * (R)cx(k);
            my += v * (R)cy(k);
            mz += v * (R)cz(k);
        }
        tx = -mx;
        ty = -my;
        tz = -mz;
#pragma unroll
        for (int k = 1; k < 19; ++k) {
            const R sum = __shfl_sync(0xffffffffu, sum_mine, k);
            if (!(live_bits & (1u << k))) continue;
            tx -= sum * (R)cx(k);
            ty -= sum * (R)cy(k);
            tz -= sum * (R)cz(k);
        }
    }
    if (lane == 0) {
        const V3 world = cell_world(fp, x, y, z);
        add_load<R>(acc, tx, ty, tz, (R)world.x, (R)world.y, (R)world.z, a.b.state->body, fp.f2p);
        acc[(m1 & kCovered) ? 6 : 7] += 1.0;
    }
}

// Per-block counts of cut links and topology events over the geometry box.
// Geometry only (masks and keys), so the pipelined path runs it with the
// next step's geometry, beside the fluid kernel.  Each active cell of a counted
// block also stores its link sources (bits 1-18) and event flag (bit 0) in
// cell_bits, so the emission reads one word instead of the 20 mask and key
// loads again.
__device__ __forceinline__ void count_block(const GeomArgs& a, int bxi, int byi, int bzi, int block,
                                            uint32_t* wcount) {
    if (block_inactive_at(a, bxi, byi, bzi)) {
        // no key, link or topology change in this block
        if (linear_tid() == 0) {
            a.b.block_counts[block] = 0;
            a.b.event_counts[block] = 0;
        }
        return;
    }
    uint32_t links = 0, events = 0;
    {
        int x, y, z;
        int64_t bidx;
        if (box_cell_at(a, bxi, byi, bzi, x, y, z, bidx) && cell_active(a, x, y, z)) {
            const int64_t gid = flat(a.g, x, y, z);
            const uint8_t m1 = a.b.mask_next[gid];
            const uint8_t m0 = a.b.mask_prev[gid];
            events = topology_event(a.fp, m1) ? 1u : 0u;
            const uint32_t sources = may_have_links(a, bidx, m1, m0) ? link_sources(a.g, a.b.mask_next, x, y, z) : 0u;
            links = __popc(sources);
            a.b.cell_bits[bidx] = sources | events;
        }
    }
    // links (at most 18 a cell) in the low half, events in the high half
    uint32_t w = links | events << 16;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    const int t = linear_tid();
    if ((t & 31) == 0) wcount[t >> 5] = w;
    __syncthreads();
    if (t == 0) {
        uint32_t tl = 0, te = 0;
        for (int k = 0; k < 8; ++k) {
            tl += wcount[k] & 0xFFFFu;
            te += wcount[k] >> 16;
        }
        a.b.block_counts[block] = tl;
        a.b.event_counts[block] = te;
    }
}
__global__ void __launch_bounds__(256) k_link_count(const GeomArgs a) {
    __shared__ uint32_t wcount[8];
    count_block(a, blockIdx.x, blockIdx.y, blockIdx.z, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                wcount);
}
// The same over the live list of the mesh resolve (the other blocks' counts
// are zeroed before): a fixed grid, list entry i to block i mod gridDim.x;
// (gx, gy) are the box launch's grid extents.
__global__ void __launch_bounds__(256) k_link_count_live(const GeomArgs a, int gx, int gy) {
    __shared__ uint32_t wcount[8];
    const uint32_t n = *a.b.live_count;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int b = (int)a.b.live_list[i];
        count_block(a, b % gx, (b / gx) % gy, b / (gx * gy), b, wcount);
        __syncthreads();
    }
}

// Topology impulses over the event list: a fixed grid of topo_blocks blocks of
// four warps, event i to warp i mod (4 topo_blocks) in list order, then
// fixed-order block trees into 8 partials per block (reduced by the link
// kernel's last block).
template <class S>
__global__ void __launch_bounds__(128) k_topology(const GeomArgs a, int rep_s) {
    __shared__ double sh[8][256];
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const uint32_t count = *a.b.event_total;
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    for (uint32_t i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); i < count; i += warps)
        topology_impulse_warp<S>(a, rep_s, a.b.event_cell[i], lane, acc);
    // most blocks hold no event: skip their FP64 tree
    bool nonzero = false;
    for (int k = 0; k < 8; ++k) nonzero = nonzero || acc[k] != 0.0;
    const bool block_nonzero = __syncthreads_or(nonzero) != 0;
    if (block_nonzero) block_sum<8>(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < 8; ++k) a.b.topo_partials[8 * blockIdx.x + k] = block_nonzero ? acc[k] : 0.0;
}

// Exclusive scans of the per-block link counts (blockIdx.y 0) and event
// counts (blockIdx.y 1) into block offsets, in two levels: k_scan_reduce sums
// each segment of kScanSegment counts (a block per segment); k_scan_apply adds
// the sums of the segments before its own and scans its segment (32
// consecutive counts per thread).  Block 0 also sets the totals (and the link
// list's overflow flag).  256-thread blocks: on the pipelined path they run
// beside the persistent fluid kernel, in the registers it leaves free.
// Integer sums: the offsets do not depend on the split.
constexpr int kScanThreads = 256;
constexpr int kScanPerThread = kScanSegment / kScanThreads;
__device__ __forceinline__ uint32_t block_sum_scan(uint32_t v, uint32_t* wtot) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) wtot[warp] = v;
    __syncthreads();
    uint32_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += wtot[w];
    return t;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const GeomArgs a) {
    __shared__ uint32_t wtot[kScanThreads / 32];
    const uint32_t* counts = blockIdx.y ? a.b.event_counts : a.b.block_counts;
    uint32_t* sums = blockIdx.y ? a.b.event_sums : a.b.scan_sums;
    const int nb = a.b.scan_blocks;
    const int lo = blockIdx.x * kScanSegment;
    const int hi = lo + kScanSegment < nb ? lo + kScanSegment : nb;
    uint32_t t = 0;
    for (int i = lo + threadIdx.x; i < hi; i += kScanThreads) t += counts[i];
    t = block_sum_scan(t, wtot);
    if (threadIdx.x == 0) sums[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const GeomArgs a, int nseg) {
    __shared__ uint32_t wtot[kScanThreads / 32];
    __shared__ uint32_t seg_base;
    const bool ev = blockIdx.y != 0;
    const uint32_t* counts = ev ? a.b.event_counts : a.b.block_counts;
    const uint32_t* sums = ev ? a.b.event_sums : a.b.scan_sums;
    uint32_t* offsets = ev ? a.b.event_offsets : a.b.block_offsets;
    const int nb = a.b.scan_blocks;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        uint32_t b = 0;
        for (int k = 0; k < (int)blockIdx.x; ++k) b += sums[k];
        seg_base = b;
        if (blockIdx.x == 0) {
            uint64_t total = 0;
            for (int k = 0; k < nseg; ++k) total += sums[k];
            if (ev) {
                *a.b.event_total = (uint32_t)total;  // at most one event a box cell
            } else {
                a.b.state->link_count = (int64_t)total;
                a.b.state->link_overflow = total > a.b.link_capacity ? 1u : 0u;
            }
        }
    }
    // kScanPerThread consecutive counts per thread
    const int first = blockIdx.x * kScanSegment + kScanPerThread * threadIdx.x;
    uint32_t c[kScanPerThread];
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) {
        c[k] = first + k < nb ? counts[first + k] : 0u;
        mine += c[k];
    }
    // block-exclusive prefix of the thread sums
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wtot[warp] = incl;
    __syncthreads();
    uint32_t base = seg_base;
    for (int w = 0; w < warp; ++w) base += wtot[w];
    base += incl - mine;
#pragma unroll
    for (int k = 0; k < kScanPerThread; ++k) {
        if (first + k < nb) offsets[first + k] = base;
        base += c[k];
    }
}

// Cut-link and event compaction: every persistent fluid cell appends its
// links (in direction order) at the block offset plus the shuffle prefix of
// the preceding threads, so the list is ordered by box cell then direction;
// every event cell appends itself to the event list in box-cell order.
__device__ __forceinline__ void emit_block(const GeomArgs& a, int bxi, int byi, int bzi, int block, uint32_t* wsum) {
    // blocks without links or events (most of the box) emit nothing; the
    // others were counted, so their active cells' bits are this step's
    if (a.b.block_counts[block] == 0 && a.b.event_counts[block] == 0) return;
    const Grid& g = a.g;
    uint32_t mine = 0, bits = 0, event = 0;
    int x = 0, y = 0, z = 0;
    int64_t bidx = 0, gid = 0;
    if (box_cell_at(a, bxi, byi, bzi, x, y, z, bidx) && cell_active(a, x, y, z)) {
        gid = flat(g, x, y, z);
        const uint32_t cb = a.b.cell_bits[bidx];
        event = cb & 1u;
        bits = cb & ~1u;
        mine = __popc(bits);
    }
    // block-exclusive prefix of (links, events), packed low / high 16 bits
    // (a block holds at most 256 x 18 links and 256 events)
    const uint32_t own = mine | event << 16;
    const int t = linear_tid();
    const int lane = t & 31, warp = t >> 5;
    uint32_t incl = own;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += wsum[w];
    const uint32_t excl = wbase + incl - own;
    if (event) a.b.event_cell[a.b.event_offsets[block] + (excl >> 16)] = (uint32_t)gid;
    if (mine == 0) return;
    uint32_t pos = a.b.block_offsets[block] + (excl & 0xFFFFu);
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        if (!(bits & (1u << q))) continue;
        if (pos < a.b.link_capacity) {
            int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
            wrap(g, sx, sy, sz);  // inside: the source is solid
            a.b.link_cell[pos] = (uint32_t)gid;
            a.b.link_meta[pos] = (uint32_t)q | ((uint32_t)(a.b.mask_next[flat(g, sx, sy, sz)] & kPartMask) << 8);
        }
        ++pos;
    }
}
__global__ void __launch_bounds__(256) k_links_emit(const GeomArgs a) {
    __shared__ uint32_t wsum[8];
    emit_block(a, blockIdx.x, blockIdx.y, blockIdx.z, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
               wsum);
}
// The same over the live list (k_link_count_live).
__global__ void __launch_bounds__(256) k_links_emit_live(const GeomArgs a, int gx, int gy) {
    __shared__ uint32_t wsum[8];
    const uint32_t n = *a.b.live_count;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const int b = (int)a.b.live_list[i];
        emit_block(a, b % gx, (b / gx) % gy, b / (gx * gy), b, wsum);
        __syncthreads();
    }
}

// Link fractions, one thread per emitted link (the bisections and ray roots
// are long and occur only at the surface: a thread per box cell would leave
// most lanes idle while a few run them).
__global__ void __launch_bounds__(128) k_links_fraction(const GeomArgs a, int geometry, int link_rule, int interpolated) {
    const Grid& g = a.g;
    int64_t count = a.b.state->link_count;
    if (count > (int64_t)a.b.link_capacity) count = a.b.link_capacity;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gid = a.b.link_cell[i];
        const int q = (int)(a.b.link_meta[i] & 0xFF);
        int x, y, z;
        unflat(g, gid, x, y, z);
        int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
        float qf = 0.5f;
        if (interpolated && wrap(g, sx, sy, sz)) {
            const int64_t s = flat(g, sx, sy, sz);
            if (geometry == BFX_GEOMETRY_ELLIPSOID) {
                qf = ellipsoid_link_fraction(a, x, y, z, sx, sy, sz);
            } else if (geometry == BFX_GEOMETRY_FLAPPING_WING) {
                qf = wing_link_fraction(a, q, sx, sy, sz);
            } else if (geometry == BFX_GEOMETRY_MESH) {
                if (link_rule == BFX_LINK_RAY_ROOT) {
                    qf = mesh_ray_root(a, x, y, z, sx, sy, sz);
                } else {
                    float sd = fminf(a.b.wall[s].w, 0.0f);
                    float fd = fmaxf(a.b.wall[gid].w, 0.0f);
                    qf = clampf(fd / fmaxf(fd - sd, 1.0e-6f), 1.0e-4f, 1.0f);
                }
            }
        }
        a.b.link_q[i] = qf;
    }
}

// Ray-root link fractions of a mesh, one link per 16-lane group
// (mesh_ray_root_group).
__global__ void __launch_bounds__(128) k_links_fraction_ray(const GeomArgs a) {
    const Grid& g = a.g;
    int64_t count = a.b.state->link_count;
    if (count > (int64_t)a.b.link_capacity) count = a.b.link_capacity;
    const int gl = threadIdx.x & 15;
    const int gshift = threadIdx.x & 16;
    const unsigned gmask = 0xFFFFu << gshift;
    const int64_t groups = (int64_t)gridDim.x * (blockDim.x / 16);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 16; i < count; i += groups) {
        const int64_t gid = a.b.link_cell[i];
        const int q = (int)(a.b.link_meta[i] & 0xFF);
        int x, y, z;
        unflat(g, gid, x, y, z);
        int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
        float qf = 0.5f;
        if (wrap(g, sx, sy, sz)) qf = mesh_ray_root_group(a, x, y, z, sx, sy, sz, gl, gmask, gshift);
        if (gl == 0) a.b.link_q[i] = qf;
    }
}

// ---------------------------------------------------------------------------
// Moving-wall bounce-back on the link list (BF.metal:2727-2873): reconstruct
// the incoming population, write it where the fluid step will read it, and
// accumulate the momentum-exchange load in FP64.
// ---------------------------------------------------------------------------
__device__ void finish_state(const GeomArgs& a, float gx, float gy, float gz, int substeps, int free_flight,
                             const bfx_bird* bird_ptr);

template <class S>
__global__ void __launch_bounds__(256) k_links_apply(const GeomArgs a, int rep_s, int with_topology, int fuse_finish,
                                                     const FinishParams fin) {
    __shared__ double sh[8][256];
    __shared__ int last_block;
    using T = typename S::T;
    using R = typename S::R;
    const FluidParams& fp = a.fp;
    const Grid& g = a.g;
    const int sel = fp.interpolated;
    const int mode = sel ? fp.force_mode : 6;
    const int include_link = !sel || fp.load_component != 2;
    T* A = (T*)a.pops;
    const double* body = a.b.state->body;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t count = a.b.state->link_count;
    if (count > (int64_t)a.b.link_capacity) count = a.b.link_capacity;
    const R cs2 = Lat<R>::cs2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gid = a.b.link_cell[i];
        const uint32_t meta = a.b.link_meta[i];
        const int q = (int)(meta & 0xFF);
        const int part = (int)(meta >> 8);
        int x, y, z;
        unflat(g, gid, x, y, z);
        int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
        if (!wrap(g, sx, sy, sz)) continue;  // cannot happen for an emitted link; keeps every index in range
        const int64_t src = flat(g, sx, sy, sz);
        R mwd = (R)fp.far[3];
        if (fp.local_density) {
            mwd = 0;
            for (int k = 0; k < 19; ++k) mwd += canon_load<S>(A, g, rep_s, k, x, y, z);
        }
        const R reflected = canon_load<S>(A, g, rep_s, opp(q), x, y, z);
        const R dx_ = (R)cx(q), dy_ = (R)cy(q), dz_ = (R)cz(q);
        R qf = R(0.5);
        const float4 ws = a.b.wall[src];
        R wvx = ws.x, wvy = ws.y, wvz = ws.z;
        int interp = sel;
        int fx = 0, fy = 0, fz = 0;
        if (interp) {
            // clamp(q, 1e-4, 1) and the wall velocity at the intersection (BF.metal:2737-2775)
            R ql = (R)a.b.link_q[i];
            ql = ql < R(1.0e-4) ? R(1.0e-4) : ql;
            qf = ql > R(1) ? R(1) : ql;
            const float4 wx = a.b.wall[gid];
            wvx = (R)wx.x + ((R)ws.x - (R)wx.x) * qf;
            wvy = (R)wx.y + ((R)ws.y - (R)wx.y) * qf;
            wvz = (R)wx.z + ((R)ws.z - (R)wx.z) * qf;
            if (qf <= R(0.5)) {
                fx = x + cx(q);
                fy = y + cy(q);
                fz = z + cz(q);
                const bool fin = inside(g, fx, fy, fz);
                if (!fin || (a.b.mask_next[flat(g, fx, fy, fz)] & kPartMask) != 0) {
                    interp = 0;
                    qf = R(0.5);
                    wvx = ws.x;
                    wvy = ws.y;
                    wvz = ws.z;
                }
            }
        }
        const R wqv = q <= 6 ? Lat<R>::w1 : Lat<R>::w2;
        const R wc = R(2) * wqv * mwd * (dx_ * wvx + dy_ * wvy + dz_ * wvz) / cs2;
        R value = reflected + wc;
        if (interp) {
            if (qf <= R(0.5)) {
                const R fo = canon_load<S>(A, g, rep_s, opp(q), fx, fy, fz);
                value = R(2) * qf * reflected + (R(1) - R(2) * qf) * fo + wc;
            } else {
                const R pin = canon_load<S>(A, g, rep_s, q, x, y, z);
                value = (reflected + wc) / (R(2) * qf) + (R(2) * qf - R(1)) * pin / (R(2) * qf);
            }
        }
        int slot_dir = q;
        T* slot = incoming_slot<S>(A, g, rep_s, q, x, y, z, slot_dir);
        if (slot) S::st_rt(slot, slot_dir, value);
        if (fp.accumulate && include_link && (fp.selected_part == 0 || fp.selected_part == part)) {
            R lx, ly, lz;
            switch (mode) {
            case 0:
                lx = -(value * (dx_ - wvx) - reflected * (-dx_ - wvx));
                ly = -(value * (dy_ - wvy) - reflected * (-dy_ - wvy));
                lz = -(value * (dz_ - wvz) - reflected * (-dz_ - wvz));
                break;
            case 1:
            case 6:
                lx = -(value + reflected) * dx_;
                ly = -(value + reflected) * dy_;
                lz = -(value + reflected) * dz_;
                break;
            case 2:
                lx = R(-2) * reflected * dx_;
                ly = R(-2) * reflected * dy_;
                lz = R(-2) * reflected * dz_;
                break;
            case 3:
                lx = -wc * dx_;
                ly = -wc * dy_;
                lz = -wc * dz_;
                break;
            case 4: {
                R r = value - reflected - wc;
                lx = -r * dx_;
                ly = -r * dy_;
                lz = -r * dz_;
                break;
            }
            case 5:
                lx = (value - reflected) * wvx;
                ly = (value - reflected) * wvy;
                lz = (value - reflected) * wvz;
                break;
            default: lx = ly = lz = 0; break;
            }
            const V3 world = cell_world(fp, x, y, z);
            const R dxs = (R)fp.dx;
            const R bpx = (R)world.x - qf * dx_ * dxs, bpy = (R)world.y - qf * dy_ * dxs, bpz = (R)world.z - qf * dz_ * dxs;
            add_load<R>(acc, lx, ly, lz, bpx, bpy, bpz, body, fp.f2p);
            acc[6] += (double)lx * (double)wvx + (double)ly * (double)wvy + (double)lz * (double)wvz;
        }
        if (a.b.link_tape) {
            // record the link for the adjoint: values, the bounce-back case and
            // the tangents of q and of the wall velocity at the link
            LinkTape<R>& t = ((LinkTape<R>*)a.b.link_tape)[i];
            const float* tg = a.b.link_tangent + (size_t)kLinkTangentWords * i;
            t.cell = (uint32_t)gid;
            t.dir = (uint32_t)q;
            t.kase = interp ? (qf <= R(0.5) ? 1u : 2u) : 0u;
            t._pad = 0;
            t.value = value;
            t.reflected = reflected;
            t.other = R(0);
            if (t.kase == 1) t.other = canon_load<S>(A, g, rep_s, opp(q), fx, fy, fz);
            if (t.kase == 2) t.other = canon_load<S>(A, g, rep_s, q, x, y, z);
            t.q = qf;
            t.wv[0] = wvx;
            t.wv[1] = wvy;
            t.wv[2] = wvz;
            const float4 wxf = a.b.wall[gid];
            const float ud[3] = {ws.x - wxf.x, ws.y - wxf.y, ws.z - wxf.z};
            for (int k = 0; k < kKinematicParams; ++k) {
                const float dqk = t.kase ? tg[k] : 0.0f;
                t.dq[k] = dqk;
                for (int c = 0; c < 3; ++c) {
                    const float duf = tg[4 + 3 * k + c], dus = tg[16 + 3 * k + c];
                    const float qv = (float)qf;
                    t.dwv[k][c] = t.kase ? (1.0f - qv) * duf + qv * dus + ud[c] * dqk : dus;
                }
            }
        }
    }
    // Block sums: the link loads, then this block's contiguous share of the
    // topology partials (most blocks hold no link and no topology impulse).
    bool nonzero = false;
    for (int k = 0; k < 8; ++k) nonzero = nonzero || acc[k] != 0.0;
    if (__syncthreads_or(nonzero)) block_sum<8>(acc, sh);
    double tp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (with_topology) {
        const int nb = a.b.topo_blocks;
        const int per = (nb + (int)gridDim.x - 1) / (int)gridDim.x;
        const int lo = (int)blockIdx.x * per;
        const int hi = lo + per < nb ? lo + per : nb;
        for (int i = lo + (int)threadIdx.x; i < hi; i += blockDim.x)
            for (int k = 0; k < 8; ++k) tp[k] += a.b.topo_partials[8 * (int64_t)i + k];
        bool tnz = false;
        for (int k = 0; k < 8; ++k) tnz = tnz || tp[k] != 0.0;
        if (__syncthreads_or(tnz)) block_sum<8>(tp, sh);
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < 8; ++k) {
            a.b.link_partials[16 * blockIdx.x + k] = acc[k];
            a.b.link_partials[16 * blockIdx.x + 8 + k] = tp[k];
        }
        __threadfence();
        last_block = atomicAdd(&a.b.state->apply_done, 1u) == gridDim.x - 1 ? 1 : 0;
    }
    __syncthreads();
    if (!last_block) return;
    // Last block: fixed-order sums of the per-block partials (the result does
    // not depend on which block finishes last).
    __threadfence();
    double l[8] = {0, 0, 0, 0, 0, 0, 0, 0}, t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x)
        for (int k = 0; k < 8; ++k) {
            l[k] += __ldcg(a.b.link_partials + 16 * i + k);
            t[k] += __ldcg(a.b.link_partials + 16 * i + 8 + k);
        }
    block_sum<8>(l, sh);
    block_sum<8>(t, sh);
    if (threadIdx.x == 0) {
        DeviceState* st = a.b.state;
        for (int k = 0; k < 3; ++k) {
            st->loads_lattice[k] = t[k] + l[k];
            st->loads_torque[k] = t[3 + k] + l[3 + k];
        }
        st->power_lattice = l[6];
        if (with_topology) {
            st->covered_count = (int64_t)t[6];
            st->uncovered_count = (int64_t)t[7];
        }
        st->apply_done = 0;
        if (fuse_finish)
            finish_state(a, fin.gravity[0], fin.gravity[1], fin.gravity[2], fin.substeps, fin.free_flight, a.b.bird);
    }
}

// ---------------------------------------------------------------------------
// End of step: FP64 6-DOF update (integrateBirdBody BF.metal:6574-6627 in
// FP64), runtime safety ledger (monitorBirdRuntimeSafety BF.metal:6629-6707),
// step counter.  One thread.
// ---------------------------------------------------------------------------
__device__ void qnormalize_d(double* q) {
    double n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    if (n2 > 1.0e-40) {
        double n = sqrt(n2);
        for (int k = 0; k < 4; ++k) q[k] = q[k] / n;
    } else {
        q[0] = q[1] = q[2] = 0.0;
        q[3] = 1.0;
    }
}

__device__ void finish_state(const GeomArgs& a, float gx, float gy, float gz, int substeps, int free_flight,
                             const bfx_bird* bird_ptr) {
    DeviceState* st = a.b.state;
    const FluidParams& fp = a.fp;
    if (free_flight) {
        const bfx_bird& bird = *bird_ptr;
        double force[3], torque[3];
        for (int k = 0; k < 3; ++k) {
            force[k] = st->loads_lattice[k] * (double)fp.f2p;
            force[k] = force[k] + (double)st->wing_reaction[k] + (double)st->wing_reaction[8 + k];
            torque[k] = st->loads_torque[k] + (double)st->wing_reaction[4 + k] + (double)st->wing_reaction[12 + k];
        }
        int n = substeps < 1 ? 1 : substeps;
        double dt = (double)fp.dt / (double)n;
        double mass = (double)bird.body_radii_mass.v[3];
        double inertia[3] = {(double)bird.inertia.v[0], (double)bird.inertia.v[1], (double)bird.inertia.v[2]};
        double grav[3] = {(double)gx, (double)gy, (double)gz};
        double* b = st->body;
        double v[3] = {b[7], b[8], b[9]}, x[3] = {b[0], b[1], b[2]}, o[4] = {b[3], b[4], b[5], b[6]},
               w[3] = {b[10], b[11], b[12]};
        qnormalize_d(o);
        for (int s = 0; s < n; ++s) {
            for (int k = 0; k < 3; ++k) v[k] += (force[k] / mass + grav[k]) * dt;
            for (int k = 0; k < 3; ++k) x[k] += v[k] * dt;
            // torque into the body frame: rotate by the conjugate
            double cq[3] = {-o[0], -o[1], -o[2]};
            double t1[3] = {cq[1] * torque[2] - cq[2] * torque[1], cq[2] * torque[0] - cq[0] * torque[2],
                            cq[0] * torque[1] - cq[1] * torque[0]};
            t1[0] *= 2.0;
            t1[1] *= 2.0;
            t1[2] *= 2.0;
            double c2[3] = {cq[1] * t1[2] - cq[2] * t1[1], cq[2] * t1[0] - cq[0] * t1[2], cq[0] * t1[1] - cq[1] * t1[0]};
            double tb[3];
            for (int k = 0; k < 3; ++k) tb[k] = torque[k] + o[3] * t1[k] + c2[k];
            double am[3] = {inertia[0] * w[0], inertia[1] * w[1], inertia[2] * w[2]};
            double gyr[3] = {w[1] * am[2] - w[2] * am[1], w[2] * am[0] - w[0] * am[2], w[0] * am[1] - w[1] * am[0]};
            for (int k = 0; k < 3; ++k) w[k] += ((tb[k] - gyr[k]) / inertia[k]) * dt;
            double cr[3] = {o[1] * w[2] - o[2] * w[1], o[2] * w[0] - o[0] * w[2], o[0] * w[1] - o[1] * w[0]};
            double d[4];
            for (int k = 0; k < 3; ++k) d[k] = o[3] * w[k] + cr[k];
            d[3] = -(o[0] * w[0] + o[1] * w[1] + o[2] * w[2]);
            double nq[4];
            for (int k = 0; k < 4; ++k) nq[k] = o[k] + 0.5 * dt * d[k];
            qnormalize_d(nq);
            for (int k = 0; k < 4; ++k) o[k] = nq[k];
        }
        b[0] = x[0]; b[1] = x[1]; b[2] = x[2];
        b[3] = o[0]; b[4] = o[1]; b[5] = o[2]; b[6] = o[3];
        b[7] = v[0]; b[8] = v[1]; b[9] = v[2];
        b[10] = w[0]; b[11] = w[1]; b[12] = w[2];

        // runtime safety on the FP32 view of the body
        float4 of = qnormalize(make_float4((float)b[3], (float)b[4], (float)b[5], (float)b[6]));
        const float* le = bird.safety_geometry.v;
        V3 ea = qrotate(of, v3(le[0], 0, 0)), eb = qrotate(of, v3(0, le[1], 0)), ec = qrotate(of, v3(0, 0, le[2]));
        V3 we = v3(fabsf(ea.x) + fabsf(eb.x) + fabsf(ec.x), fabsf(ea.y) + fabsf(eb.y) + fabsf(ec.y),
                   fabsf(ea.z) + fabsf(eb.z) + fabsf(ec.z));
        float dx = fp.dx;
        float margin = (fp.sponge_width + 3.0f) * dx;
        const int dims[3] = {a.g.nx, a.g.ny, a.g.nz};
        float pos[3] = {(float)b[0], (float)b[1], (float)b[2]};
        float wef[3] = {we.x, we.y, we.z};
        float clearance = __int_as_float(0x7f800000);
        for (int k = 0; k < 3; ++k) {
            float mn = fp.origin[k] + margin;
            float mx = fp.origin[k] + (float)dims[k] * dx - margin;
            float lc = pos[k] - wef[k] - mn;
            float uc = mx - pos[k] - wef[k];
            clearance = fminf(clearance, fminf(lc, uc));
        }
        float v2l = fp.v2l;
        V3 rv = v3((float)b[7] - fp.far[0] / v2l, (float)b[8] - fp.far[1] / v2l, (float)b[9] - fp.far[2] / v2l);
        float rel = length(rv);
        float rot = length(v3((float)b[10], (float)b[11], (float)b[12])) * bird.safety_geometry.v[3];
        float surface = rel + rot + bird.safety_limits.v[0];
        float mach = surface * v2l / sqrtf(1.0f / 3.0f);
        bool finite = isfinite(mach) && isfinite(clearance);
        for (int k = 0; k < 13; ++k) finite = finite && isfinite((float)b[k]);
        if (isfinite(mach)) st->safety_metrics[0] = fmaxf(st->safety_metrics[0], mach);
        if (isfinite(clearance)) st->safety_metrics[1] = fminf(st->safety_metrics[1], clearance);
        uint32_t flags = 0;
        if (!finite) flags |= 4u;
        if (isfinite(mach) && mach > bird.safety_limits.v[1]) flags |= 1u;
        if (isfinite(clearance) && clearance < 0.0f) flags |= 2u;
        uint64_t absolute = st->step + 1;
        if (flags != 0 && st->safety_event[2] == 0) {
            st->safety_event[0] = (uint32_t)(absolute & 0xFFFFFFFFu);
            st->safety_event[1] = (uint32_t)(absolute >> 32);
            st->safety_event[2] = flags;
            st->safety_event[3] = 0;
            st->safety_metrics[2] = mach;
            st->safety_metrics[3] = clearance;
        }
    }
    Objective* ob = a.b.objective;
    if (ob && ob->enabled) {
        if (st->link_count > ob->max_links) ob->max_links = st->link_count;
        // time-averaged load objective: this step completes relative step k
        const uint64_t k = st->step + 1 - ob->start;
        if (k >= ob->first && k <= ob->last) {
            const double inv = 1.0 / (double)(ob->last - ob->first + 1);
            double j = 0.0;
            for (int c = 0; c < 3; ++c) j += ob->force_weight[c] * (st->loads_lattice[c] * (double)fp.f2p);
            j += ob->power_weight * (-st->power_lattice * (double)fp.f2p / (double)fp.v2l);
            ob->value += j * inv;
        }
    }
    st->step += 1;
}

__global__ void k_finish(const GeomArgs a, float gx, float gy, float gz, int substeps, int free_flight,
                         const bfx_bird* bird_ptr) {
    finish_state(a, gx, gy, gz, substeps, free_flight, bird_ptr);
}

__global__ void k_record_sample(const GeomArgs a, bfx_run_sample* samples, uint64_t index, float dt) {
    const DeviceState* st = a.b.state;
    bfx_run_sample& s = samples[index];
    s.time = (double)(float)((double)st->step * (double)dt);
    for (int k = 0; k < 3; ++k) s.position[k] = st->body[k];
    for (int k = 0; k < 4; ++k) s.orientation[k] = st->body[3 + k];
    for (int k = 0; k < 3; ++k) {
        s.velocity[k] = st->body[7 + k];
        s.omega_body[k] = st->body[10 + k];
        s.force[k] = st->loads_lattice[k] * (double)a.fp.f2p;
        s.torque[k] = st->loads_torque[k];
        s.left_hinge_force[k] = st->wing_reaction[k];
        s.left_hinge_torque[k] = st->wing_reaction[4 + k];
        s.right_hinge_force[k] = st->wing_reaction[8 + k];
        s.right_hinge_torque[k] = st->wing_reaction[12 + k];
    }
    s.step = st->step;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

int slab_block_count(const BoxDesc& box) {
    dim3 grid, block;
    slab_shape(box, grid, block);
    return (int)(grid.x * grid.y * grid.z);
}

int box_block_count(const BoxDesc& box) {
    dim3 grid, block;
    box_shape(box, grid, block);
    return (int)(grid.x * grid.y * grid.z);
}

void launch_prepare(int geometry, float dt, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                    const GeomBuffers& gb, int init, cudaStream_t s) {
    GeomArgs a = make_geom(g, fp, box, gb, nullptr);
    if (geometry == BFX_GEOMETRY_FLAPPING_WING) k_prepare_wing<<<1, 32, 0, s>>>(a, init, dt);
    else k_prepare<<<1, 32, 0, s>>>(a, init, dt, 0.0f);
}

void launch_classify(int geometry, int has_prev, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                     const GeomBuffers& gb, cudaStream_t s, bool lean_raster) {
    GeomArgs a = make_geom(g, fp, box, gb, nullptr);
    dim3 grid, block;
    box_shape(box, grid, block);
    if (geometry == BFX_GEOMETRY_BIRD) {
        k_classify_bird<<<grid, block, 0, s>>>(a, has_prev);
    } else if (geometry == BFX_GEOMETRY_ELLIPSOID) {
        k_classify_ellipsoid<<<grid, block, 0, s>>>(a, has_prev);
    } else if (geometry == BFX_GEOMETRY_FLAPPING_WING) {
        k_classify_wing<<<grid, block, 0, s>>>(a, has_prev);
    } else if (geometry == BFX_GEOMETRY_MESH) {
        dim3 sgrid, sblock;
        slab_shape(box, sgrid, sblock);
        k_mesh_prepare<<<(gb.nverts + 255) / 256, 256, 0, s>>>(a);
        k_mesh_clear<<<sgrid, sblock, 0, s>>>(a);
        const unsigned rblocks = (unsigned)(((int64_t)gb.ntris * 32 + 127) / 128);
        if (lean_raster) k_mesh_raster<1><<<rblocks, 128, 0, s>>>(a);
        else k_mesh_raster<0><<<rblocks, 128, 0, s>>>(a);
        if (gb.live_list) cudaMemsetAsync(gb.live_count, 0, sizeof(uint32_t), s);
        k_mesh_resolve<<<sgrid, sblock, 0, s>>>(a, has_prev);
    }
}

#define BFX_DISPATCH_STORAGE(storage, FN, ...)                             \
    switch (storage) {                                                     \
    case BFX_STORAGE_F16_DEVIATION: FN<StoreF16Dev>(__VA_ARGS__); break;   \
    case BFX_STORAGE_BF16_DEVIATION: FN<StoreBF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_F64: FN<StoreF64>(__VA_ARGS__); break;                \
    default: FN<StoreF32>(__VA_ARGS__); break;                             \
    }

void launch_link_build(int geometry, int link_rule, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                       const GeomBuffers& gb, cudaStream_t s, cudaEvent_t lists_done) {
    GeomArgs a = make_geom(g, fp, box, gb, nullptr);
    dim3 grid, block;
    box_shape(box, grid, block);
    // with the mesh resolve's live list: count and emit over those blocks only
    const unsigned live_grid = (unsigned)std::min<int64_t>((int64_t)grid.x * grid.y * grid.z, 1024);
    if (gb.live_list) {
        cudaMemsetAsync(gb.block_counts, 0, (size_t)gb.scan_blocks * sizeof(uint32_t), s);
        cudaMemsetAsync(gb.event_counts, 0, (size_t)gb.scan_blocks * sizeof(uint32_t), s);
        k_link_count_live<<<live_grid, block, 0, s>>>(a, (int)grid.x, (int)grid.y);
    } else {
        k_link_count<<<grid, block, 0, s>>>(a);
    }
    const int nseg = (a.b.scan_blocks + kScanSegment - 1) / kScanSegment;
    k_scan_reduce<<<dim3(nseg, 2), kScanThreads, 0, s>>>(a);
    k_scan_apply<<<dim3(nseg, 2), kScanThreads, 0, s>>>(a, nseg);
    if (gb.live_list) k_links_emit_live<<<live_grid, block, 0, s>>>(a, (int)grid.x, (int)grid.y);
    else k_links_emit<<<grid, block, 0, s>>>(a);
    if (lists_done) cudaEventRecord(lists_done, s);
    if (geometry == BFX_GEOMETRY_MESH && link_rule == BFX_LINK_RAY_ROOT && fp.interpolated) {
        const unsigned rblocks =
            (unsigned)std::max<int64_t>(1, std::min<int64_t>(4096, ((int64_t)gb.link_capacity * 16 + 127) / 128));
        k_links_fraction_ray<<<rblocks, 128, 0, s>>>(a);
        return;
    }
    const unsigned fblocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(4096, ((int64_t)gb.link_capacity + 127) / 128));
    k_links_fraction<<<fblocks, 128, 0, s>>>(a, geometry, link_rule, fp.interpolated);
}

template <class S>
static void topology_s(const GeomArgs& a, int rep_s, cudaStream_t s) {
    k_topology<S><<<a.b.topo_blocks, 128, 0, s>>>(a, rep_s);
}
void launch_topology(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                     const GeomBuffers& gb, const FluidBuffers& fb, cudaStream_t s) {
    GeomArgs a = make_geom(g, fp, box, gb, fb.pops);
    BFX_DISPATCH_STORAGE(storage, topology_s, a, rep_s, s);
}

template <class S>
static void apply_s(const GeomArgs& a, int rep_s, int with_topology, const FinishParams* fin, cudaStream_t s) {
    const FinishParams none = {};
    k_links_apply<S><<<a.b.apply_blocks, 256, 0, s>>>(a, rep_s, with_topology, fin ? 1 : 0, fin ? *fin : none);
}

void launch_links_apply(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const GeomBuffers& gb,
                        const FluidBuffers& fb, int with_topology, const FinishParams* fin, cudaStream_t s) {
    BoxDesc box = {1, 1, 1, 1};
    GeomArgs a = make_geom(g, fp, box, gb, fb.pops);
    BFX_DISPATCH_STORAGE(storage, apply_s, a, rep_s, with_topology, fin, s);
}

void launch_integrate(const GridDesc& g, const FluidParams& fp, const GeomBuffers& gb, float gravity_x,
                      float gravity_y, float gravity_z, int substeps, int free_flight, cudaStream_t s) {
    BoxDesc box = {1, 1, 1, 1};
    GeomArgs a = make_geom(g, fp, box, gb, nullptr);
    k_finish<<<1, 1, 0, s>>>(a, gravity_x, gravity_y, gravity_z, substeps, free_flight, gb.bird);
}

void launch_record_sample(const GeomBuffers& gb, const FluidParams& fp, bfx_run_sample* samples, uint64_t index,
                          float dt, cudaStream_t s) {
    GridDesc g = {};
    BoxDesc box = {1, 1, 1, 1};
    GeomArgs a = make_geom(g, fp, box, gb, nullptr);
    k_record_sample<<<1, 1, 0, s>>>(a, samples, index, dt);
}

void launch_fill_wall(float4* wall, int64_t n, float w, cudaStream_t s) {
    k_fill_wall_w<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(wall, n, w);
}

}  // namespace bfx
