// TMA-staged fused stream + collide (see bfx_stream.cuh for the pipeline), for
// the 16-bit deviation formats with the TRT, regularized and RR3 operators.
// Included in the contracted translation unit only (bfx_fluid_fast.cu, after
// bfx_bulk_kernels.cuh).
//
// Two cells per lane (x and x + 32 of the warp's 64-cell row) are collided in
// packed f32x2 arithmetic (add / sub / mul.rn.f32x2, FFMA2), which halves the
// arithmetic instruction count.  The packed form is not used for the
// bit-identical FP32 step: the assembler fuses packed multiply / add pairs into
// FFMA2 even when each carries an explicit rounding mode (measured: a 1-ulp
// change of x*x + y*y + z*z in 17 % of cases under --fmad=false).
//
// The collision runs on the stored quantity itself, the scaled deviation
// d_q = s (f_q - w_q) (s = 4096 for FP16, 1 for BF16): a load or store is one
// conversion with no offset arithmetic, and the moments and non-equilibrium
// parts are formed from numbers of size s |f - w| rather than differences of
// numbers of size w.  With D = sum d / s (so rho = 1 + D) every term of the
// operator is linear in d or in the equilibrium deviation
//   e_q = s (feq_q - w_q) = w_q s D + s rho w_q (3 cu + 4.5 cu^2 - 1.5 u^2),
// split into its even part E_q (w_q s D + s rho w_q (4.5 cu^2 - 1.5 u^2)) and
// odd part O_q (3 s rho w_q cu), so TRT and the regularized operators keep
// their form with f -> d and feq -> e.
#include "bfx_stream.cuh"

#if !defined(BFX_VARIANT) || !defined(BFX_CONTRACTED)
#error "bfx_stream_kernels.cuh belongs to the contracted variant (bfx_fluid_fast.cu)"
#endif

namespace bfx {
namespace BFX_VARIANT {

// sponge_factor with a fast quotient (2 ulp; the 16-bit storage quantum is far larger).
__device__ __forceinline__ float sponge_factor_fast(const Grid& g, const FluidParams& fp, int x, int y, int z) {
    const unsigned dx = min((unsigned)x, (unsigned)(g.nx - 1 - x));
    const unsigned dy = min((unsigned)y, (unsigned)(g.ny - 1 - y));
    const unsigned dz = min((unsigned)z, (unsigned)(g.nz - 1 - z));
    const float distance = (float)min(dx, min(dy, dz));
    const float width = fp.sponge_width;
    if (distance >= width) return 0.0f;
    const float nd = fminf(fmaxf(__fdividef(width - distance, fmaxf(width, 1.0f)), 0.0f), 1.0f);
    return fp.sponge_strength * nd * nd;
}

// Collision of two cells in scaled deviation space (see above).  d: incoming
// deviations; post: outgoing deviations.  For the regularized operators,
// `slow` flags a lane where some outgoing population may fall below its
// positivity floor; the caller then runs admit_dev_lane on it.
template <int COLL>
__device__ __forceinline__ void collide_dev2(const P2 (&d)[19], float s, float inv_s, float omega_p, float omega_m,
                                             P2 (&post)[19], P2& rho, P2& ux, P2& uy, P2& uz, bool (&slow)[2]) {
    constexpr float cs2 = Lat<float>::cs2;
    P2 ps[19], md[19];
    P2 dsum = d[0];
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        ps[q] = d[q] + d[q + 1];
        md[q] = d[q] - d[q + 1];
        dsum = dsum + ps[q];
    }
    const P2 mx = pair_dot<0>(md), my = pair_dot<1>(md), mz = pair_dot<2>(md);
    P2 k;
#pragma unroll
    for (int l = 0; l < 2; ++l) {
        float r = __fmaf_rn(Lanes<P2>::get(dsum, l), inv_s, 1.0f);
        r = r > 1.0e-8f ? r : 1.0e-8f;
        Lanes<P2>::set(rho, l, r);
        Lanes<P2>::set(k, l, __fdividef(inv_s, r));  // 2 ulp: far below the 16-bit storage quantum
        slow[l] = r > 1.0e3f;
    }
    ux = mx * k;
    uy = my * k;
    uz = mz * k;
    const P2 t15 = 1.5f * ((ux * ux + uy * uy) + uz * uz);
    const P2 sr = s * rho;
    const P2 sr1 = Lat<float>::w1 * sr, sr2 = Lat<float>::w2 * sr;
    const P2 e0 = Lat<float>::w0 * dsum - (Lat<float>::w0 * sr) * t15;
    // per weight class: E = a + b cu^2 with a = w D - s rho w t15, b = 4.5 s rho w;
    // O = o cu with o = 3 s rho w
    const P2 a1 = Lat<float>::w1 * dsum - sr1 * t15, a2 = Lat<float>::w2 * dsum - sr2 * t15;
    const P2 b1 = 4.5f * sr1, b2 = 4.5f * sr2, o1 = 3.0f * sr1, o2 = 3.0f * sr2;
    auto even_odd = [&](int q, P2& E, P2& O) {
        const P2 cu = cdot_pair(q, ux, uy, uz);
        E = (q <= 6 ? a1 : a2) + ((q <= 6 ? b1 : b2) * cu) * cu;
        O = (q <= 6 ? o1 : o2) * cu;
    };
    if constexpr (COLL == BFX_COLLISION_TRT) {
        // BF.metal:3063-3093 on the deviations (w_q is its own even part):
        // with d_q = p + m, d_q' = p - m (p, m the pair's even and odd halves)
        // post_q = P + M, post_q' = P - M, P = p - w+ (p - E), M = m - w- (m - O)
        post[0] = d[0] - omega_p * (d[0] - e0);
        const float kp = 0.5f * (1.0f - omega_p), km = 0.5f * (1.0f - omega_m);
        // w+ E = w+ a + (w+ b) cu^2 and w- O = (w- o) cu with the class factors scaled once
        const P2 pa1 = omega_p * a1, pa2 = omega_p * a2, pb1 = omega_p * b1, pb2 = omega_p * b2;
        const P2 mo1 = omega_m * o1, mo2 = omega_m * o2;
#pragma unroll
        for (int q = 1; q < 19; q += 2) {
            const P2 cu = cdot_pair(q, ux, uy, uz);
            const P2 P = kp * ps[q] + ((q <= 6 ? pa1 : pa2) + ((q <= 6 ? pb1 : pb2) * cu) * cu);
            const P2 M = km * md[q] + (q <= 6 ? mo1 : mo2) * cu;
            post[q] = P + M;
            post[q + 1] = P - M;
        }
        slow[0] = slow[1] = false;
    } else {
        P2 E[19], O[19];
#pragma unroll
        for (int q = 1; q < 19; q += 2) even_odd(q, E[q], O[q]);
        // regularized / RR3 (BF.metal:2917-3062), pair-restated as in collide_pairs
        P2 nps[19];
        P2 ntot = d[0] - e0;
#pragma unroll
        for (int q = 1; q < 19; q += 2) {
            nps[q] = ps[q] - 2.0f * E[q];
            ntot = ntot + nps[q];
        }
        const P2 dsx = pair_second<0, 0>(nps) - cs2 * ntot;
        const P2 dsy = pair_second<1, 1>(nps) - cs2 * ntot;
        const P2 dsz = pair_second<2, 2>(nps) - cs2 * ntot;
        const P2 odx = pair_second<0, 1>(nps), ody = pair_second<0, 2>(nps), odz = pair_second<1, 2>(nps);
        const P2 aXxy = (2.0f * ux) * odx + uy * dsx;
        const P2 aXxz = (2.0f * ux) * ody + uz * dsx;
        const P2 aXyy = ux * dsy + (2.0f * uy) * odx;
        const P2 aXzz = ux * dsz + (2.0f * uz) * ody;
        const P2 aYyz = (2.0f * uy) * odz + uz * dsy;
        const P2 aYzz = uy * dsz + (2.0f * uz) * odz;
        const P2 trace = (dsx + dsy) + dsz;
        const P2 cax = dsx - cs2 * trace, cay = dsy - cs2 * trace, caz = dsz - cs2 * trace;
        const float om = 1.0f - omega_p;
        const float om0 = om * (Lat<float>::w0 * 4.5f * -cs2);
        const float om1 = om * (Lat<float>::w1 * 4.5f), om2 = om * (Lat<float>::w2 * 4.5f);
        const float ot1 = om * (Lat<float>::w1 * 13.5f), ot2 = om * (Lat<float>::w2 * 13.5f);
        // positivity floor max(1e-12, 1e-6 feq) <= w_q / 2 unless rho > 1e3 (flagged
        // above), so a population at or above w_q / 2 needs no admission:
        // the exact test runs only on a lane with a deviation below -s w_q / 2
        post[0] = e0 + om0 * trace;
        const float h0 = -0.5f * Lat<float>::w0 * s, h1 = -0.5f * Lat<float>::w1 * s, h2 = -0.5f * Lat<float>::w2 * s;
#pragma unroll
        for (int l = 0; l < 2; ++l) slow[l] = slow[l] || Lanes<P2>::get(post[0], l) < h0;
#pragma unroll
        for (int q = 1; q < 19; q += 2) {
            const float hx = (float)(cx(q) * cx(q)) - cs2, hy = (float)(cy(q) * cy(q)) - cs2,
                        hz = (float)(cz(q) * cz(q)) - cs2;
            P2 contraction;
            if (cx(q) != 0 && cy(q) != 0) contraction = (cax + dsy) + 2.0f * (cx(q) * cy(q) > 0 ? odx : -odx);
            else if (cx(q) != 0 && cz(q) != 0) contraction = (cax + dsz) + 2.0f * (cx(q) * cz(q) > 0 ? ody : -ody);
            else if (cy(q) != 0 && cz(q) != 0) contraction = (cay + dsz) + 2.0f * (cy(q) * cz(q) > 0 ? odz : -odz);
            else contraction = cx(q) != 0 ? cax : (cy(q) != 0 ? cay : caz);
            const P2 X = E[q] + (q <= 6 ? om1 : om2) * contraction;
            P2 Y = O[q];
            if (COLL == BFX_COLLISION_RR3) {
                P2 third = pv(0.0f);
                bool any = false;
                auto add = [&](int da, float hb, P2 amp) {
                    if (da == 0) return;
                    const P2 t = ((float)da * hb) * amp;
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
            const float hq = q <= 6 ? h1 : h2;
#pragma unroll
            for (int l = 0; l < 2; ++l)
                slow[l] = slow[l] || Lanes<P2>::get(post[q], l) < hq || Lanes<P2>::get(post[q + 1], l) < hq;
        }
    }
}

// x faces without their halo fill (BulkArgs::face_values): at x = 0 (SGN +1)
// every direction with c_x > 0 comes from beyond the -x face, at x = nx - 1
// (SGN -1) every direction with c_x < 0 from beyond the +x face; the halo
// fill takes the x face first for a source outside in several axes, so these
// are its values for every such direction, rows at the y / z faces included.
// The values are kernel parameters: no load waits on memory.
template <int SGN>
__device__ __forceinline__ void x_face_values(const BulkArgs& a, int l, P2 (&dv)[19]) {
    constexpr int f = SGN > 0 ? 0 : 1;
#pragma unroll
    for (int q = 1; q < 19; ++q)
        if (cx(q) == SGN) Lanes<P2>::set(dv[q], l, a.face_dev[f][q]);
}

// Exact positivity admission of one lane (BF.metal:3035-3052) on absolute
// populations f = w_q + d / s: the admissible scale over every direction, and
// the scaled blend feq + scale (cand - feq) when it is below 1.
__device__ __forceinline__ void admit_dev_lane(P2 (&post)[19], int l, float rho, float ux, float uy, float uz,
                                               float s, float inv_s, float& activation, float& restriction) {
    float scale = 1.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const float fe = feq_rt<float>(q, rho, ux, uy, uz);
        const float cand = __fmaf_rn(Lanes<P2>::get(post[q], l), inv_s, wq<float>(q));
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
        activation = 1.0f;
        restriction = 1.0f - scale;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const float fe = feq_rt<float>(q, rho, ux, uy, uz);
            const float cand = __fmaf_rn(Lanes<P2>::get(post[q], l), inv_s, wq<float>(q));
            Lanes<P2>::set(post[q], l, (fe + scale * (cand - fe) - wq<float>(q)) * s);
        }
    }
}

// Tile coordinates (x tile, y tile, z plane) of a CTA's tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...: decomposed once, then advanced by the grid
// stride (decomposed on the host, StreamTiles) with carries, with no integer
// division per tile.
// INCR 0 decomposes each tile index instead: measured faster for the
// regularized operators (their register allocation at the 128 cap), slower
// for TRT (0.523 against 0.496 ms on the 512x256x256 plates).
template <bool INCR>
struct TileWalk {
    int tx, ty, tz;
    __device__ __forceinline__ void at(const StreamTiles& tl, int tile) {
        tx = tile % tl.tiles_x;
        const int r = tile / tl.tiles_x;
        ty = r % tl.tiles_y;
        tz = r / tl.tiles_y;
    }
    __device__ __forceinline__ void start(const StreamTiles& tl) { at(tl, (int)blockIdx.x); }
    // to tile `tile` (the current one plus gridDim.x)
    __device__ __forceinline__ void next(const StreamTiles& tl, int tile) {
        if (!INCR) {
            at(tl, tile);
            return;
        }
        tx += tl.step_x;
        int carry = tx >= tl.tiles_x;
        tx -= carry ? tl.tiles_x : 0;
        ty += tl.step_y + carry;
        carry = ty >= tl.tiles_y;
        ty -= carry ? tl.tiles_y : 0;
        tz += tl.step_z + carry;
    }
};

// ---------------------------------------------------------------------------
// The staged kernel.  CAPTURE 1 also writes the macroscopic fields.
// ---------------------------------------------------------------------------
// One CTA per SM with the operator's tile shape (StreamShape).
template <class S, int REP_S, int COLL, int CAPTURE>
__global__ void __maxnreg__(StreamShape<COLL>::max_regs)
    k_stream(const __grid_constant__ CUtensorMap map, const BulkArgs a, const StreamTiles tl) {
    using T = typename S::T;
    using G = StreamGeom<T, COLL>;
    using SH = StreamShape<COLL>;
    constexpr int NS = G::stages;
    extern __shared__ __align__(128) uint8_t smem_raw[];
    // bulk-tensor destinations must start on 128 B: align the ring explicitly
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t sbase = (raw + 127u) & ~127u;
    uint8_t* smem = smem_raw + (sbase - raw);
    const uint32_t full0 = sbase + NS * G::stage_bytes;
    const uint32_t empty0 = full0 + 8 * NS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, SH::consumers);
        }
        mbar_fence_init();
    }
    __syncthreads();
    const Grid& g = a.g;
    // bounded waits; the test hook can shorten them and withhold one tile
    const uint32_t hook_limit = a.state->test_wait_limit;
    const uint32_t wait_limit = hook_limit ? hook_limit : kWaitLimit;
    if (warp == SH::consumers) {
        // producer: one thread issues the 19 box loads of each tile
        if (lane != 0) return;
        const int stall_tile = (int)a.state->test_stall_tile1 - 1;
        int issued = 0;
        bool failed = false, stalled = false;
        TileWalk<SH::trt> walk;
        walk.start(tl);
        for (int k = 0;; ++k) {
            const int tile = blockIdx.x + k * gridDim.x;
            if (tile >= tl.ntiles) break;
            if (k > 0) walk.next(tl, tile);
            const int s = k % NS;
            if (k >= NS && !mbar_wait(empty0 + 8 * s, ((k / NS) + 1) & 1, wait_limit)) {
                atomicOr(&a.state->stream_error, 1u);
                failed = true;
                break;
            }
            if (tile == stall_tile) {
                // test hook: no loads (and no arrival) for this tile, so its
                // consumers' wait runs out; nothing is left in flight for it
                issued = k + 1;
                stalled = true;
                continue;
            }
            const int y0 = walk.ty * SH::Y;
            const int z = walk.tz;
            const int x0 = walk.tx * kTileX * SH::W;
            const uint32_t bar = full0 + 8 * s;
            mbar_expect_tx(bar, G::tx_bytes);
            const uint32_t dst = sbase + s * G::stage_bytes;
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                if (REP_S) tma_load_4d(dst + q * G::plane_bytes, &map, x0, y0 + 1, z + 1, q, bar);
                else tma_load_4d(dst + q * G::plane_bytes, &map, x0, y0 + 1 - cy(q), z + 1 - cz(q), opp(q), bar);
            }
            issued = k + 1;
        }
        if (failed || stalled) {
            // leave no bulk copy in flight into this CTA's shared memory (the
            // consumers may have stopped consuming): wait (bounded) for the
            // loads of the last NS tiles issued, the only ones that can still
            // be in flight, to complete
            for (int k = issued - NS < 0 ? 0 : issued - NS; k < issued; ++k)
                if ((int)blockIdx.x + k * (int)gridDim.x != stall_tile)
                    (void)mbar_wait(full0 + 8 * (k % NS), (k / NS) & 1, wait_limit);
        }
        return;
    }
    // consumers: warp w takes row y0 + w % Y and the 64 cells from
    // x0 + 64 (w / Y); lane l the cells at +l and +l + 32 of those.
    // The mask bytes of the next tile are loaded one tile ahead, so their HBM
    // latency overlaps the current tile's collision.
    const FluidParams& fp = a.fp;
    const uint32_t step_seed = S::kStochastic ? (uint32_t)a.state->step : 0u;
    struct Cells {
        int xa, y, z;
        uint32_t gida;
        bool va, vb;
        uint8_t ma, mb;
    };
    auto locate = [&](const TileWalk<SH::trt>& w, Cells& c) {
        c.y = w.ty * SH::Y + warp % SH::Y;
        c.z = w.tz;
        c.xa = w.tx * kTileX * SH::W + kTileX * (warp / SH::Y) + lane;
        const bool row_ok = c.y < g.ny;
        c.gida = (uint32_t)c.xa + (uint32_t)g.nx * ((uint32_t)c.y + (uint32_t)g.ny * (uint32_t)c.z);
        c.va = row_ok && c.xa < g.nx;
        c.vb = row_ok && c.xa + 32 < g.nx;
        c.ma = 0;
        c.mb = 0;
        if (a.mask) {
            if (c.va) c.ma = a.mask[c.gida];
            if (c.vb) c.mb = a.mask[c.gida + 32];
        }
    };
    Cells next;
    TileWalk<SH::trt> walk;
    walk.start(tl);
    if ((int)blockIdx.x < tl.ntiles) locate(walk, next);
    for (int k = 0;; ++k) {
        const int tile = blockIdx.x + k * gridDim.x;
        if (tile >= tl.ntiles) break;
        const int s = k % NS;
        const Cells cur = next;
        if (tile + (int)gridDim.x < tl.ntiles) {
            walk.next(tl, tile + (int)gridDim.x);
            locate(walk, next);
        }
        const int xa = cur.xa, xb = cur.xa + 32, y = cur.y, z = cur.z;
        const uint32_t gida = cur.gida;
        bool va = cur.va, vb = cur.vb;
        const uint8_t ma = cur.ma, mb = cur.mb;
        if (!mbar_wait(full0 + 8 * s, (k / NS) & 1, wait_limit)) {
            atomicOr(&a.state->stream_error, 2u);
            break;
        }
        const T* row = (const T*)(smem + s * G::stage_bytes) + (warp % SH::Y) * G::row + kTileX * (warp / SH::Y);
        constexpr float dscale = S::kDevScale, inv_dscale = 1.0f / S::kDevScale;
        P2 dv[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int base = REP_S ? 1 : 1 - cx(q);
            const T* p = row + q * (G::plane_bytes / (int)sizeof(T)) + base + lane;
            dv[q] = make_float2(S::ld_dev(p), S::ld_dev(p + 32));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * s);
        if (a.face_values) {
            // no x-halo fill: the warp's cells at x = 0 or x = nx - 1 take the
            // x-face values (one warp-uniform test for the warp's 64 cells)
            const int xbase = xa - lane;
            if (xbase == 0 || xbase + kTileX >= g.nx) {
                if (xa == 0) x_face_values<1>(a, 0, dv);
                if (xa == g.nx - 1) x_face_values<-1>(a, 0, dv);
                if (xb == g.nx - 1) x_face_values<-1>(a, 1, dv);
            }
        }
        // solid and newly uncovered cells (mask byte set) are left to k_rare
        va = va && ma == 0;
        vb = vb && mb == 0;
        if (!__any_sync(0xffffffffu, va || vb)) continue;
        P2 post[19], rho, ux, uy, uz;
        bool slow[2];
        float activation[2] = {0.0f, 0.0f}, restriction[2] = {0.0f, 0.0f};
        collide_dev2<COLL>(dv, dscale, inv_dscale, fp.omega_p, fp.omega_m, post, rho, ux, uy, uz, slow);
        if (COLL != BFX_COLLISION_TRT) {
#pragma unroll
            for (int l = 0; l < 2; ++l)
                if (slow[l])
                    admit_dev_lane(post, l, Lanes<P2>::get(rho, l), Lanes<P2>::get(ux, l), Lanes<P2>::get(uy, l),
                                   Lanes<P2>::get(uz, l), dscale, inv_dscale, activation[l], restriction[l]);
        }
        if (fp.has_sponge) {
            const float spa = va ? sponge_factor_fast(g, fp, xa, y, z) : 0.0f;
            const float spb = vb ? sponge_factor_fast(g, fp, xb, y, z) : 0.0f;
            if (spa > 0.0f || spb > 0.0f) {
                // post + (far - post) * sp on the deviations in packed
                // arithmetic; a lane with a zero factor adds zero (its value
                // is unchanged, a negative zero at most turning positive)
                const P2 sp = make_float2(spa, spb);
#pragma unroll
                for (int q = 0; q < 19; ++q) post[q] = post[q] + (pv(a.far_dev[q]) - post[q]) * sp;
            }
        }
        if (CAPTURE) {
            P2 cd = pv(0.0f), cmx = pv(0.0f), cmy = pv(0.0f), cmz = pv(0.0f);
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                cd = cd + post[q];
                if (cx(q) > 0) cmx = cmx + post[q];
                if (cx(q) < 0) cmx = cmx - post[q];
                if (cy(q) > 0) cmy = cmy + post[q];
                if (cy(q) < 0) cmy = cmy - post[q];
                if (cz(q) > 0) cmz = cmz + post[q];
                if (cz(q) < 0) cmz = cmz - post[q];
            }
            // rho = 1 + sum d / s, momentum = sum c d / s (sum w_q c_q = 0)
#pragma unroll
            for (int l = 0; l < 2; ++l) {
                if (!(l ? vb : va)) continue;
                float r = __fmaf_rn(Lanes<P2>::get(cd, l), inv_dscale, 1.0f);
                r = r > 1.0e-8f ? r : 1.0e-8f;
                const uint32_t gl = gida + 32 * l;
                a.density[gl] = r;
                a.velocity[gl] = make_float4(Lanes<P2>::get(cmx, l) * inv_dscale / r,
                                             Lanes<P2>::get(cmy, l) * inv_dscale / r,
                                             Lanes<P2>::get(cmz, l) * inv_dscale / r, 0.0f);
            }
        }
        if (COLL != BFX_COLLISION_TRT) {
            for (int l = 0; l < 2; ++l)
                if ((l ? vb : va) && activation[l] != 0.0f) {
                    atomicAdd(&a.state->limiter_count, 1.0);
                    atomicMax(&a.state->limiter_max_bits, __float_as_uint(restriction[l]));
                }
        }
        const uint32_t pid =
            (uint32_t)(xa + 1) + (uint32_t)g.px * ((uint32_t)(y + 1) + (uint32_t)g.py * (uint32_t)(z + 1));
        if constexpr (S::kStochastic) {
            // BF16: stochastic rounding (sr_seed), one stream per cell
            uint32_t ra = sr_seed(gida, step_seed), rb = sr_seed(gida + 32, step_seed);
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                T* p = REP_S ? (T*)a.plane[opp(q)] + pid : (T*)a.plane[q] + (uint32_t)(pid + (uint32_t)a.doff[q]);
                ra = sr_next(ra);
                rb = sr_next(rb);
                if (va) S::st_dev_sr(p, post[q].x, ra);
                if (vb) S::st_dev_sr(p + 32, post[q].y, rb);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                T* p = REP_S ? (T*)a.plane[opp(q)] + pid : (T*)a.plane[q] + (uint32_t)(pid + (uint32_t)a.doff[q]);
                if (va) S::st_dev(p, post[q].x);
                if (vb) S::st_dev(p + 32, post[q].y);
            }
        }
    }
}

// Resident CTAs per SM of one instantiation; the first call also raises its
// dynamic shared-memory limit (done at simulation creation, outside any capture).
template <class S, int REP, int COLL, int CAPTURE>
static int stream_blocks_per_sm() {
    using G = StreamGeom<typename S::T, COLL>;
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaFuncSetAttribute(k_stream<S, REP, COLL, CAPTURE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             G::smem_bytes);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stream<S, REP, COLL, CAPTURE>,
                                                      StreamShape<COLL>::threads, G::smem_bytes);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

template <class S, int REP, int COLL, int C>
static void stream_launch(const GridDesc& gd, const BulkArgs& a, const CUtensorMap& map, int sm_count,
                          cudaStream_t s) {
    using G = StreamGeom<typename S::T, COLL>;
    using SH = StreamShape<COLL>;
    StreamTiles tl;
    tl.tiles_x = (gd.nx + kTileX * SH::W - 1) / (kTileX * SH::W);
    tl.tiles_y = (gd.ny + SH::Y - 1) / SH::Y;
    tl.ntiles = tl.tiles_x * tl.tiles_y * gd.nz;
    int blocks = stream_blocks_per_sm<S, REP, COLL, C>() * sm_count;
    if (blocks > tl.ntiles) blocks = tl.ntiles;
    tl.step_x = blocks % tl.tiles_x;
    tl.step_y = (blocks / tl.tiles_x) % tl.tiles_y;
    tl.step_z = blocks / tl.tiles_x / tl.tiles_y;
    k_stream<S, REP, COLL, C><<<blocks, SH::threads, G::smem_bytes, s>>>(map, a, tl);
}

template <class S, int REP, int COLL>
static void stream_t(const GridDesc& gd, const BulkArgs* a, const CUtensorMap* map, int sm_count, cudaStream_t s) {
    if (!a) {
        // preparation only
        stream_blocks_per_sm<S, REP, COLL, 0>();
        stream_blocks_per_sm<S, REP, COLL, 1>();
        return;
    }
    if (a->capture == 1) stream_launch<S, REP, COLL, 1>(gd, *a, *map, sm_count, s);
    else stream_launch<S, REP, COLL, 0>(gd, *a, *map, sm_count, s);
}

// Launch (a non-null) or prepare (a null) the staged kernel of one storage
// type and collision operator (TRT, regularized or RR3).
template <class S>
static void stream_s(int collision, int rep_s, const GridDesc& g, const BulkArgs* a, const CUtensorMap* map,
                     int sm_count, cudaStream_t s) {
    switch (collision * 2 + rep_s) {
    case 1: stream_t<S, 1, BFX_COLLISION_TRT>(g, a, map, sm_count, s); break;
    case 4: stream_t<S, 0, BFX_COLLISION_REGULARIZED>(g, a, map, sm_count, s); break;
    case 5: stream_t<S, 1, BFX_COLLISION_REGULARIZED>(g, a, map, sm_count, s); break;
    case 6: stream_t<S, 0, BFX_COLLISION_RR3>(g, a, map, sm_count, s); break;
    case 7: stream_t<S, 1, BFX_COLLISION_RR3>(g, a, map, sm_count, s); break;
    default: stream_t<S, 0, BFX_COLLISION_TRT>(g, a, map, sm_count, s); break;
    }
}

}  // namespace BFX_VARIANT
}  // namespace bfx
