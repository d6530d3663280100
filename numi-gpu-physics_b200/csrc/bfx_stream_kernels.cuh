// TMA-staged fused stream + collide (see bfx_stream.cuh for the pipeline), for
// the 16-bit deviation formats with the TRT operator.  Included in the
// contracted translation unit only (bfx_fluid_fast.cu, after
// bfx_bulk_kernels.cuh).
//
// Two cells per lane (x and x + 32 of the warp's 64-cell row) are collided in
// packed f32x2 arithmetic (add / sub / mul.rn.f32x2, FFMA2), which halves the
// arithmetic instruction count.  The packed form is not used for the
// bit-identical FP32 step: the assembler fuses packed multiply / add pairs into
// FFMA2 even when each carries an explicit rounding mode (measured: a 1-ulp
// change of x*x + y*y + z*z in 17 % of cases under --fmad=false).
#include "bfx_stream.cuh"

#if !defined(BFX_VARIANT) || !defined(BFX_CONTRACTED)
#error "bfx_stream_kernels.cuh belongs to the contracted variant (bfx_fluid_fast.cu)"
#endif

namespace bfx {
namespace BFX_VARIANT {

// c_q . u with the zero products dropped (cdotq on pairs)
__device__ __forceinline__ P2 cdot2(int q, P2 ux, P2 uy, P2 uz) {
    P2 r = pv(0.0f);
    bool first = true;
    if (cx(q) != 0) { r = cx(q) > 0 ? ux : -ux; first = false; }
    if (cy(q) != 0) { r = first ? (cy(q) > 0 ? uy : -uy) : (cy(q) > 0 ? r + uy : r - uy); first = false; }
    if (cz(q) != 0) { r = first ? (cz(q) > 0 ? uz : -uz) : (cz(q) > 0 ? r + uz : r - uz); }
    return r;
}

// Moments in the reference order (moments<R> on pairs).
__device__ __forceinline__ void moments2(const P2 (&f)[19], P2& rho, P2& ux, P2& uy, P2& uz) {
    P2 r = pv(0.0f), mx = pv(0.0f), my = pv(0.0f), mz = pv(0.0f);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        r = r + f[q];
        if (cx(q) > 0) mx = mx + f[q];
        if (cx(q) < 0) mx = mx - f[q];
        if (cy(q) > 0) my = my + f[q];
        if (cy(q) < 0) my = my - f[q];
        if (cz(q) > 0) mz = mz + f[q];
        if (cz(q) < 0) mz = mz - f[q];
    }
    r.x = r.x > 1.0e-8f ? r.x : 1.0e-8f;
    r.y = r.y > 1.0e-8f ? r.y : 1.0e-8f;
    rho = r;
    const P2 inv = make_float2(1.0f / r.x, 1.0f / r.y);
    ux = mx * inv;
    uy = my * inv;
    uz = mz * inv;
}

// collide<float, COLL> on two cells; the limiter runs lane by lane through
// the scalar operator.
template <int COLL>
__device__ __forceinline__ void collide2(const P2 (&f)[19], P2 rho, P2 ux, P2 uy, P2 uz, float omega_p, float omega_m,
                                         P2 (&post)[19], float (&activation)[2], float (&restriction)[2]) {
    if (COLL == BFX_COLLISION_TRT_LIMITER) {
#pragma unroll
        for (int l = 0; l < 2; ++l) {
            float fs[19], ps[19];
#pragma unroll
            for (int q = 0; q < 19; ++q) fs[q] = l ? f[q].y : f[q].x;
            collide<float, COLL>(fs, l ? rho.y : rho.x, l ? ux.y : ux.x, l ? uy.y : uy.x, l ? uz.y : uz.x, omega_p,
                                 omega_m, ps, activation[l], restriction[l]);
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                if (l) post[q].y = ps[q];
                else post[q].x = ps[q];
            }
        }
        return;
    }
    const P2 u2 = ux * ux + uy * uy + uz * uz;
    const P2 t15 = 1.5f * u2;
    const P2 wr0 = Lat<float>::w0 * rho, wr1 = Lat<float>::w1 * rho, wr2 = Lat<float>::w2 * rho;
    P2 feqv[19];
    // 1 + 3*0 + 4.5*0*0 is exactly 1
    feqv[0] = wr0 * (pv(1.0f) - t15);
#pragma unroll
    for (int q = 1; q < 19; q += 2) {
        const P2 cu = cdot2(q, ux, uy, uz);
        const P2 t3 = 3.0f * cu;
        const P2 t45 = (4.5f * cu) * cu;
        const P2 wr = q <= 6 ? wr1 : wr2;
        feqv[q] = wr * (((pv(1.0f) + t3) + t45) - t15);
        feqv[q + 1] = wr * (((pv(1.0f) - t3) + t45) - t15);
    }
    {
        // TRT; the regularized operators run through collide_pairs
        post[0] = f[0] - omega_p * (f[0] - feqv[0]);
#pragma unroll
        for (int q = 1; q < 19; q += 2) {
            const P2 fp_ = 0.5f * (f[q] + f[q + 1]);
            const P2 fm = 0.5f * (f[q] - f[q + 1]);
            const P2 ep = 0.5f * (feqv[q] + feqv[q + 1]);
            const P2 em = 0.5f * (feqv[q] - feqv[q + 1]);
            const P2 A = omega_p * (fp_ - ep);
            const P2 B = omega_m * (fm - em);
            post[q] = (f[q] - A) - B;
            post[q + 1] = (f[q + 1] - A) + B;
        }
    }
}

// Storage conversions of one population (ld_rt / st_rt on pairs).
template <class S>
__device__ __forceinline__ float ld1(const typename S::T* p, int q) {
    return S::ld_rt(p, q);
}

// ---------------------------------------------------------------------------
// The staged kernel.  CAPTURE 1 also writes the macroscopic fields.
// ---------------------------------------------------------------------------
// Four CTAs per SM (16 consumer warps) for TRT; the heavier operators keep
// their registers at three.
template <class S, int REP_S, int COLL, int CAPTURE>
__global__ void __launch_bounds__(kStreamThreads, 4)
    k_stream(const __grid_constant__ CUtensorMap map, const BulkArgs a, const StreamTiles tl) {
    using T = typename S::T;
    using G = StreamGeom<T>;
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
            mbar_init(empty0 + 8 * s, kTileY);
        }
        mbar_fence_init();
    }
    __syncthreads();
    const Grid& g = a.g;
    if (warp == kTileY) {
        // producer: one thread issues the 19 box loads of each tile
        if (lane != 0) return;
        int issued = 0;
        bool failed = false;
        for (int k = 0;; ++k) {
            const int tile = blockIdx.x + k * gridDim.x;
            if (tile >= tl.ntiles) break;
            const int s = k % NS;
            if (k >= NS && !mbar_wait(empty0 + 8 * s, ((k / NS) + 1) & 1)) {
                atomicOr(&a.state->stream_error, 1u);
                failed = true;
                break;
            }
            const int txi = tile % tl.tiles_x;
            const int rest = tile / tl.tiles_x;
            const int y0 = (rest % tl.tiles_y) * kTileY;
            const int z = rest / tl.tiles_y;
            const int x0 = txi * kTileX;
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
        if (failed) {
            // leave no bulk copy in flight into this CTA's shared memory: wait
            // (bounded) for the last loads issued to complete
            for (int k = issued - NS < 0 ? 0 : issued - NS; k < issued; ++k)
                (void)mbar_wait(full0 + 8 * (k % NS), (k / NS) & 1);
        }
        return;
    }
    // consumers: warp w takes row y0 + w, lane l the cells x0 + l and x0 + l + 32.
    // The mask bytes of the next tile are loaded one tile ahead, so their HBM
    // latency overlaps the current tile's collision.
    const FluidParams& fp = a.fp;
    struct Cells {
        int xa, y, z;
        uint32_t gida;
        bool va, vb;
        uint8_t ma, mb;
    };
    auto locate = [&](int tile, Cells& c) {
        const int txi = tile % tl.tiles_x;
        const int rest = tile / tl.tiles_x;
        c.y = (rest % tl.tiles_y) * kTileY + warp;
        c.z = rest / tl.tiles_y;
        c.xa = txi * kTileX + lane;
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
    if ((int)blockIdx.x < tl.ntiles) locate(blockIdx.x, next);
    for (int k = 0;; ++k) {
        const int tile = blockIdx.x + k * gridDim.x;
        if (tile >= tl.ntiles) break;
        const int s = k % NS;
        const Cells cur = next;
        if (tile + (int)gridDim.x < tl.ntiles) locate(tile + gridDim.x, next);
        const int xa = cur.xa, xb = cur.xa + 32, y = cur.y, z = cur.z;
        const uint32_t gida = cur.gida;
        bool va = cur.va, vb = cur.vb;
        const uint8_t ma = cur.ma, mb = cur.mb;
        if (!mbar_wait(full0 + 8 * s, (k / NS) & 1)) {
            atomicOr(&a.state->stream_error, 2u);
            break;
        }
        const T* row = (const T*)(smem + s * G::stage_bytes) + warp * G::row;
        P2 f[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const int base = REP_S ? 1 : 1 - cx(q);
            const T* p = row + q * (G::plane_bytes / (int)sizeof(T)) + base + lane;
            const int slot = REP_S ? q : opp(q);
            f[q] = make_float2(S::ld_rt(p, slot), S::ld_rt(p + 32, slot));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * s);
        // solid and newly uncovered cells (mask byte set) are left to k_rare
        va = va && ma == 0;
        vb = vb && mb == 0;
        if (!__any_sync(0xffffffffu, va || vb)) continue;
        P2 post[19];
        float activation[2] = {0.0f, 0.0f}, restriction[2] = {0.0f, 0.0f};
        if constexpr (COLL == BFX_COLLISION_RR3 || COLL == BFX_COLLISION_REGULARIZED) {
            collide_pairs<P2, COLL>(f, fp.omega_p, post, activation, restriction);
        } else {
            P2 rho, ux, uy, uz;
            moments2(f, rho, ux, uy, uz);
            collide2<COLL>(f, rho, ux, uy, uz, fp.omega_p, fp.omega_m, post, activation, restriction);
        }
        if (fp.has_sponge) {
            const float spa = va ? sponge_factor(g, fp, xa, y, z) : 0.0f;
            const float spb = vb ? sponge_factor(g, fp, xb, y, z) : 0.0f;
            if (spa > 0.0f || spb > 0.0f) {
                // post + (far - post) * sp, a zero factor leaving the lane unchanged
                const P2 sp = make_float2(spa, spb);
#pragma unroll
                for (int q = 0; q < 19; ++q) {
                    const P2 d = (pv(a.far_eq_f[q]) - post[q]) * sp;
                    post[q] = make_float2(spa > 0.0f ? post[q].x + d.x : post[q].x,
                                          spb > 0.0f ? post[q].y + d.y : post[q].y);
                }
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
            cd.x = cd.x > 1.0e-8f ? cd.x : 1.0e-8f;
            cd.y = cd.y > 1.0e-8f ? cd.y : 1.0e-8f;
            if (va) {
                a.density[gida] = cd.x;
                a.velocity[gida] = make_float4(cmx.x / cd.x, cmy.x / cd.x, cmz.x / cd.x, 0.0f);
            }
            if (vb) {
                a.density[gida + 32] = cd.y;
                a.velocity[gida + 32] = make_float4(cmx.y / cd.y, cmy.y / cd.y, cmz.y / cd.y, 0.0f);
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
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            T* p = REP_S ? (T*)a.plane[opp(q)] + pid : (T*)a.plane[q] + (uint32_t)(pid + (uint32_t)a.doff[q]);
            const int slot = REP_S ? opp(q) : q;
            if (va) S::st_rt(p, slot, post[q].x);
            if (vb) S::st_rt(p + 32, slot, post[q].y);
        }
    }
}

// Resident CTAs per SM of one instantiation; the first call also raises its
// dynamic shared-memory limit (done at simulation creation, outside any capture).
template <class S, int REP, int COLL, int CAPTURE>
static int stream_blocks_per_sm() {
    using G = StreamGeom<typename S::T>;
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaFuncSetAttribute(k_stream<S, REP, COLL, CAPTURE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             G::smem_bytes);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_stream<S, REP, COLL, CAPTURE>, kStreamThreads,
                                                      G::smem_bytes);
        if (per_sm < 1) per_sm = 1;
    }
    return per_sm;
}

template <class S, int REP, int COLL, int C>
static void stream_launch(const GridDesc& gd, const BulkArgs& a, const CUtensorMap& map, int sm_count,
                          cudaStream_t s) {
    using G = StreamGeom<typename S::T>;
    StreamTiles tl;
    tl.tiles_x = (gd.nx + kTileX - 1) / kTileX;
    tl.tiles_y = (gd.ny + kTileY - 1) / kTileY;
    tl.ntiles = tl.tiles_x * tl.tiles_y * gd.nz;
    int blocks = stream_blocks_per_sm<S, REP, COLL, C>() * sm_count;
    if (blocks > tl.ntiles) blocks = tl.ntiles;
    k_stream<S, REP, COLL, C><<<blocks, kStreamThreads, G::smem_bytes, s>>>(map, a, tl);
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
