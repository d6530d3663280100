// Coupled momentum ledger: the per-step source terms of the fluid's
// linear-momentum balance (measureFluidMassMomentumChange and
// captureExternalFluidSources, BF.metal:4322-4552), reduced in FP64.
//
// The populations are updated in place, so the balance is taken in two passes
// around a step:
//   in   after the geometry of the step is built, before the halo fill and the
//        cut links write anything: the momentum of the cells that were fluid,
//        the open far-field faces (what the halo will bring in, what the face
//        cells send out) and the persistent cut-link exchange, all from the
//        pre-step populations;
//   out  after the step: the momentum of the cells that are fluid, and the
//        sponge impulse recovered from f_out = (1 - s) f_post + s f_far.
// Each pass writes one row of partial sums per block (fixed grid, fixed
// order); the host adds the rows.
#include "bfx_bulk.cuh"
#include "bfx_internal.h"

namespace bfx {
namespace {

constexpr int kLedgerIn = 16;   // mass, momentum (old fluid) | far field (4) | link exchange (4) | counts (4)
constexpr int kLedgerOut = 9;   // mass, momentum (new fluid) | sponge (4) | sponge cells

template <int K>
__device__ __forceinline__ void ledger_block_sum(double (&v)[K], double* out) {
    __shared__ double sh[K][256];
    for (int k = 0; k < K; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < K; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < K; ++k) out[K * blockIdx.x + k] = sh[k][0];
}

// The value the halo fill writes for the population cell b pulls from the
// outside cell h = b - c_q across a non-periodic face (k_halo's rules).
template <class S>
__device__ __forceinline__ double face_incoming(const BulkArgs& a, const uint8_t* mask, int rep_s, int q, int bx,
                                                int by, int bz, int hx, int hy, int hz) {
    using R = typename S::R;
    const Grid& g = a.g;
    const FluidParams& fp = a.fp;
    const int f = exit_face(g, hx, hy, hz);
    const int bc = fp.face_bc[f];
    if (bc == BFX_BC_OUTFLOW) {
        const int ax = f >> 1;
        const int sgn = (f & 1) ? 1 : -1;
        int tx = bx - (ax == 0 ? sgn : 0) - cx(q), ty = by - (ax == 1 ? sgn : 0) - cy(q),
            tz = bz - (ax == 2 ? sgn : 0) - cz(q);
        if (wrap(g, tx, ty, tz) && (mask == nullptr || (mask[flat(g, tx, ty, tz)] & kPartMask) == 0))
            return (double)canon_load<S>((const typename S::T*)a.pops, g, rep_s, q, tx, ty, tz);
    } else if (bc == BFX_BC_VELOCITY) {
        return (double)feq_rt<R>(q, (R)fp.far[3], (R)fp.face_u[f][0], (R)fp.face_u[f][1], (R)fp.face_u[f][2]);
    }
    return sizeof(R) == 8 ? a.far_eq_d[q] : (double)a.far_eq_f[q];
}

template <class S>
__global__ void __launch_bounds__(256) k_ledger_in(const BulkArgs a, const uint8_t* mprev, const uint8_t* mnext,
                                                   int rep_s, double* partials) {
    using R = typename S::R;
    const Grid& g = a.g;
    const FluidParams& fp = a.fp;
    const typename S::T* A = (const typename S::T*)a.pops;
    double acc[kLedgerIn] = {};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < g.n; gid += stride) {
        int x, y, z;
        unflat(g, gid, x, y, z);
        const bool was_solid = mprev && (mprev[gid] & kPartMask);
        const bool is_solid = mnext && (mnext[gid] & kPartMask);
        if (was_solid != is_solid) acc[15] += 1.0;
        if (!was_solid) {
            for (int q = 0; q < 19; ++q) {
                const double v = (double)canon_load<S>(A, g, rep_s, q, x, y, z);
                acc[0] += v;
                acc[1] += v * cx(q);
                acc[2] += v * cy(q);
                acc[3] += v * cz(q);
            }
        }
        if (is_solid) continue;
        const bool persistent_target = !was_solid;
        double mwd = (double)fp.far[3];
        if (fp.local_density) {
            mwd = 0.0;
            for (int q = 0; q < 19; ++q) mwd += (double)canon_load<S>(A, g, rep_s, q, x, y, z);
        }
        for (int q = 1; q < 19; ++q) {
            int sx = x - cx(q), sy = y - cy(q), sz = z - cz(q);
            if (!inside(g, sx, sy, sz)) {
                int wx = sx, wy = sy, wz = sz;
                if (!wrap(g, wx, wy, wz)) {
                    // open face: in from the halo, out the population f*_{opp q}(x) that leaves
                    const double in = face_incoming<S>(a, mnext, rep_s, q, x, y, z, sx, sy, sz);
                    const double out = (double)canon_load<S>(A, g, rep_s, opp(q), x, y, z);
                    acc[4] += in - out;
                    acc[5] += (in + out) * cx(q);
                    acc[6] += (in + out) * cy(q);
                    acc[7] += (in + out) * cz(q);
                    acc[12] += 1.0;
                    continue;
                }
                sx = wx;
                sy = wy;
                sz = wz;
            }
            const int64_t src = flat(g, sx, sy, sz);
            const bool persistent_solid = mprev && mnext && (mprev[src] & kPartMask) && (mnext[src] & kPartMask);
            if (persistent_target && persistent_solid) {
                // halfway moving-wall reflection (the reference's ledger rule)
                const double reflected = (double)canon_load<S>(A, g, rep_s, opp(q), x, y, z);
                const float4 w = a.wall[src];
                const double wq = q <= 6 ? (double)Lat<float>::w1 : (double)Lat<float>::w2;
                const double wc = 2.0 * wq * mwd * ((double)cx(q) * w.x + (double)cy(q) * w.y + (double)cz(q) * w.z) /
                                  (double)Lat<float>::cs2;
                const double incoming = reflected + wc;
                acc[8] += incoming - reflected;
                acc[9] += (incoming + reflected) * cx(q);
                acc[10] += (incoming + reflected) * cy(q);
                acc[11] += (incoming + reflected) * cz(q);
                acc[14] += 1.0;
            }
        }
    }
    ledger_block_sum<kLedgerIn>(acc, partials);
}

template <class S>
__global__ void __launch_bounds__(256) k_ledger_out(const BulkArgs a, const uint8_t* mnext, int rep_s,
                                                    double* partials) {
    using R = typename S::R;
    const Grid& g = a.g;
    const FluidParams& fp = a.fp;
    const typename S::T* A = (const typename S::T*)a.pops;
    double acc[kLedgerOut] = {};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gid < g.n; gid += stride) {
        if (mnext && (mnext[gid] & kPartMask)) continue;
        int x, y, z;
        unflat(g, gid, x, y, z);
        R f[19];
        for (int q = 0; q < 19; ++q) {
            f[q] = canon_load<S>(A, g, rep_s, q, x, y, z);
            const double v = (double)f[q];
            acc[0] += v;
            acc[1] += v * cx(q);
            acc[2] += v * cy(q);
            acc[3] += v * cz(q);
        }
        if (!fp.has_sponge) continue;
        const float sp = sponge_factor(g, fp, x, y, z);
        if (!(sp > 0.0f)) continue;
        const double inv = 1.0 / fmax(1.0 - (double)sp, 1.0e-7);
        for (int q = 0; q < 19; ++q) {
            const double far = sizeof(R) == 8 ? a.far_eq_d[q] : (double)a.far_eq_f[q];
            const double d = (double)sp * (far - (double)f[q]) * inv;
            acc[4] += d;
            acc[5] += d * cx(q);
            acc[6] += d * cy(q);
            acc[7] += d * cz(q);
        }
        acc[8] += 1.0;
    }
    ledger_block_sum<kLedgerOut>(acc, partials);
}

template <class S>
void ledger_in_s(const BulkArgs& a, const uint8_t* mprev, const uint8_t* mnext, int rep_s, double* partials,
                 int blocks, cudaStream_t s) {
    k_ledger_in<S><<<blocks, 256, 0, s>>>(a, mprev, mnext, rep_s, partials);
}
template <class S>
void ledger_out_s(const BulkArgs& a, const uint8_t* mnext, int rep_s, double* partials, int blocks, cudaStream_t s) {
    k_ledger_out<S><<<blocks, 256, 0, s>>>(a, mnext, rep_s, partials);
}

}  // namespace

#define BFX_LEDGER_DISPATCH(storage, FN, ...)                              \
    switch (storage) {                                                     \
    case BFX_STORAGE_F16_DEVIATION: FN<StoreF16Dev>(__VA_ARGS__); break;   \
    case BFX_STORAGE_BF16_DEVIATION: FN<StoreBF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_F64: FN<StoreF64>(__VA_ARGS__); break;                \
    default: FN<StoreF32>(__VA_ARGS__); break;                             \
    }

void launch_ledger_in(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                      const uint8_t* mprev, const uint8_t* mnext, double* partials, int blocks, cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    BFX_LEDGER_DISPATCH(storage, ledger_in_s, a, mprev, mnext, rep_s, partials, blocks, s);
}

void launch_ledger_out(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                       const uint8_t* mnext, double* partials, int blocks, cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    BFX_LEDGER_DISPATCH(storage, ledger_out_s, a, mnext, rep_s, partials, blocks, s);
}

}  // namespace bfx
