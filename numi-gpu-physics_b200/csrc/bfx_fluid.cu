// Fused D3Q19 stream + collide on the in-place AA population layout.
//
// One thread per lattice cell, one launch per step.  The kernel restates the
// fluid, solid and newly-uncovered branches of the reference's stepFluidTRT
// (Sources/BirdFlowMetal/Metal/BirdFlow.metal:2507-3236) in the same FP32
// operation order.  Two kinds of work happen before it: the halo fill writes
// the values boundary cells pull from outside the lattice (periodic images,
// far field, inlet, zero-gradient outflow), and the link kernels
// (bfx_geometry.cu) write the moving-wall bounce-back populations.  Both write
// into the slots this kernel reads, so every fluid cell runs the same
// branch-free path: 19 loads, moments, collision, optional sponge, 19 stores
// (152 B per cell in FP32, 76 B in the 16-bit formats).
#define BFX_VARIANT exact
#include "bfx_bulk_kernels.cuh"
#include "bfx_stream.cuh"

namespace bfx {



// ---------------------------------------------------------------------------
// Halo fill.  For every halo cell h and direction q whose target h + c_q is a
// real cell b, write the population b pulls from outside the lattice into the
// slot the next step reads (rep E: A[opp q][h]; rep S: A[q][b]):
//   periodic image of h is a real cell w  ->  f*_q(w)
//   far-field face                         ->  equilibrium(far density, far velocity)
//   velocity face                          ->  equilibrium(far density, face velocity)
//   zero-gradient outflow face             ->  f*_q(b - n - c_q), what the interior
//                                              neighbour of b receives (far field if
//                                              that cell is solid or outside)
// The reference has only the far-field rule and an all-axes periodic flag
// (BF.metal:2696-2725).
// ---------------------------------------------------------------------------

template <class S>
__global__ void __launch_bounds__(128) k_halo(const BulkArgs a, int rep_s, int64_t halo_cells) {
    using T = typename S::T;
    using R = typename S::R;
    const Grid& g = a.g;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= halo_cells) return;
    int hx, hy, hz;
    if (!padded_shell_cell(g, t, hx, hy, hz)) return;
    hx -= 1;
    hy -= 1;
    hz -= 1;
    T* A = (T*)a.pops;
    const FluidParams& fp = a.fp;
    // Two passes: every value is loaded before any is stored, so the loads of
    // one cell overlap.  No load of this launch reads a stored slot: rep E
    // loads A[opp q][w] and stores A[opp q][h], rep S loads A[q][w + c_q] and
    // stores A[q][h + c_q], with w always a real cell and h a halo cell.
    R vals[19];
    uint32_t live = 0;
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        const int bx = hx + cx(q), by = hy + cy(q), bz = hz + cz(q);
        if (!inside(g, bx, by, bz)) continue;
        live |= 1u << q;
        int wx = hx, wy = hy, wz = hz;
        R val;
        if (wrap(g, wx, wy, wz)) {
            val = canon_load<S>(A, g, rep_s, q, wx, wy, wz);
        } else {
            const int f = exit_face(g, wx, wy, wz);
            const int bc = fp.face_bc[f];
            float ux = fp.far[0], uy = fp.far[1], uz = fp.far[2];
            bool done = false;
            val = R(0);
            if (bc == BFX_BC_OUTFLOW) {
                const int ax = f >> 1;
                const int sgn = (f & 1) ? 1 : -1;
                int tx = bx - (ax == 0 ? sgn : 0) - cx(q), ty = by - (ax == 1 ? sgn : 0) - cy(q),
                    tz = bz - (ax == 2 ? sgn : 0) - cz(q);
                if (wrap(g, tx, ty, tz) && (a.mask == nullptr || (a.mask[flat(g, tx, ty, tz)] & kPartMask) == 0)) {
                    val = canon_load<S>(A, g, rep_s, q, tx, ty, tz);
                    done = true;
                }
            } else if (bc == BFX_BC_VELOCITY) {
                ux = fp.face_u[f][0];
                uy = fp.face_u[f][1];
                uz = fp.face_u[f][2];
            }
            if (!done) {
                // far-field faces take the precomputed equilibrium (same expression, evaluated on the host)
                if (bc == BFX_BC_VELOCITY) val = feq_rt<R>(q, (R)fp.far[3], (R)ux, (R)uy, (R)uz);
                else val = sizeof(R) == 8 ? (R)a.far_eq_d[q] : (R)a.far_eq_f[q];
            }
        }
        vals[q] = val;
    }
#pragma unroll
    for (int q = 1; q < 19; ++q) {
        if (!(live & (1u << q))) continue;
        if (rep_s) S::st_rt(A + (int64_t)q * g.pn + pflat(g, hx + cx(q), hy + cy(q), hz + cz(q)), q, vals[q]);
        else S::st_rt(A + (int64_t)opp(q) * g.pn + pflat(g, hx, hy, hz), opp(q), vals[q]);
    }
}

// The values k_halo writes across a far-field or velocity face depend only on
// the face and the direction.  When both x faces are of those kinds the
// staged kernel takes their values from this table instead of the x-halo
// slots, whose fill (one scattered store per row and direction) it skips:
// out[19 f + q] = the stored value of direction q across face f (0: -x,
// 1: +x), read back as the staged kernel reads a population (scaled deviation).
template <class S>
__global__ void k_halo_values(const BulkArgs a, float* out) {
    using T = typename S::T;
    using R = typename S::R;
    const int t = threadIdx.x;
    if (t >= 2 * 19) return;
    const int f = t / 19, q = t % 19;
    const FluidParams& fp = a.fp;
    R val = sizeof(R) == 8 ? (R)a.far_eq_d[q] : (R)a.far_eq_f[q];
    if (fp.face_bc[f] == BFX_BC_VELOCITY)
        val = feq_rt<R>(q, (R)fp.far[3], (R)fp.face_u[f][0], (R)fp.face_u[f][1], (R)fp.face_u[f][2]);
    T stored;
    S::st_rt(&stored, q, val);
    out[t] = S::ld_dev(&stored);
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
        canon_store<S>(A, g, 0, q, x, y, z, (R)v);
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
        out[(int64_t)q * g.n + gid] = (float)canon_load<S>((const typename S::T*)a.pops, g, rep_s, q, x, y, z);
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
        canon_store<S>((typename S::T*)a.pops, g, rep_s, q, x, y, z, (typename S::R)in[(int64_t)q * g.n + gid]);
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
        R v = canon_load<S>((const typename S::T*)a.pops, g, rep_s, q, x, y, z);
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
            double v = (double)canon_load<S>((const typename S::T*)a.pops, g, rep_s, q, x, y, z);
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

Grid device_grid(const GridDesc& gd) {
    Grid g;
    g.nx = gd.nx;
    g.ny = gd.ny;
    g.nz = gd.nz;
    g.per_x = gd.per_x;
    g.per_y = gd.per_y;
    g.per_z = gd.per_z;
    g.n = gd.n;
    g.nxy = gd.nxy;
    g.px = gd.px;
    g.py = gd.ny + 2;
    g.pz = gd.nz + 2;
    g.pxy = (int64_t)g.px * g.py;
    g.pn = g.pxy * g.pz;
    return g;
}

BulkArgs make_bulk_args(const GridDesc& gd, const FluidParams& fp, const FluidBuffers& b, int capture,
                        int storage) {
    BulkArgs a;
    a.box[0] = a.box[1] = a.box[2] = 0;
    a.g = device_grid(gd);
    for (int q = 0; q < 19; ++q) {
        a.plane[q] = (char*)b.pops + (size_t)q * (size_t)a.g.pn * elem_bytes(storage);
        a.doff[q] = (int32_t)((int64_t)cx(q) + (int64_t)a.g.px * cy(q) + a.g.pxy * cz(q));
        a.far_eq_f[q] = host_feq<float>(q, fp.far[3], fp.far[0], fp.far[1], fp.far[2]);
        a.far_eq_d[q] = host_feq<double>(q, (double)fp.far[3], (double)fp.far[0], (double)fp.far[1], (double)fp.far[2]);
        const double scale = storage == BFX_STORAGE_F16_DEVIATION ? (double)StoreF16Dev::kDevScale : 1.0;
        a.far_dev[q] = (float)((a.far_eq_d[q] - wq<double>(q)) * scale);
    }
    a.face_values = b.face_dev ? 1 : 0;
    for (int f = 0; f < 2; ++f)
        for (int q = 0; q < 19; ++q) a.face_dev[f][q] = b.face_dev ? b.face_dev[19 * f + q] : 0.0f;
    a.pops = b.pops;
    a.mask = b.mask;
    a.wall = b.wall;
    a.density = b.density;
    a.velocity = b.velocity;
    a.state = b.state;
    a.tape = b.tape;
    a.fp = fp;
    a.capture = capture;
    return a;
}

void cell_launch_shape(const GridDesc& g, dim3& grid, dim3& block) {
    int bx = g.nx >= 128 ? 128 : ((g.nx + 31) / 32) * 32;
    int by = 256 / bx;
    block = dim3(bx, by, 1);
    grid = dim3((g.nx + bx - 1) / bx, (g.ny + by - 1) / by, g.nz);
}

#define BFX_DISPATCH_STORAGE(storage, FN, ...)                             \
    switch (storage) {                                                     \
    case BFX_STORAGE_F16_DEVIATION: FN<StoreF16Dev>(__VA_ARGS__); break;   \
    case BFX_STORAGE_BF16_DEVIATION: FN<StoreBF16Dev>(__VA_ARGS__); break; \
    case BFX_STORAGE_F64: FN<StoreF64>(__VA_ARGS__); break;                \
    default: FN<StoreF32>(__VA_ARGS__); break;                             \
    }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

bool encode_population_map(CUtensorMap* map, void* pops, int storage, int collision, int64_t px, int64_t py,
                           int64_t pz) {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || p == nullptr)
            return false;
        fn = (EncodeTiledFn)p;
    }
    CUtensorMapDataType dt;
    switch (storage) {
    case BFX_STORAGE_F16_DEVIATION: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; break;
    case BFX_STORAGE_BF16_DEVIATION: dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; break;
    default: return false;
    }
    // the box is the tile shape of the operator's staged kernel (both formats are 2 bytes)
    const size_t e = 2;
    const bool trt = collision == BFX_COLLISION_TRT;
    const cuuint32_t row = trt ? StreamGeom<__half, BFX_COLLISION_TRT>::row : StreamGeom<__half, BFX_COLLISION_RR3>::row;
    const cuuint32_t rows = trt ? StreamShape<BFX_COLLISION_TRT>::Y : StreamShape<BFX_COLLISION_RR3>::Y;
    static_assert(StreamGeom<__half, BFX_COLLISION_RR3>::row == StreamGeom<__half, BFX_COLLISION_REGULARIZED>::row &&
                      StreamShape<BFX_COLLISION_RR3>::Y == StreamShape<BFX_COLLISION_REGULARIZED>::Y,
                  "the regularized operators share one tile shape");
    const cuuint64_t dims[4] = {(cuuint64_t)px, (cuuint64_t)py, (cuuint64_t)pz, 19};
    const cuuint64_t strides[3] = {(cuuint64_t)(px * e), (cuuint64_t)(px * py * e), (cuuint64_t)(px * py * pz * e)};
    const cuuint32_t box[4] = {row, rows, 1, 1};
    const cuuint32_t elem_strides[4] = {1, 1, 1, 1};
    return fn(map, dt, 4, pops, dims, strides, box, elem_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

bool staged_collision(int collision) {
    return collision == BFX_COLLISION_TRT || collision == BFX_COLLISION_RR3 ||
           collision == BFX_COLLISION_REGULARIZED;
}

void prepare_stream(int storage, int collision) {
    const GridDesc g = {};
    for (int rep = 0; rep < 2; ++rep) launch_stream_fast(storage, collision, rep, g, nullptr, nullptr, 0, nullptr);
}

static bool use_staged(int storage, int collision, int capture, bool tma_ok) {
    const bool sixteen = storage == BFX_STORAGE_F16_DEVIATION || storage == BFX_STORAGE_BF16_DEVIATION;
    return tma_ok && sixteen && staged_collision(collision) && capture != 2;
}
bool bulk_staged(int storage, int collision, int capture, bool tma_ok) {
    return use_staged(storage, collision, capture, tma_ok);
}

int launch_bulk_count(int storage, int collision, int capture, bool tma_ok, bool geometry) {
    return use_staged(storage, collision, capture, tma_ok) && geometry ? 2 : 1;
}

void launch_bulk(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, int capture, const int* box, cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, capture, storage);
    if (box) {
        a.box[0] = box[0];
        a.box[1] = box[1];
        a.box[2] = box[2];
    }
    const bool contracted = storage == BFX_STORAGE_F16_DEVIATION || storage == BFX_STORAGE_BF16_DEVIATION ||
                            (storage == BFX_STORAGE_F32 && fp.fast_math);
    // 16-bit TRT / regularized / RR3: the TMA-staged kernel, measured faster
    // there (16-bit loads leave k_bulk latency-bound; the packed pair
    // arithmetic halves the regularized operators' issue time), with the
    // geometry box's solid and uncovered cells in a second launch (inlined,
    // their path cost the staged kernel registers).  FP32 and FP64 keep k_bulk
    // (bit-identical scalar arithmetic), which takes those cells inline.
    if (use_staged(storage, collision, capture, b.tmap != nullptr)) {
        launch_stream_fast(storage, collision, rep_s, g, &a, (const CUtensorMap*)b.tmap, b.sm_count, s);
        if (box && a.mask) launch_rare_fast(storage, collision, rep_s, a, s);
        return;
    }
    if (contracted) {
        launch_bulk_fast(storage, collision, rep_s, g, a, s);
    } else if (storage == BFX_STORAGE_F64) {
        exact::bulk_s<StoreF64>(a, g, collision, rep_s, s);
    } else {
        exact::bulk_s<StoreF32>(a, g, collision, rep_s, s);
    }
}

// The staged path of launch_bulk in its two launches, so that other work can
// be queued between them: the geometry box's solid and newly uncovered cells
// (k_rare), then the fluid cells (k_stream).  Every population slot is read
// and written by one cell only in a step, and the two launches cover disjoint
// cells, so their order does not change the result.
void launch_bulk_rare(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                      const FluidBuffers& b, const int* box, cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    for (int k = 0; k < 3; ++k) a.box[k] = box[k];
    launch_rare_fast(storage, collision, rep_s, a, s);
}
void launch_bulk_stream(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                        const FluidBuffers& b, const int* box, cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    for (int k = 0; k < 3; ++k) a.box[k] = box[k];
    launch_stream_fast(storage, collision, rep_s, g, &a, (const CUtensorMap*)b.tmap, b.sm_count, s);
}

template <class S>
static void halo_s(const BulkArgs& a, int rep_s, cudaStream_t s) {
    const int64_t halo = a.g.pn - a.g.n;
    k_halo<S><<<(unsigned)((halo + 127) / 128), 128, 0, s>>>(a, rep_s, halo);
}
// The z planes and y rows of the shell come first in padded_shell_cell's
// order, the x columns last: the first 2 (fz + fy) cells are the y / z faces.
template <class S>
static void halo_yz_s(const BulkArgs& a, int rep_s, cudaStream_t s) {
    const int64_t yz = 2 * ((int64_t)a.g.px * a.g.py + (int64_t)a.g.px * (a.g.pz - 2));
    k_halo<S><<<(unsigned)((yz + 127) / 128), 128, 0, s>>>(a, rep_s, yz);
}
void launch_halo_values(int storage, const GridDesc& g, const FluidParams& fp, float* out, cudaStream_t s) {
    FluidBuffers b = {};
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    if (storage == BFX_STORAGE_F16_DEVIATION) k_halo_values<StoreF16Dev><<<1, 128, 0, s>>>(a, out);
    else if (storage == BFX_STORAGE_BF16_DEVIATION) k_halo_values<StoreBF16Dev><<<1, 128, 0, s>>>(a, out);
}

void launch_halo_yz(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                    cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    BFX_DISPATCH_STORAGE(storage, halo_yz_s, a, rep_s, s);
}

void launch_halo(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                 cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    BFX_DISPATCH_STORAGE(storage, halo_s, a, rep_s, s);
}

template <class S>
static void init_s(const BulkArgs& a, const GridDesc& g, int kind, float amplitude, cudaStream_t s) {
    dim3 grid, block;
    cell_launch_shape(g, grid, block);
    k_init<S><<<grid, block, 0, s>>>(a, kind, amplitude);
}
void launch_init(int storage, int init_kind, float amplitude, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, cudaStream_t s) {
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
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
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
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
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
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
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
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
    BulkArgs a = make_bulk_args(g, fp, b, 0, storage);
    BFX_DISPATCH_STORAGE(storage, mass_s, a, rep_s, partials, blocks, result, s);
}

}  // namespace bfx
