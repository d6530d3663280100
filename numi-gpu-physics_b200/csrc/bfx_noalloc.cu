// FP64 fluid mass / momentum reduction that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they need this sum:
// applications whose device memory budget is already reserved by their own
// allocator (for example a framework's caching pool), where a fresh
// allocation fails or fragments that pool, and loops with a fixed time budget
// per iteration, where cudaMalloc / cudaFree would synchronise the device.
// They hold the dense FP32 population field and an output slot already; this
// entry point needs nothing else.
//
// Its scratch (the per-group partial sums) lives in one file-scope device
// array of fixed size, 32,768 groups x 4 doubles = 1 MiB.  Every GPU that loads
// the library keeps that array until the process exits.  All calls share it:
// calls whose kernels overlap on the GPU (different streams, threads or
// processes sharing a context) race on it and must be serialised by the caller.
// Each call writes every partial it later reads, so nothing needs clearing and
// a call never sees a previous call's values.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/bfx.h"

namespace bfx {
void set_global_error(const std::string& message);  // bfx_api.cu
}

namespace {

constexpr int kGroupCells = 256;
constexpr uint32_t kMaxGroups = 32768;  // lattices up to 8,388,608 cells
constexpr int kMaxDevices = 64;

// Partial sums (mass, momentum x, y, z) of each 256-cell group.
static __device__ __align__(256) double g_mass_momentum_scratch[kMaxGroups * 4];

__device__ __forceinline__ int dcx(int q) {
    return (q == 1 || q == 7 || q == 9 || q == 11 || q == 13) ? 1
         : (q == 2 || q == 8 || q == 10 || q == 12 || q == 14) ? -1 : 0;
}
__device__ __forceinline__ int dcy(int q) {
    return (q == 3 || q == 7 || q == 10 || q == 15 || q == 17) ? 1
         : (q == 4 || q == 8 || q == 9 || q == 16 || q == 18) ? -1 : 0;
}
__device__ __forceinline__ int dcz(int q) {
    return (q == 5 || q == 11 || q == 14 || q == 15 || q == 18) ? 1
         : (q == 6 || q == 12 || q == 13 || q == 16 || q == 17) ? -1 : 0;
}

// One block per group of 256 cells, fixed-order tree inside the block
// (the group structure of measureFluidMassMomentum, BirdFlow.metal:4272-4297).
__global__ void __launch_bounds__(kGroupCells) k_group_sums(const float* pops, const uint8_t* mask, uint32_t n,
                                                            double* scratch) {
    __shared__ double sh[4][kGroupCells];
    const uint32_t cell = blockIdx.x * kGroupCells + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (cell < n && (mask == nullptr || (mask[cell] & 0x3F) == 0)) {
        for (int q = 0; q < 19; ++q) {
            const double v = (double)pops[(size_t)q * n + cell];
            acc[0] += v;
            acc[1] += v * dcx(q);
            acc[2] += v * dcy(q);
            acc[3] += v * dcz(q);
        }
    }
    for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int s = kGroupCells / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < 4; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 4; ++k) scratch[4 * blockIdx.x + k] = sh[k][0];
}

// One block: strided fixed-order sums of the group partials, then a tree.
__global__ void __launch_bounds__(256) k_final_sum(const double* scratch, uint32_t groups, double* out) {
    __shared__ double sh[4][256];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (uint32_t i = threadIdx.x; i < groups; i += blockDim.x)
        for (int k = 0; k < 4; ++k) acc[k] += scratch[4 * i + k];
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

std::mutex g_mutex;
double* g_scratch_address[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The array's
// name is only a host-side stand-in, so the address is resolved once per
// device with that device current and cached.  The cached address belongs to
// the context that was current at the first call on the device.
int scratch_address(int device, double** out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_address[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_mass_momentum_scratch);
        if (e != cudaSuccess) {
            bfx::set_global_error(std::string("scratch address lookup failed: ") + cudaGetErrorString(e));
            return BFX_ERR_KERNEL;
        }
        g_scratch_address[device] = (double*)p;
    }
    *out = g_scratch_address[device];
    return BFX_OK;
}

}  // namespace

extern "C" int bfx_fluid_mass_momentum_noalloc(const float* populations, const uint8_t* mask, uint32_t nx,
                                               uint32_t ny, uint32_t nz, double* out) {
    const uint64_t n = (uint64_t)nx * ny * nz;
    if (n == 0) {
        bfx::set_global_error("the lattice is empty");
        return BFX_ERR_INVALID_ARGUMENT;
    }
    const uint64_t groups = (n + kGroupCells - 1) / kGroupCells;
    if (groups > kMaxGroups) {
        bfx::set_global_error("lattice of " + std::to_string(n) + " cells exceeds the no-allocation reduction's " +
                              "fixed scratch (at most " + std::to_string((uint64_t)kMaxGroups * kGroupCells) +
                              " cells); use bfx_fluid_mass_momentum instead");
        return BFX_ERR_CAPACITY;
    }
    if (!populations || !out) {
        bfx::set_global_error("populations and out must be device pointers");
        return BFX_ERR_INVALID_ARGUMENT;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess || device < 0 || device >= kMaxDevices) {
        bfx::set_global_error("no current CUDA device");
        return BFX_ERR_DEVICE_UNAVAILABLE;
    }
    double* scratch = nullptr;
    int rc = scratch_address(device, &scratch);
    if (rc != BFX_OK) return rc;
    k_group_sums<<<(unsigned)groups, kGroupCells>>>(populations, mask, (uint32_t)n, scratch);
    k_final_sum<<<1, 256>>>(scratch, (uint32_t)groups, out);
    e = cudaStreamSynchronize(0);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        bfx::set_global_error(std::string("no-allocation reduction failed: ") + cudaGetErrorString(e));
        return BFX_ERR_KERNEL;
    }
    return BFX_OK;
}
