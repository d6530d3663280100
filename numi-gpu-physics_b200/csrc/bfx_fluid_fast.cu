// Fused-step kernels compiled with FMA contraction (--fmad=true): the 16-bit
// deviation storage formats, whose collision arithmetic is FP32 but which are
// not part of the bit-exact FP32 parity contract, and the opt-in fast_math FP32
// mode (the reference's SimulationConfiguration.fastMath).
#define BFX_VARIANT fast
#define BFX_CONTRACTED 1
#include "bfx_bulk_kernels.cuh"
#include "bfx_stream_kernels.cuh"

namespace bfx {

void launch_stream_fast(int storage, int collision, int rep_s, const GridDesc& g, const BulkArgs* a,
                        const CUtensorMap* map, int sm_count, cudaStream_t s) {
    if (storage == BFX_STORAGE_BF16_DEVIATION) fast::stream_s<StoreBF16Dev>(collision, rep_s, g, a, map, sm_count, s);
    else fast::stream_s<StoreF16Dev>(collision, rep_s, g, a, map, sm_count, s);
}

void launch_rare_fast(int storage, int collision, int rep_s, const BulkArgs& a, cudaStream_t s) {
    if (storage == BFX_STORAGE_BF16_DEVIATION) fast::rare_s<StoreBF16Dev>(a, collision, rep_s, s);
    else fast::rare_s<StoreF16Dev>(a, collision, rep_s, s);
}

void launch_bulk_fast(int storage, int collision, int rep_s, const GridDesc& g, const BulkArgs& a, cudaStream_t s) {
    switch (storage) {
    case BFX_STORAGE_F16_DEVIATION: fast::bulk_s<StoreF16Dev>(a, g, collision, rep_s, s); break;
    case BFX_STORAGE_BF16_DEVIATION: fast::bulk_s<StoreBF16Dev>(a, g, collision, rep_s, s); break;
    default: fast::bulk_s<StoreF32>(a, g, collision, rep_s, s); break;
    }
}

}  // namespace bfx
