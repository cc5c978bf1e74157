// Host side of tma.cuh: cuTensorMapEncodeTiled through the runtime's driver
// entry point (no link against libcuda).
#include <atomic>
#include <mutex>
#include "tma.cuh"

namespace cd {
namespace tma {
namespace {

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encoder()
{
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

std::atomic<int> g_persistent{1};

}  // namespace

bool persistent_enabled() { return g_persistent.load(std::memory_order_relaxed) != 0; }
void set_persistent_enabled(bool on) { g_persistent.store(on ? 1 : 0, std::memory_order_relaxed); }

bool encode_image(CUtensorMap *map, const void *base, bool bytes, int C, int W, int H, int B, int box_x, int box_y)
{
    const int e = bytes ? 1 : 4;
    const uint64_t row = (uint64_t)C * W * e;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || row % 16 || (box_x * e) % 16 || box_x > 256 || box_y > 256 ||
        box_x < 1 || box_y < 1)
        return false;
    EncodeTiled enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)C * W, (cuuint64_t)H, (cuuint64_t)B};
    const cuuint64_t strides[2] = {row, row * (uint64_t)H};
    const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1}, es[3] = {1, 1, 1};
    return enc(map, bytes ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
               const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace tma
}  // namespace cd
