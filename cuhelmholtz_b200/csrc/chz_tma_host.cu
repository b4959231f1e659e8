// Host support of the TMA-pipelined pass: tensor-map encoding through the
// driver entry point (no link against the driver library), the device flag
// word of the kernels' bounded waits, and the shared-memory limit.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace tma {

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encoder() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Bit 0: the producer gave up waiting for a finished tile; bit 1: a compute
// thread gave up waiting for a tile load; bit 2: misaligned shared memory.
__device__ int g_flags;
}  // namespace

bool encode_map(CUtensorMap* map, bool is_double, const void* base, const unsigned long long dims[3],
                const unsigned long long strides[2], const unsigned box[3]) {
    EncodeTiledFn fn = encoder();
    if (!fn) return false;
    for (int i = 0; i < 3; ++i)
        if (dims[i] < 1 || dims[i] > (1ull << 32) || box[i] < 1 || box[i] > 256) return false;
    for (int i = 0; i < 2; ++i)
        if (strides[i] % 16 || strides[i] >= (1ull << 40)) return false;
    const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
    const cuuint64_t s[2] = {strides[0], strides[1]};
    const cuuint32_t b[3] = {box[0], box[1], box[2]};
    const cuuint32_t e[3] = {1, 1, 1};
    const CUresult r = fn(map, is_double ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                          const_cast<void*>(base), d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 3-D FP64 map with the 128-byte swizzle (the contiguous-pass tiles).
bool encode_map_swz(CUtensorMap* map, const void* base, const unsigned long long dims[3],
                    const unsigned long long strides[2], const unsigned box[3]) {
    EncodeTiledFn fn = encoder();
    if (!fn) return false;
    for (int i = 0; i < 3; ++i)
        if (dims[i] < 1 || dims[i] > (1ull << 32) || box[i] < 1 || box[i] > 256) return false;
    for (int i = 0; i < 2; ++i)
        if (strides[i] % 16 || strides[i] >= (1ull << 40)) return false;
    if (box[0] * 8 != 128 || (reinterpret_cast<uintptr_t>(base) & 15)) return false;
    const cuuint64_t d[3] = {dims[0], dims[1], dims[2]};
    const cuuint64_t s[2] = {strides[0], strides[1]};
    const cuuint32_t b[3] = {box[0], box[1], box[2]};
    const cuuint32_t e[3] = {1, 1, 1};
    const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), d, s, b, e,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

int* device_flags() {
    static std::atomic<int*> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    int* p = cached[dev].load(std::memory_order_acquire);
    if (!p) {
        void* q = nullptr;
        if (cudaGetSymbolAddress(&q, g_flags) != cudaSuccess) return nullptr;
        p = static_cast<int*>(q);
        cached[dev].store(p, std::memory_order_release);
    }
    return p;
}

int max_optin_smem() {
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) v = 0;
        if (v > 0) cached[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

}  // namespace tma
}  // namespace chz

extern "C" int chz_debug_flags(int reset) {
    int* p = chz::tma::device_flags();
    if (!p) return -1;
    int v = 0;
    if (cudaMemcpy(&v, p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (reset) {
        const int z = 0;
        if (cudaMemcpy(p, &z, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    }
    return v;
}
