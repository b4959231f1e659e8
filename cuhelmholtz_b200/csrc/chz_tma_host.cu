// Host support of the TMA-pipelined pass: tensor-map encoding through the
// driver entry point (no link against the driver library), the device flag
// word and the limit of the kernels' bounded waits, the status check that
// reads the flag word, a self-test of a wait that runs out, and the
// shared-memory limit.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include "chz_internal.h"
#include "chz_tma.cuh"
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

// Bits of WaitFlag (chz_tma.cuh) raised by the waits that ran out.
__device__ int g_flags;

// Limit of every bounded wait of the pipelined kernels, in SM clock cycles
// (about a second at the B200's clocks by default).
constexpr long long kDefaultWaitLimit = 2000000000LL;
constexpr long long kMinWaitLimit = 1000000LL;
std::atomic<long long> g_wait_limit{kDefaultWaitLimit};

// One CTA that waits on an mbarrier nothing ever arrives at: the wait must
// run out after `limit` cycles and raise kFlagSelfTest.  No copy is issued,
// so nothing is in flight when the CTA ends.
__global__ void wait_selftest_kernel(int* flags, long long limit) {
    __shared__ uint64_t bar;
    __shared__ int abort;
    if (threadIdx.x == 0) {
        abort = 0;
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (!mbar_wait(&bar, 0u, &abort, limit)) {
        if (threadIdx.x == 0) atomicOr(flags, kFlagSelfTest);
    }
    __syncthreads();
}
}  // namespace

long long wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }

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

extern "C" long long chz_set_wait_limit(long long cycles) {
    using namespace chz::tma;
    if (cycles <= 0) cycles = kDefaultWaitLimit;
    if (cycles < kMinWaitLimit) cycles = kMinWaitLimit;
    return g_wait_limit.exchange(cycles);
}

extern "C" int chz_stream_status(void* stream) {
    const cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return chz::cuda_fail((int)e, "chz_stream_status");
    const int v = chz_debug_flags(1);
    if (v < 0) return chz::cuda_fail((int)cudaGetLastError(), "chz_stream_status: reading the wait flags");
    if (v != 0)
        return chz::fail(CHZ_ERROR_TIMEOUT,
                         "a kernel wait ran out (flags 0x%x): the results of the work queued since the last "
                         "status check are not valid",
                         v);
    return CHZ_SUCCESS;
}

extern "C" int chz_wait_selftest(long long cycles, void* stream) {
    int* flags = chz::tma::device_flags();
    if (!flags) return chz::cuda_fail((int)cudaGetLastError(), "chz_wait_selftest");
    if (cycles < 1000) cycles = 1000;
    if (cycles > chz::tma::kDefaultWaitLimit) cycles = chz::tma::kDefaultWaitLimit;
    chz::tma::wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(flags, cycles);
    chz::count_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CHZ_SUCCESS : chz::cuda_fail((int)e, "chz_wait_selftest");
}
