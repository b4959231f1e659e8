// Launch of the persistent register-resident kernels (included by the
// per-length translation units chz_fast_m*.cu, which instantiate it).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <type_traits>

#include "chz_fast.cuh"

namespace chz {
namespace fast {

int device_sm_count();

template <typename T, typename TI, typename TO, int M, bool CONTIG, int KIND, int K2>
int launch_one(const void* in, void* out, const PassArgs& a, const LineTables<T>& tb, int nv,
               cudaStream_t stream, const char* label) {
    using CF = Cfg<M>;
    auto kern = fast_pass<T, TI, TO, M, CONTIG, KIND, K2>;
    const size_t smem = SmemLayout<T, M, (K2 >= 0), acc_staged<T, TO, CONTIG>()>::total;
    // per instantiation: opt in to the dynamic shared memory, ask how many CTAs fit
    static std::atomic<int> ctas_per_sm{0};
    int cps = ctas_per_sm.load(std::memory_order_relaxed);
    if (cps == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, kern, kNT, smem);
        if (e != cudaSuccess) return (int)e;
        if (cps < 1) cps = 1;
        ctas_per_sm.store(cps, std::memory_order_relaxed);
    }
    const int ntx = (a.nu + CF::W - 1) / CF::W;
    const long long ntiles = (long long)ntx * nv;
    if (ntiles <= 0) return 0;
    const long long cap = (long long)cps * device_sm_count();
    const int grid = (int)(ntiles < cap ? ntiles : cap);
    trace_begin(stream, label);
    kern<<<grid, kNT, smem, stream>>>(static_cast<const TI*>(in), static_cast<TO*>(out), a, tb, ntx, (int)ntiles);
    count_launch();
    trace_end(stream);
    return (int)cudaGetLastError();
}

// Which (input type, output type, layout, kind) combinations are built: same
// type everywhere; FP64 -> FP32 only for the first (x, forward) pass of the
// FP32 solve; FP32 -> FP64 only for its last (x, inverse) pass.
template <typename T, typename TI, typename TO, bool C, int K, int K2>
constexpr bool wanted() {
    constexpr bool same = std::is_same<TI, T>::value && std::is_same<TO, T>::value;
    constexpr bool fwdk = (K == kR2C || K == kDST1 || K == kDST3 || K == kDCT1 || K == kDCT3);
    constexpr bool invk = (K == kC2R || K == kDST1 || K == kDST2 || K == kDCT1 || K == kDCT2);
    if (same) return true;
    if (std::is_same<TI, double>::value && std::is_same<TO, float>::value) return C && fwdk && K2 < 0;
    if (std::is_same<TI, float>::value && std::is_same<TO, double>::value) return C && invk && K2 < 0;
    return false;
}

template <typename T, typename TI, typename TO, int M>
int launch_fast_kind(bool contig, int kind, int kind2, const void* in, void* out, const PassArgs& a,
                     const LineTables<T>& tb, int nv, cudaStream_t stream, const char* label) {
#define CHZ_ONE(C, K, K2)                                                                   \
    do {                                                                                    \
        if constexpr (wanted<T, TI, TO, C, K, K2>())                                        \
            return launch_one<T, TI, TO, M, C, K, K2>(in, out, a, tb, nv, stream, label);   \
        else                                                                                \
            return (int)cudaErrorInvalidValue;                                              \
    } while (0)
#define CHZ_SINGLE(K)                  \
    case K:                            \
        if (contig) CHZ_ONE(true, K, -1); \
        CHZ_ONE(false, K, -1);
    if (kind2 < 0) {
        switch (kind) {
            CHZ_SINGLE(kDCT1)
            CHZ_SINGLE(kDCT2)
            CHZ_SINGLE(kDCT3)
            CHZ_SINGLE(kDST1)
            CHZ_SINGLE(kDST2)
            CHZ_SINGLE(kDST3)
            CHZ_SINGLE(kR2C)
            CHZ_SINGLE(kC2R)
            default: return (int)cudaErrorInvalidValue;
        }
    }
    if (contig) return (int)cudaErrorInvalidValue;
    // fused forward / divide / inverse pairs of the solver's boundary codes
    if (kind == kR2C && kind2 == kC2R) CHZ_ONE(false, kR2C, kC2R);
    if (kind == kDST1 && kind2 == kDST1) CHZ_ONE(false, kDST1, kDST1);
    if (kind == kDST3 && kind2 == kDST2) CHZ_ONE(false, kDST3, kDST2);
    if (kind == kDCT1 && kind2 == kDCT1) CHZ_ONE(false, kDCT1, kDCT1);
    if (kind == kDCT3 && kind2 == kDCT2) CHZ_ONE(false, kDCT3, kDCT2);
#undef CHZ_SINGLE
#undef CHZ_ONE
    return (int)cudaErrorInvalidValue;
}

// One group of a batched pass (FP64): the members' tiles are split into
// contiguous ranges over as many CTAs as fit the device.
template <int M, bool CONTIG, int KIND, int K2>
int launch_batch_one(const FastBatchArgs& g, const LineTables<double>& tb, cudaStream_t stream) {
    auto kern = fast_batch_pass<M, CONTIG, KIND, K2>;
    constexpr size_t smem = batch_smem_bytes<M, (K2 >= 0)>();
    static std::atomic<int> ctas_per_sm{0};
    int cps = ctas_per_sm.load(std::memory_order_relaxed);
    if (cps == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, kern, kNT, smem);
        if (e != cudaSuccess) return (int)e;
        if (cps < 1) cps = 1;
        ctas_per_sm.store(cps, std::memory_order_relaxed);
    }
    if (g.ntiles <= 0) return 0;
    const long long cap = (long long)cps * device_sm_count();
    const int grid = (int)(g.ntiles < cap ? g.ntiles : cap);
    kern<<<grid, kNT, smem, stream>>>(g, tb);
    return (int)cudaGetLastError();
}

template <int M>
int launch_fast_batch_kind(bool contig, int kind, int kind2, const FastBatchArgs& g, const LineTables<double>& tb,
                           cudaStream_t stream) {
#define CHZ_SINGLE(K)                                                        \
    case K:                                                                  \
        if (contig) return launch_batch_one<M, true, K, -1>(g, tb, stream);  \
        return launch_batch_one<M, false, K, -1>(g, tb, stream);
    if (kind2 < 0) {
        switch (kind) {
            CHZ_SINGLE(kDCT1)
            CHZ_SINGLE(kDCT2)
            CHZ_SINGLE(kDCT3)
            CHZ_SINGLE(kDST1)
            CHZ_SINGLE(kDST2)
            CHZ_SINGLE(kDST3)
            CHZ_SINGLE(kR2C)
            CHZ_SINGLE(kC2R)
            default: return (int)cudaErrorInvalidValue;
        }
    }
#undef CHZ_SINGLE
    if (contig) return (int)cudaErrorInvalidValue;
    if (kind == kR2C && kind2 == kC2R) return launch_batch_one<M, false, kR2C, kC2R>(g, tb, stream);
    if (kind == kDST1 && kind2 == kDST1) return launch_batch_one<M, false, kDST1, kDST1>(g, tb, stream);
    if (kind == kDST3 && kind2 == kDST2) return launch_batch_one<M, false, kDST3, kDST2>(g, tb, stream);
    if (kind == kDCT1 && kind2 == kDCT1) return launch_batch_one<M, false, kDCT1, kDCT1>(g, tb, stream);
    if (kind == kDCT3 && kind2 == kDCT2) return launch_batch_one<M, false, kDCT3, kDCT2>(g, tb, stream);
    return (int)cudaErrorInvalidValue;
}

}  // namespace fast
}  // namespace chz
