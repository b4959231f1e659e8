// Host side of the TMA-pipelined contiguous pass (included by the per-length
// translation units chz_xtma_m*.cu, which instantiate it).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "chz_xtma.cuh"

namespace chz {
namespace fast {
int device_sm_count();
}
namespace tma {
bool encode_map_swz(CUtensorMap* map, const void* base, const unsigned long long dims[3],
                    const unsigned long long strides[2], const unsigned box[3]);
int* device_flags();
long long wait_limit();
int max_optin_smem();
}  // namespace tma
namespace xtma {

// True when rows of `p` with pitch `pitch` values (FP64) start on 16-byte
// boundaries (the copy engine's requirement).
inline bool rows_aligned(const void* p, long long pitch, long long plane) {
    return !(reinterpret_cast<uintptr_t>(p) & 15) && (pitch * 8) % 16 == 0 && (plane * 8) % 16 == 0;
}

template <int M, int KIND, bool LD, bool ST>
int launch_one(const double* in, double* out, const PassArgs& a, const LineTables<double>& tb, int nv,
               cudaStream_t stream, const char* label) {
    using CF = XCfg<M>;
    using SL = XSmem<double, M>;
    constexpr int W = CF::W, N = CF::N;
    constexpr int LO = fast::InWin<KIND, N>::lo, HI = fast::InWin<KIND, N>::hi;
    if ((long long)SL::total > (long long)tma::max_optin_smem()) return -1;
    XGeom g{};
    CUtensorMap ldmap, stmap;
    std::memset(&ldmap, 0, sizeof(ldmap));
    std::memset(&stmap, 0, sizeof(stmap));
    const unsigned box[3] = {16u, 16u, 1u};
    if (LD) {
        g.ld_blk0 = LO >> 4;
        g.ld_nblk = (HI >> 4) - g.ld_blk0 + 1;
        const unsigned long long dims[3] = {(unsigned long long)(a.ld_hi + 1), (unsigned long long)(a.u0 + a.nu),
                                            (unsigned long long)(a.v0 + nv)};
        const unsigned long long strides[2] = {(unsigned long long)(a.in_su * 8), (unsigned long long)(a.in_sv * 8)};
        if (!tma::encode_map_swz(&ldmap, in, dims, strides, box)) return -1;
    }
    if (ST) {
        g.st_blk0 = a.st_lo >> 4;
        g.st_nblk = (a.st_hi >> 4) - g.st_blk0 + 1;
        const unsigned long long dims[3] = {(unsigned long long)(a.st_hi + 1), (unsigned long long)(a.u0 + a.nu),
                                            (unsigned long long)(a.v0 + nv)};
        const unsigned long long strides[2] = {(unsigned long long)(a.out_su * 8),
                                               (unsigned long long)(a.out_sv * 8)};
        if (!tma::encode_map_swz(&stmap, out, dims, strides, box)) return -1;
    }
    int* flags = tma::device_flags();
    if (!flags) return -1;
    auto kern = xtma_pass<double, M, KIND, LD, ST>;
    constexpr int threads = CF::NT + 32;
    static std::atomic<int> cps_cached{0};
    int cps = cps_cached.load(std::memory_order_relaxed);
    if (cps == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SL::total);
        if (e != cudaSuccess) return (int)e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, kern, threads, SL::total);
        if (e != cudaSuccess) return (int)e;
        if (cps < 1) return -1;
        cps_cached.store(cps, std::memory_order_relaxed);
    }
    const int ntx = (a.nu + W - 1) / W;
    const long long ntiles = (long long)ntx * nv;
    if (ntiles <= 0) return 0;
    if (ntiles > 0x7fffffffLL) return -1;
    const long long cap = (long long)cps * fast::device_sm_count();
    const int grid = (int)std::min(ntiles, cap);
    trace_begin(stream, label);
    kern<<<grid, threads, SL::total, stream>>>(ldmap, stmap, in, out, a, tb, g, ntx, (int)ntiles, flags, tma::wait_limit());
    count_launch();
    trace_end(stream);
    return (int)cudaGetLastError();
}

template <int M, int KIND>
int launch_mode(const double* in, double* out, const PassArgs& a, const LineTables<double>& tb, int nv,
                cudaStream_t stream, const char* label) {
    // Only passes whose both sides the copy engine can move are taken: with one
    // side on cp.async (the solver's f, 8-byte-aligned rows) this kernel
    // measured no faster than the cp.async register kernel (x forward at
    // 512^3: 1.04 vs 0.80 ms; x inverse 0.76 vs 0.73 ms), with both it is
    // (do_transform x pass at 512^3: R2C 0.41 vs 0.60 ms, DCT-I 0.66 vs 0.75).
    const bool ld = rows_aligned(in, a.in_su, a.in_sv);
    const bool st = rows_aligned(out, a.out_su, a.out_sv) && !a.use_scale;
    if (ld && st) return launch_one<M, KIND, true, true>(in, out, a, tb, nv, stream, label);
    return -1;
}

// Returns -1 when the pass is not one this kernel takes (the caller then uses
// the cp.async kernel), else a CUDA error code.
template <int M>
int launch_xtma_kind(int kind, int kind2, const void* in, void* out, const PassArgs& a,
                     const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label) {
    if (kind2 >= 0 || a.in_sl != 1 || a.out_sl != 1 || a.acc || a.nu <= 0 || nv <= 0) return -1;
    const double* pi = static_cast<const double*>(in);
    double* po = static_cast<double*>(out);
    switch (kind) {
        case kDCT1: return launch_mode<M, kDCT1>(pi, po, a, tb, nv, stream, label);
        case kDCT2: return launch_mode<M, kDCT2>(pi, po, a, tb, nv, stream, label);
        case kDCT3: return launch_mode<M, kDCT3>(pi, po, a, tb, nv, stream, label);
        case kDST1: return launch_mode<M, kDST1>(pi, po, a, tb, nv, stream, label);
        case kDST2: return launch_mode<M, kDST2>(pi, po, a, tb, nv, stream, label);
        case kDST3: return launch_mode<M, kDST3>(pi, po, a, tb, nv, stream, label);
        case kR2C: return launch_mode<M, kR2C>(pi, po, a, tb, nv, stream, label);
        case kC2R: return launch_mode<M, kC2R>(pi, po, a, tb, nv, stream, label);
        default: return -1;
    }
}

}  // namespace xtma
}  // namespace chz
