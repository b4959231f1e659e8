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

// Launches one instantiation; -1 when the geometry does not fit it.
template <int M, int KIND, int LDM, int STM>
int launch_one(const double* in, double* out, const PassArgs& a, const LineTables<double>& tb, int nv,
               cudaStream_t stream, const char* label) {
    using CF = XCfg<M>;
    using SL = XSmem<double, M>;
    constexpr int W = CF::W, TW = CF::TW, N = CF::N;
    constexpr int LO = fast::InWin<KIND, N>::lo, HI = fast::InWin<KIND, N>::hi;
    if ((long long)SL::total > (long long)tma::max_optin_smem()) return -1;
    XGeom g{};
    CUtensorMap ldmap, stmap;
    std::memset(&ldmap, 0, sizeof(ldmap));
    std::memset(&stmap, 0, sizeof(stmap));
    // a box is one 16-entry block of the W lines of a compute group
    const unsigned box[3] = {16u, (unsigned)W, 1u};
    // the maps start at the pass's first plane v0 (16-byte aligned: whole
    // planes of 16-byte-aligned rows); a caller may hand a base moved back by
    // planes it never addresses (the slab solve), and a tensor map's base must
    // lie in its allocation
    g.v_off = a.v0;
    if (LDM == kLdTensor) {
        g.ld_blk0 = LO >> 4;
        g.ld_nblk = (HI >> 4) - g.ld_blk0 + 1;
        const unsigned long long dims[3] = {(unsigned long long)(a.ld_hi + 1), (unsigned long long)(a.u0 + a.nu),
                                            (unsigned long long)nv};
        const unsigned long long strides[2] = {(unsigned long long)(a.in_su * 8), (unsigned long long)(a.in_sv * 8)};
        if (!tma::encode_map_swz(&ldmap, in + (long long)a.v0 * a.in_sv, dims, strides, box)) return -1;
    } else {
        // whole rows of the span, row-major: the kind's input window inside a
        // row, and a group's W rows (plus the span's misalignment) inside its
        // region of a stage
        if (HI > a.in_su - 1 || a.in_sv < a.in_su * (a.u0 + a.nu) || W * a.in_su + 2 > CF::GBUF) return -1;
    }
    if (STM == kStTensor) {
        g.st_blk0 = a.st_lo >> 4;
        g.st_nblk = (a.st_hi >> 4) - g.st_blk0 + 1;
        const unsigned long long dims[3] = {(unsigned long long)(a.st_hi + 1), (unsigned long long)(a.u0 + a.nu),
                                            (unsigned long long)nv};
        const unsigned long long strides[2] = {(unsigned long long)(a.out_su * 8),
                                               (unsigned long long)(a.out_sv * 8)};
        if (!tma::encode_map_swz(&stmap, out + (long long)a.v0 * a.out_sv, dims, strides, box)) return -1;
    } else {
        // the kind's output window inside a row (the row-major sink writes
        // every entry of it), the W rows inside a stage, 8-byte-aligned rows
        int o0, o1;
        kind_out_window(KIND, N, o0, o1);
        if (o1 > a.out_su - 1 || a.st_lo < 0 || a.st_hi > a.out_su - 1 || W * a.out_su + 2 > CF::GBUF ||
            (reinterpret_cast<uintptr_t>(out) & 7))
            return -1;
    }
    int* flags = tma::device_flags();
    if (!flags) return -1;
    auto kern = xtma_pass<double, M, KIND, LDM, STM>;
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
    const int ntx = (a.nu + TW - 1) / TW;
    const long long ntiles = (long long)ntx * nv;
    if (ntiles <= 0) return 0;
    if (ntiles > 0x7fffffffLL) return -1;
    const long long cap = (long long)cps * fast::device_sm_count();
    const int grid = (int)std::min(ntiles, cap);
    trace_begin(stream, label);
    kern<<<grid, threads, SL::total, stream>>>(ldmap, stmap, in, out, a, tb, g, ntx, (int)ntiles, flags,
                                                tma::wait_limit());
    count_launch();
    trace_end(stream);
    return (int)cudaGetLastError();
}

// Side modes of a pass: a 16-byte-aligned array moves by tensor boxes, rows
// of an 8-byte-aligned array (the solver's f) by bulk copies of the span.
inline bool span_side(const void* p, long long pitch) {
    return !(reinterpret_cast<uintptr_t>(p) & 7) && pitch > 0;
}

// Kinds instantiated per side combination: every kind with tensor copies on
// both sides (do_transform), the solver's forward kinds with a span input
// (f -> work array) and its inverse kinds with row stores (work array -> f).
int launch_span_tensor_m256(int kind, const double* in, double* out, const PassArgs& a,
                            const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label);
int launch_tensor_rows_m256(int kind, const double* in, double* out, const PassArgs& a,
                            const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label);
int launch_span_tensor_m128(int kind, const double* in, double* out, const PassArgs& a,
                            const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label);
int launch_tensor_rows_m128(int kind, const double* in, double* out, const PassArgs& a,
                            const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label);

template <int M, int LDM, int STM>
int launch_kinds(int kind, const double* in, double* out, const PassArgs& a, const LineTables<double>& tb, int nv,
                 cudaStream_t stream, const char* label) {
    if constexpr (LDM == kLdTensor && STM == kStTensor) {
        switch (kind) {
            case kDCT1: return launch_one<M, kDCT1, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDCT2: return launch_one<M, kDCT2, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDCT3: return launch_one<M, kDCT3, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST1: return launch_one<M, kDST1, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST2: return launch_one<M, kDST2, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST3: return launch_one<M, kDST3, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kR2C: return launch_one<M, kR2C, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kC2R: return launch_one<M, kC2R, LDM, STM>(in, out, a, tb, nv, stream, label);
            default: return -1;
        }
    } else if constexpr (LDM == kLdSpan && STM == kStTensor) {
        switch (kind) {
            case kR2C: return launch_one<M, kR2C, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST1: return launch_one<M, kDST1, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST3: return launch_one<M, kDST3, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDCT1: return launch_one<M, kDCT1, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDCT3: return launch_one<M, kDCT3, LDM, STM>(in, out, a, tb, nv, stream, label);
            default: return -1;
        }
    } else if constexpr (LDM == kLdTensor && STM == kStRows) {
        switch (kind) {
            case kC2R: return launch_one<M, kC2R, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST1: return launch_one<M, kDST1, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDST2: return launch_one<M, kDST2, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDCT1: return launch_one<M, kDCT1, LDM, STM>(in, out, a, tb, nv, stream, label);
            case kDCT2: return launch_one<M, kDCT2, LDM, STM>(in, out, a, tb, nv, stream, label);
            default: return -1;
        }
    } else {
        return -1;
    }
}

// Returns -1 when the pass is not one this kernel takes (the caller then uses
// the cp.async kernel), else a CUDA error code.
template <int M>
int launch_xtma_kind(int kind, int kind2, const void* in, void* out, const PassArgs& a,
                     const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label) {
    if (kind2 >= 0 || a.in_sl != 1 || a.out_sl != 1 || a.acc || a.nu <= 0 || nv <= 0) return -1;
    const double* pi = static_cast<const double*>(in);
    double* po = static_cast<double*>(out);
    const bool ld_tensor = rows_aligned(in, a.in_su, a.in_sv);
    const bool st_tensor = rows_aligned(out, a.out_su, a.out_sv) && !a.use_scale;
    if (ld_tensor && st_tensor) return launch_kinds<M, kLdTensor, kStTensor>(kind, pi, po, a, tb, nv, stream, label);
    auto span = M == 256 ? launch_span_tensor_m256 : launch_span_tensor_m128;
    auto rows = M == 256 ? launch_tensor_rows_m256 : launch_tensor_rows_m128;
    if (!ld_tensor && st_tensor && span_side(in, a.in_su)) return span(kind, pi, po, a, tb, nv, stream, label);
    if (ld_tensor && (!rows_aligned(out, a.out_su, a.out_sv) || a.use_scale) && span_side(out, a.out_su))
        return rows(kind, pi, po, a, tb, nv, stream, label);
    return -1;
}

}  // namespace xtma
}  // namespace chz
