// Host side of the TMA-pipelined strided pass (included by the per-length
// translation units chz_tma_*.cu, which instantiate it).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "chz_tma.cuh"

namespace chz {
namespace fast {
int device_sm_count();
}
namespace tma {

// Encodes a 3-D tiled tensor map (driver entry point, resolved once); false
// when the driver refuses the geometry.
bool encode_map(CUtensorMap* map, bool is_double, const void* base, const unsigned long long dims[3],
                const unsigned long long strides[2], const unsigned box[3]);
int* device_flags();
// limit of the kernels' bounded waits, in SM clock cycles (chz_set_wait_limit)
long long wait_limit();
int max_optin_smem();

template <int KIND, int N>
using InWin = fast::InWin<KIND, N>;

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

template <typename T, int M, int KIND, int K2>
int launch_one(const T* in, T* out, const PassArgs& a, const LineTables<T>& tb, int nv, cudaStream_t stream,
               const char* label) {
    using CF = TCfg<T, M>;
    constexpr int W = CF::W, N = CF::N;
    constexpr long long ES = sizeof(T);
    constexpr int LO = InWin<KIND, N>::lo, HI = InWin<KIND, N>::hi;
    if (a.in_su != 1 || a.out_su != 1 || nv <= 0 || a.nu <= 0) return -1;
    const bool l_mid = a.in_sl < a.in_sv;
    if (l_mid != (a.out_sl < a.out_sv)) return -1;
    // column 0 of the maps: u0 rounded down to a 16-byte boundary
    const int col0 = a.u0 & ~(int)(16 / ES - 1);
    const int du = a.u0 + a.nu - col0;
    const int dv = a.v0 + nv;
    TmaGeom g{};
    g.col0 = col0;
    g.l_mid = l_mid ? 1 : 0;
    const int rows_ld = HI - LO + 1;
    g.ld_nch = ceil_div(rows_ld, 256);
    g.ld_box = ceil_div(rows_ld, g.ld_nch);
    g.ld_row0 = LO;
    g.ld_coord0 = LO - a.ld_lo;
    const int rows_st = a.st_hi - a.st_lo + 1;
    if (rows_st <= 0 || a.ld_hi < a.ld_lo) return -1;
    g.st_nch = ceil_div(rows_st, 256);
    g.st_box = ceil_div(rows_st, g.st_nch);
    g.st_row0 = a.st_lo;
    int rows = std::max(N + 2, std::max(LO + g.ld_nch * g.ld_box, a.st_lo + g.st_nch * g.st_box));
    g.rows_buf = (rows + 7) & ~7;
    g.tx_bytes = (unsigned)(g.ld_nch * g.ld_box * W * ES);

    using SL = TmaSmem<T, M, (K2 >= 0), UsesDctTables<KIND, K2>::value>;
    const size_t smem = SL::total(g.rows_buf);
    if ((long long)smem > (long long)max_optin_smem()) return -1;

    const T* ld_base = in + col0 + (long long)a.ld_lo * a.in_sl;
    T* st_base = out + col0 + (long long)a.st_lo * a.out_sl;
    if ((reinterpret_cast<uintptr_t>(ld_base) & 15) || (reinterpret_cast<uintptr_t>(st_base) & 15)) return -1;
    // The maps start at the pass's first plane v0 where that stays 16-byte
    // aligned: a caller may hand a base moved back by planes it never
    // addresses (the slab solve), and a tensor map's base must lie in its
    // allocation.  Otherwise they start at plane 0 of the array.
    g.v_off = 0;
    {
        const T* l2 = ld_base + (long long)a.v0 * a.in_sv;
        T* s2 = st_base + (long long)a.v0 * a.out_sv;
        if (!(reinterpret_cast<uintptr_t>(l2) & 15) && !(reinterpret_cast<uintptr_t>(s2) & 15)) {
            ld_base = l2;
            st_base = s2;
            g.v_off = a.v0;
        }
    }
    const int dvm = dv - g.v_off;   // planes the maps cover
    CUtensorMap ldmap, stmap;
    {
        const unsigned long long dl = (unsigned long long)(a.ld_hi - a.ld_lo + 1);
        const unsigned long long dims[3] = {(unsigned long long)du, l_mid ? dl : (unsigned long long)dvm,
                                            l_mid ? (unsigned long long)dvm : dl};
        const unsigned long long sl = (unsigned long long)(a.in_sl * ES), sv = (unsigned long long)(a.in_sv * ES);
        const unsigned long long strides[2] = {l_mid ? sl : sv, l_mid ? sv : sl};
        const unsigned box[3] = {(unsigned)W, l_mid ? (unsigned)g.ld_box : 1u, l_mid ? 1u : (unsigned)g.ld_box};
        if (!encode_map(&ldmap, ES == 8, ld_base, dims, strides, box)) return -1;
    }
    {
        const unsigned long long dl = (unsigned long long)rows_st;
        const unsigned long long dims[3] = {(unsigned long long)du, l_mid ? dl : (unsigned long long)dvm,
                                            l_mid ? (unsigned long long)dvm : dl};
        const unsigned long long sl = (unsigned long long)(a.out_sl * ES), sv = (unsigned long long)(a.out_sv * ES);
        const unsigned long long strides[2] = {l_mid ? sl : sv, l_mid ? sv : sl};
        const unsigned box[3] = {(unsigned)W, l_mid ? (unsigned)g.st_box : 1u, l_mid ? 1u : (unsigned)g.st_box};
        if (!encode_map(&stmap, ES == 8, st_base, dims, strides, box)) return -1;
    }
    int* flags = device_flags();
    if (!flags) return -1;

    auto kern = tma_pass<T, M, KIND, K2>;
    constexpr int threads = CF::NT + 32;
    // shared-memory opt-in (raised as needed) and CTAs per SM, per instantiation
    static std::atomic<int> opted{0};
    static std::atomic<long long> occ_key{-1};
    static std::atomic<int> occ_val{0};
    if ((int)smem > opted.load(std::memory_order_relaxed)) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return (int)e;
        opted.store((int)smem, std::memory_order_relaxed);
    }
    int cps;
    if (occ_key.load(std::memory_order_relaxed) == (long long)smem) {
        cps = occ_val.load(std::memory_order_relaxed);
    } else {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, kern, threads, smem);
        if (e != cudaSuccess) return (int)e;
        occ_val.store(cps, std::memory_order_relaxed);
        occ_key.store((long long)smem, std::memory_order_relaxed);
    }
    if (cps < 1) return -1;
    const int ntx = ceil_div(du, W);
    const long long ntiles = (long long)ntx * nv;
    if (ntiles > 0x7fffffffLL) return -1;
    const long long cap = (long long)cps * fast::device_sm_count();
    const int grid = (int)std::min(ntiles, cap);
    trace_begin(stream, label);
    kern<<<grid, threads, smem, stream>>>(ldmap, stmap, a, tb, g, ntx, (int)ntiles, flags, wait_limit());
    count_launch();
    trace_end(stream);
    return (int)cudaGetLastError();
}

// Returns -1 when the pass is not one this kernel takes (the caller then
// uses the cp.async kernel), else a CUDA error code.
template <typename T, int M>
int launch_tma_kind(int kind, int kind2, const void* in, void* out, const PassArgs& a, const LineTables<T>& tb,
                    int nv, cudaStream_t stream, const char* label) {
    const T* pi = static_cast<const T*>(in);
    T* po = static_cast<T*>(out);
    if (kind2 < 0) {
        switch (kind) {
            case kDCT1: return launch_one<T, M, kDCT1, -1>(pi, po, a, tb, nv, stream, label);
            case kDCT2: return launch_one<T, M, kDCT2, -1>(pi, po, a, tb, nv, stream, label);
            case kDCT3: return launch_one<T, M, kDCT3, -1>(pi, po, a, tb, nv, stream, label);
            case kDST1: return launch_one<T, M, kDST1, -1>(pi, po, a, tb, nv, stream, label);
            case kDST2: return launch_one<T, M, kDST2, -1>(pi, po, a, tb, nv, stream, label);
            case kDST3: return launch_one<T, M, kDST3, -1>(pi, po, a, tb, nv, stream, label);
            case kR2C: return launch_one<T, M, kR2C, -1>(pi, po, a, tb, nv, stream, label);
            case kC2R: return launch_one<T, M, kC2R, -1>(pi, po, a, tb, nv, stream, label);
            default: return -1;
        }
    }
    if (kind == kR2C && kind2 == kC2R) return launch_one<T, M, kR2C, kC2R>(pi, po, a, tb, nv, stream, label);
    if (kind == kDST1 && kind2 == kDST1) return launch_one<T, M, kDST1, kDST1>(pi, po, a, tb, nv, stream, label);
    if (kind == kDST3 && kind2 == kDST2) return launch_one<T, M, kDST3, kDST2>(pi, po, a, tb, nv, stream, label);
    if (kind == kDCT1 && kind2 == kDCT1) return launch_one<T, M, kDCT1, kDCT1>(pi, po, a, tb, nv, stream, label);
    if (kind == kDCT3 && kind2 == kDCT2) return launch_one<T, M, kDCT3, kDCT2>(pi, po, a, tb, nv, stream, label);
    return -1;
}

}  // namespace tma
}  // namespace chz
