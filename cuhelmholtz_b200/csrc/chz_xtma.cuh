// TMA-pipelined line pass for the contiguous (x) passes, FP64.
//
// A tile is 16 lines (rows) of one plane.  Lines along x are contiguous in
// memory, so a tile is held as 16 x 16 blocks: block t holds entries
// 16t .. 16t+15 of the 16 lines, one 128-byte row per line, with the copy
// engine's 128-byte swizzle (16-byte chunk j of row c stored at chunk
// j ^ (c mod 8)) -- exactly what a {16 entries, 16 rows} tensor box with
// CU_TENSOR_MAP_SWIZZLE_128B lands as.  Entry l of line c is therefore at
//   (l / 16) * 256 + c * 16 + 2 * (((l / 2) mod 8) ^ (c mod 8)) + (l mod 2).
// A side of the pass on a 16-byte-aligned array (a padded do_transform array,
// the solver's work array) moves by tensor copies; a side on an array with
// 8-byte-aligned rows (the solver's f) is copied by the producer warp with
// cp.async (32 consecutive entries of a row per instruction, each a whole
// swizzled row: conflict-free), whose completion the stage's mbarrier tracks
// (cp.async.mbarrier.arrive.noinc), or stored by the compute warps.  The host
// takes the kernel only where both sides are tensor copies (the faster case).  The transform is the register-resident
// radix-16 line transform of chz_fast.cuh on this layout (real-view reads of
// one entry by the 16 lines of a slot hit each bank pair at most twice).
#pragma once
#include "chz_tma.cuh"

namespace chz {
namespace xtma {

using fast::OutSink;
using fast::transform_lines;
using tma::kStages;
using tma::mbar_arrive;
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait;
using tma::saddr;
using tma::tma_load;
using tma::tma_store;

__device__ __forceinline__ int swz(int l, int c) {
    return ((l >> 4) << 8) + (c << 4) + ((((l >> 1) & 7) ^ (c & 7)) << 1) + (l & 1);
}

template <typename T>
struct SwzView {
    const T* __restrict__ line;  // buf + 16 c
    int c7;                      // c mod 8
    __device__ __forceinline__ T operator()(int l) const {
        return line[((l >> 4) << 8) + ((((l >> 1) & 7) ^ c7) << 1) + (l & 1)];
    }
};

template <int M_>
struct XCfg {
    static constexpr int M = M_;
    static constexpr int P = M / fast::kR;
    static constexpr int W = 16;
    static constexpr int NT = P * W;
    static constexpr int N = 2 * M;
    static constexpr int L = N + 2;
    static constexpr int NBLK = (L + 15) / 16;   // 16-entry blocks per line
    static constexpr int BUF = NBLK * 256;       // values per tile (>= 2 M W)
    static constexpr int BAR = 1;
    static constexpr int A16 = (M >= 256) ? 2 : 1;
    static constexpr int R0 = M / (A16 == 2 ? 256 : 16);
    static constexpr int NST = A16 + (R0 > 1 ? 1 : 0);
    static constexpr int RED = P * W;
    __device__ static __forceinline__ void sync() { asm volatile("bar.sync 1, %0;\n" ::"n"(NT) : "memory"); }
    template <typename T>
    __device__ static __forceinline__ SwzView<T> reader(const T* buf, int c) {
        return SwzView<T>{buf + (c << 4), c & 7};
    }
    __device__ static __forceinline__ int zi(int m, int c) { return m * W + c; }
};

// Output sink writing the swizzled real view.
template <typename T>
struct SwzSink {
    T* buf;
    int c;
    __device__ __forceinline__ void put(int l, T v) const { buf[swz(l, c)] = v; }
    __device__ __forceinline__ void put_pair(int l, T re, T im) const {
        buf[swz(l, c)] = re;
        buf[swz(l + 1, c)] = im;
    }
};

struct XGeom {
    int ld_blk0, ld_nblk;   // tensor-loaded blocks (LD_TMA)
    int st_blk0, st_nblk;   // tensor-stored blocks (ST_TMA)
};

template <typename T, int M>
struct XSmem {
    using CF = XCfg<M>;
    static constexpr size_t stage = sizeof(T) * CF::BUF;                  // multiple of 2048
    static constexpr size_t twM = kStages * stage;
    static constexpr size_t twN = twM + sizeof(C2<T>) * M;
    static constexpr size_t tw4N = twN + sizeof(C2<T>) * (M + 1);
    static constexpr size_t inv4sin = tw4N + sizeof(C2<T>) * (M + 1);
    static constexpr size_t red = (inv4sin + sizeof(T) * (M + 1) + 15) & ~size_t(15);
    static constexpr size_t bars = (red + sizeof(T) * CF::RED + 15) & ~size_t(15);
    static constexpr size_t abort = bars + 2 * kStages * sizeof(uint64_t);
    static constexpr size_t total = abort + 16 + 1024;  // + alignment slack
};

__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* b) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(saddr(b)) : "memory");
}

// LD_TMA: the input moves by tensor loads (ldmap), else the producer warp
// copies it with cp.async; ST_TMA: the output moves by tensor stores (stmap),
// else the compute warps store it.
template <typename T, int M, int KIND, bool LD_TMA, bool ST_TMA>
__global__ void __launch_bounds__(XCfg<M>::NT + 32, 1)
xtma_pass(const __grid_constant__ CUtensorMap ldmap, const __grid_constant__ CUtensorMap stmap, const T* in,
          T* out, PassArgs a, LineTables<T> tg, XGeom g, int ntx, int ntiles, int* flags,
          long long wait_limit) {
    using CF = XCfg<M>;
    using SL = XSmem<T, M>;
    constexpr int W = CF::W, NT = CF::NT, N = CF::N;
    constexpr int LO = fast::InWin<KIND, N>::lo, HI = fast::InWin<KIND, N>::hi;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const int t = threadIdx.x;
    if ((int)blockIdx.x >= ntiles) return;
    // the 128-byte swizzle needs 1024-byte-aligned boxes (1 KB of slack is allocated)
    unsigned char* smem_raw = smem_dyn + ((1024u - (saddr(smem_dyn) & 1023u)) & 1023u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + SL::bars);
    uint64_t* ready = full + kStages;
    volatile int* abort = reinterpret_cast<volatile int*>(smem_raw + SL::abort);
    T* red = reinterpret_cast<T*>(smem_raw + SL::red);

    LineTables<T> tb = tg;
    {
        C2<T>* sM = reinterpret_cast<C2<T>*>(smem_raw + SL::twM);
        C2<T>* sN = reinterpret_cast<C2<T>*>(smem_raw + SL::twN);
        C2<T>* s4 = reinterpret_cast<C2<T>*>(smem_raw + SL::tw4N);
        T* sI = reinterpret_cast<T*>(smem_raw + SL::inv4sin);
        for (int i = t; i < M; i += blockDim.x) sM[i] = tg.twM[i];
        for (int i = t; i <= M; i += blockDim.x) {
            sN[i] = tg.twN[i];
            s4[i] = tg.tw4N[i];
            sI[i] = tg.inv4sin[i];
        }
        tb.twM = sM;
        tb.twN = sN;
        tb.tw4N = s4;
        tb.inv4sin = sI;
    }
    if (t == 0) {
        *abort = 0;
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full + s, LD_TMA ? 1 : 32);
            mbar_init(ready + s, NT);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    const int nloc = (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;
    auto stage_of = [&](int s) { return reinterpret_cast<T*>(smem_raw + (size_t)s * SL::stage); };

    if (t >= NT) {
        // ---------------- producer warp ----------------
        const int lane = t - NT;
        auto issue_load = [&](int i) {
            const int s = i % kStages;
            const int tile = (int)blockIdx.x + i * (int)gridDim.x;
            const int ub = a.u0 + (tile % ntx) * W;
            const int v = a.v0 + tile / ntx;
            T* dst = stage_of(s);
            if constexpr (LD_TMA) {
                if (lane == 0) {
                    mbar_expect_tx(full + s, (uint32_t)(g.ld_nblk * 256 * sizeof(T)));
                    for (int q = 0; q < g.ld_nblk; ++q) {
                        const int blk = g.ld_blk0 + q;
                        tma_load(dst + blk * 256, &ldmap, blk * 16, ub, v, full + s);
                    }
                }
            } else {
                const int nl = min(W, a.u0 + a.nu - ub);
                for (int r = 0; r < W; ++r) {
                    const bool ok = r < nl;
                    const T* row = in + (long long)v * a.in_sv + (long long)(ok ? ub + r : ub) * a.in_su;
                    for (int l = LO + lane; l <= HI; l += 32) {
                        const bool valid = ok && l >= a.ld_lo && l <= a.ld_hi;
                        cp_async_elem<sizeof(T)>(dst + swz(l, r), valid ? row + l : in, valid);
                    }
                }
                cp_async_arrive_noinc(full + s);
            }
        };
        if (!LD_TMA || !ST_TMA || lane == 0) {
            if (LD_TMA && lane == 0) {
                asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&ldmap)) : "memory");
            }
            if (ST_TMA && lane == 0) {
                asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&stmap)) : "memory");
            }
            const int pre = nloc < kStages ? nloc : kStages;
            for (int i = 0; i < pre; ++i) issue_load(i);
            for (int i = 0; i < nloc; ++i) {
                const int s = i % kStages;
                if (!mbar_wait(ready + s, (uint32_t)((i / kStages) & 1), abort, wait_limit))
                    atomicOr(flags, tma::kFlagProducer);
                if constexpr (ST_TMA) {
                    if (lane == 0) {
                        const int tile = (int)blockIdx.x + i * (int)gridDim.x;
                        const int ub = a.u0 + (tile % ntx) * W;
                        const int v = a.v0 + tile / ntx;
                        const T* src = stage_of(s);
                        for (int q = 0; q < g.st_nblk; ++q) {
                            const int blk = g.st_blk0 + q;
                            tma_store(&stmap, blk * 16, ub, v, src + blk * 256);
                        }
                        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
                    }
                }
                if (i + kStages < nloc) {
                    if constexpr (ST_TMA) {
                        if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
                    }
                    if constexpr (!LD_TMA) __syncwarp();
                    issue_load(i + kStages);
                }
            }
            if constexpr (ST_TMA) {
                if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
            }
            if constexpr (!LD_TMA) asm volatile("cp.async.wait_all;\n" ::: "memory");
            if constexpr (LD_TMA) {
                if (lane == 0) tma::drain_loads(full, nloc, kStages, wait_limit, flags);
            }
        }
        return;
    }

    // ---------------- compute ----------------
    const int c = t % W;
    const int slot = t / W;
    const double sc = a.use_scale ? a.scale : 1.0;
    for (int i = 0; i < nloc; ++i) {
        const int s = i % kStages;
        if (!mbar_wait(full + s, (uint32_t)((i / kStages) & 1), abort, wait_limit)) {
            if (t == 0) atomicOr(flags, tma::kFlagConsumer);
        }
        T* buf = stage_of(s);
        const int tile = (int)blockIdx.x + i * (int)gridDim.x;
        const int ub = a.u0 + (tile % ntx) * W;
        const int v = a.v0 + tile / ntx;
        const int nl = min(W, a.u0 + a.nu - ub);
        bool fix = false;
        if constexpr (LD_TMA) {
            // entries of the kind's input window outside the load window are 0
            if (LO < a.ld_lo || HI > a.ld_hi) {
                for (int e = t; e < W * (HI - LO + 1); e += NT) {
                    const int r = e % W, l = LO + e / W;
                    if (l < a.ld_lo || l > a.ld_hi) buf[swz(l, r)] = T(0);
                }
                fix = true;
            }
        }
        if (a.has_bc) {
            // boundary terms: every entry of a row on a y or z boundary, else
            // the entries at xs and xe (one (row, side) per thread)
            const BcArgs& b = a.bc;
            const bool zrow = (v == b.zs || v == b.ze);
            for (int r = 0; r < nl; ++r) {
                const int j = ub + r;
                if (!(zrow || j == b.ys || j == b.ye)) continue;
                for (int l = a.ld_lo + t; l <= a.ld_hi; l += NT)
                    buf[swz(l, r)] = (T)bc_terms((double)buf[swz(l, r)], b, l, j, v);
            }
            for (int e = t; e < 2 * nl; e += NT) {
                const int r = e >> 1, j = ub + r;
                if (zrow || j == b.ys || j == b.ye) continue;
                if ((e & 1) && b.xe == b.xs) continue;
                const int l = (e & 1) ? b.xe : b.xs;
                buf[swz(l, r)] = (T)bc_terms((double)buf[swz(l, r)], b, l, j, v);
            }
            fix = true;
        }
        if (fix) CF::sync();
        SwzSink<T> sink{buf, c};
        transform_lines<T, CF, KIND>(buf, red, c, slot, tb, sink);
        if constexpr (ST_TMA) {
            // make this thread's writes visible to the tensor store, then release
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        } else {
            // each warp stores rows r = 2w, 2w + 1: 32 consecutive entries per instruction
            const int lane = t & 31, wq = t >> 5;
            for (int r = wq; r < W; r += NT / 32) {
                if (r >= nl) continue;
                T* row = out + (long long)v * a.out_sv + (long long)(ub + r) * a.out_su;
                for (int l = a.st_lo + lane; l <= a.st_hi; l += 32) row[l] = (T)((double)buf[swz(l, r)] * sc);
            }
        }
        mbar_arrive(ready + s);
    }
}

}  // namespace xtma
}  // namespace chz
