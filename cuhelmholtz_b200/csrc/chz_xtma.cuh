// TMA-pipelined line pass for the contiguous (x) passes, FP64.
//
// A tile is 16 lines (rows) of one plane, held by G compute groups of W
// lines each (G = 2, W = 8 at N = 512; G = 1, W = 16 at N = 256), every group
// in its own region of the stage buffer.  Lines along x are contiguous in
// memory, so a group's region is held as 16 x W blocks: block t holds entries
// 16t .. 16t+15 of the W lines, one 128-byte row per line, with the copy
// engine's 128-byte swizzle (16-byte chunk j of row c stored at chunk
// j ^ (c mod 8)) -- exactly what a {16 entries, W rows} tensor box with
// CU_TENSOR_MAP_SWIZZLE_128B lands as.  Entry l of line c is therefore at
//   (l / 16) * 16 W + c * 16 + 2 * (((l / 2) mod 8) ^ (c mod 8)) + (l mod 2).
// A side of the pass on a 16-byte-aligned array (a padded do_transform array,
// the solver's work array) moves by tensor copies in that layout.  A side on
// an array whose rows are only 8-byte aligned (the solver's f, rows of N + 1
// values) moves untiled instead: the W rows of a group are one contiguous
// span of memory, so a load is a single cp.async.bulk of the span widened to
// 16-byte boundaries, landing row-major (entry l of line c at
// off + c * pitch + l, off = 0 or 1 the span's misalignment), and a store
// leaves row-major the same way: one cp.async.bulk per row of the 16-byte-
// aligned interior of its output window (one for the group's rows when the
// window is whole rows), the 8-byte ends by plain stores, so neighbouring
// groups and tiles never write the same 16 bytes.  The transform is the
// register-resident radix-16 line transform of chz_fast.cuh on either layout
// (swizzled: the lines of a slot hit each bank pair at most twice; row-major
// with an odd pitch: each bank at most twice per instruction).  The groups
// share nothing but the stage barriers, so each synchronises on its own named
// barrier and they drift apart: one group's shared-memory phases overlap the
// other's arithmetic.
#pragma once
#include "chz_tma.cuh"

namespace chz {
namespace xtma {

using fast::OutSink;
using fast::transform_lines;
using fast::transform_lines_v;
using tma::kStages;
using tma::mbar_arrive;
using tma::mbar_expect_tx;
using tma::mbar_init;
using tma::mbar_wait;
using tma::saddr;
using tma::tma_load;
using tma::tma_store;

// Entry l of line c in the swizzled layout whose 16-entry blocks hold BS
// values (16 x the lines of the region).
template <int BS>
__device__ __forceinline__ int swz(int l, int c) {
    return (l >> 4) * BS + (c << 4) + ((((l >> 1) & 7) ^ (c & 7)) << 1) + (l & 1);
}

template <typename T, int BS>
struct SwzView {
    const T* __restrict__ line;  // region + 16 c
    int c7;                      // c mod 8
    // entries 2j, 2j + 1 are one swizzled 16-byte chunk
    static constexpr bool kPair = sizeof(T) == 8;
    __device__ __forceinline__ T operator()(int l) const {
        return line[(l >> 4) * BS + ((((l >> 1) & 7) ^ c7) << 1) + (l & 1)];
    }
    __device__ __forceinline__ C2<T> pair(int l) const {   // l even
        return *reinterpret_cast<const C2<T>*>(line + (l >> 4) * BS + ((((l >> 1) & 7) ^ c7) << 1));
    }
};

// A tile is TW = 16 lines.  At N = 512 its lines are split between G = 2
// compute groups of 8 lines (four warps each), each with its own region of the
// stage buffer and its own named barrier, so the groups drift apart and one
// group's shared-memory phases overlap the other's arithmetic; at N = 256 one
// group holds all 16 lines.  The members below describe one group (W lines,
// GNT threads) -- what the line transform sees.
template <int M_>
struct XCfg {
    static constexpr int M = M_;
    static constexpr int V = fast::kR;
    static constexpr int P = M / fast::kR;
    static constexpr int TW = 16;                      // lines of a tile
    static constexpr int G = (M >= 256) ? 2 : 1;       // compute groups
    static constexpr int W = TW / G;                   // lines of a group
    static constexpr int NT = P * TW;                  // compute threads
    static constexpr int GNT = P * W;                  // threads of a group
    static constexpr int N = 2 * M;
    static constexpr int L = N + 2;
    static constexpr int NBLK = (L + 15) / 16;         // 16-entry blocks per line
    static constexpr int BS = 16 * W;                  // values of one block of a group region
    static constexpr int GBUF = NBLK * BS;             // values of a group region (>= 2 M W)
    static constexpr int BUF = G * GBUF;               // values per stage
    static constexpr int BAR = 1;
    static constexpr int A16 = (M >= 256) ? 2 : 1;
    static constexpr int R0 = M / (A16 == 2 ? 256 : 16);
    static constexpr int NST = A16 + (R0 > 1 ? 1 : 0);
    static constexpr int RED = P * W;                  // per group
    // named barrier of the calling thread's group (ids 1 .. G)
    __device__ static __forceinline__ void sync() {
        if constexpr (G == 1) {
            asm volatile("bar.sync 1, %0;\n" ::"n"(NT) : "memory");
        } else {
            asm volatile("bar.sync %0, %1;\n" ::"r"(1 + (int)threadIdx.x / GNT), "n"(GNT) : "memory");
        }
    }
    template <typename T>
    __device__ static __forceinline__ SwzView<T, BS> reader(const T* buf, int c) {
        return SwzView<T, BS>{buf + (c << 4), c & 7};
    }
    __device__ static __forceinline__ int zi(int m, int c) { return m * W + c; }
};

// Output sink writing the swizzled real view.
template <typename T, int BS>
struct SwzSink {
    T* buf;
    int c;
    __device__ __forceinline__ void put(int l, T v) const { buf[swz<BS>(l, c)] = v; }
    // l even: entries l, l + 1 are one swizzled 16-byte chunk
    __device__ __forceinline__ void put_pair(int l, T re, T im) const {
        *reinterpret_cast<C2<T>*>(buf + swz<BS>(l, c)) = mk<T>(re, im);
    }
    __device__ __forceinline__ void put2(int l, T a, T b) const { put_pair(l, a, b); }
};

struct XGeom {
    int ld_blk0, ld_nblk;   // tensor-loaded blocks (LD_TMA)
    int st_blk0, st_nblk;   // tensor-stored blocks (ST_TMA)
    int v_off;              // v of the maps' first plane
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
    static constexpr size_t bars = (red + sizeof(T) * CF::RED * CF::G + 15) & ~size_t(15);
    static constexpr size_t abort = bars + 2 * kStages * sizeof(uint64_t);
    static constexpr size_t total = abort + 16 + 1024;  // + alignment slack
};

__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* b) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(saddr(b)) : "memory");
}

// How each side of a tile moves.
enum XLoad { kLdTensor = 0, kLdSpan = 1 };
enum XStore { kStTensor = 0, kStRows = 1 };

// Row-major real view of one line (span loads): entry l at line[l].
template <typename T>
struct RowView {
    const T* __restrict__ line;
    static constexpr bool kPair = false;   // a row may start on either 8-byte phase
    __device__ __forceinline__ T operator()(int l) const { return line[l]; }
    __device__ __forceinline__ C2<T> pair(int l) const { return mk<T>(line[l], line[l + 1]); }
};

// Output sink of the row-major view (row stores), scaled as it is written.
template <typename T>
struct RowSink {
    T* line;
    double sc;
    __device__ __forceinline__ void put(int l, T v) const { line[l] = (T)((double)v * sc); }
    __device__ __forceinline__ void put_pair(int l, T re, T im) const {
        line[l] = (T)((double)re * sc);
        line[l + 1] = (T)((double)im * sc);
    }
    __device__ __forceinline__ void put2(int l, T a, T b) const { put_pair(l, a, b); }
};

// A tile's span: its first value at `p`, the 16-byte-aligned address at or
// below it and the 8-byte words between the two (0 or 1 for FP64).
struct Span {
    uintptr_t a0;
    int off;
};
template <typename T>
__device__ __forceinline__ Span span_at(const T* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    return Span{a & ~uintptr_t(15), (int)((a & 15) / sizeof(T))};
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void bulk_store(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(
                     reinterpret_cast<uint64_t>(dst)),
                 "r"(saddr(src)), "r"(bytes)
                 : "memory");
}

// The 16-byte-aligned interior [i0, i1) of the byte range [b0, b1).
__device__ __forceinline__ void interior(uintptr_t b0, uintptr_t b1, uintptr_t& i0, uintptr_t& i1) {
    i0 = (b0 + 15) & ~uintptr_t(15);
    i1 = b1 & ~uintptr_t(15);
}

// LDM: kLdTensor -- the input moves by 16 x 16 tensor boxes (ldmap, swizzled
// layout); kLdSpan -- by one bulk copy of the tile's rows (row-major, rows of
// a.in_su values).  STM: kStTensor -- the output leaves by tensor boxes
// (stmap); kStRows -- by bulk copies of each row's aligned interior (rows of
// a.out_su values), scaled by a.scale when a.use_scale.
template <typename T, int M, int KIND, int LDM, int STM>
__global__ void __launch_bounds__(XCfg<M>::NT + 32, (M <= 128 ? 2 : 1))
xtma_pass(const __grid_constant__ CUtensorMap ldmap, const __grid_constant__ CUtensorMap stmap, const T* in,
          T* out, PassArgs a, LineTables<T> tg, XGeom g, int ntx, int ntiles, int* flags,
          long long wait_limit) {
    using CF = XCfg<M>;
    using SL = XSmem<T, M>;
    constexpr int W = CF::W, TW = CF::TW, G = CF::G, NT = CF::NT, GNT = CF::GNT, N = CF::N;
    constexpr int BS = CF::BS, GBUF = CF::GBUF;
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
            mbar_init(full + s, 1);
            mbar_init(ready + s, NT);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    const int nloc = (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;
    // region of group g in stage s
    auto region_of = [&](int s, int g) { return reinterpret_cast<T*>(smem_raw + (size_t)s * SL::stage) + g * GBUF; };
    // tile i of this CTA: first line ub, plane v, lines nl
    auto tile_of = [&](int i, int& ub, int& v, int& nl) {
        const int tile = (int)blockIdx.x + i * (int)gridDim.x;
        ub = a.u0 + (tile % ntx) * TW;
        v = a.v0 + tile / ntx;
        nl = min(TW, a.u0 + a.nu - ub);
    };
    // lines of group g in a tile of nl lines
    auto group_lines = [&](int nl, int g) { return max(0, min(W, nl - g * W)); };
    auto in_row0 = [&](int ub, int v) { return in + (long long)v * a.in_sv + (long long)ub * a.in_su; };
    auto out_row0 = [&](int ub, int v) { return out + (long long)v * a.out_sv + (long long)ub * a.out_su; };

    if (t >= NT) {
        // ---------------- producer (one thread) ----------------
        if (t != NT) return;
        if constexpr (LDM == kLdTensor)
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&ldmap)) : "memory");
        if constexpr (STM == kStTensor)
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&stmap)) : "memory");
        auto issue_load = [&](int i) {
            const int s = i % kStages;
            int ub, v, nl;
            tile_of(i, ub, v, nl);
            // every group with lines gets its own copies; the stage's barrier
            // expects all of their bytes
            uint32_t bytes = 0;
            uintptr_t span0[G];
            uint32_t spanb[G];
            for (int gr = 0; gr < G; ++gr) {
                const int gl = group_lines(nl, gr);
                spanb[gr] = 0;
                if (gl == 0) continue;
                if constexpr (LDM == kLdTensor) {
                    spanb[gr] = (uint32_t)(g.ld_nblk * BS * sizeof(T));
                } else {
                    // rows of the group, whole, as one span widened to 16 bytes
                    const T* p0 = in_row0(ub + gr * W, v);
                    const Span sp = span_at(p0);
                    const uintptr_t end = (reinterpret_cast<uintptr_t>(p0 + (long long)gl * a.in_su) + 15) &
                                          ~uintptr_t(15);
                    span0[gr] = sp.a0;
                    spanb[gr] = (uint32_t)(end - sp.a0);
                }
                bytes += spanb[gr];
            }
            mbar_expect_tx(full + s, bytes);
            for (int gr = 0; gr < G; ++gr) {
                if (spanb[gr] == 0) continue;
                T* dst = region_of(s, gr);
                if constexpr (LDM == kLdTensor) {
                    for (int q = 0; q < g.ld_nblk; ++q) {
                        const int blk = g.ld_blk0 + q;
                        tma_load(dst + blk * BS, &ldmap, blk * 16, ub + gr * W, v - g.v_off, full + s);
                    }
                } else {
                    bulk_load(dst, reinterpret_cast<const void*>(span0[gr]), spanb[gr], full + s);
                }
            }
        };
        const int pre = nloc < kStages ? nloc : kStages;
        for (int i = 0; i < pre; ++i) issue_load(i);
        for (int i = 0; i < nloc; ++i) {
            const int s = i % kStages;
            if (!mbar_wait(ready + s, (uint32_t)((i / kStages) & 1), abort, wait_limit))
                atomicOr(flags, kFlagProducer);
            int ub, v, nl;
            tile_of(i, ub, v, nl);
            for (int gr = 0; gr < G; ++gr) {
                const int gl = group_lines(nl, gr);
                if (gl == 0) continue;
                const T* src = region_of(s, gr);
                if constexpr (STM == kStTensor) {
                    for (int q = 0; q < g.st_nblk; ++q) {
                        const int blk = g.st_blk0 + q;
                        tma_store(&stmap, blk * 16, ub + gr * W, v - g.v_off, src + blk * BS);
                    }
                } else {
                    // aligned interiors of the rows' output windows (the ends
                    // are stored by the compute threads)
                    T* p0 = out_row0(ub + gr * W, v);
                    const uintptr_t base = reinterpret_cast<uintptr_t>(p0) & ~uintptr_t(15);
                    const unsigned char* sb = reinterpret_cast<const unsigned char*>(src);
                    const bool whole = a.st_lo == 0 && a.st_hi == a.out_su - 1;
                    for (int r = 0; r < (whole ? 1 : gl); ++r) {
                        const T* q0 = p0 + (long long)r * a.out_su + a.st_lo;
                        const T* q1 = whole ? p0 + (long long)gl * a.out_su
                                            : p0 + (long long)r * a.out_su + a.st_hi + 1;
                        uintptr_t i0, i1;
                        interior(reinterpret_cast<uintptr_t>(q0), reinterpret_cast<uintptr_t>(q1), i0, i1);
                        if (i1 > i0) bulk_store(reinterpret_cast<void*>(i0), sb + (i0 - base), (uint32_t)(i1 - i0));
                    }
                }
            }
            asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
            if (i + kStages < nloc) {
                // the buffer is refilled once the stores have read it
                asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
                issue_load(i + kStages);
            }
        }
        asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
        tma::drain_loads(full, nloc, kStages, wait_limit, flags);
        return;
    }

    // ---------------- compute ----------------
    // group gi holds lines gi W .. gi W + W - 1 of each tile.  With two groups
    // warp q of a group takes slots q, q + 4, q + 8, q + 12 (eight lines per
    // slot): on the row-major span (odd pitch) each bank is then hit exactly
    // twice by an instruction; with one group, lanes 0-15 / 16-31 are the 16
    // lines of two consecutive slots.
    const int gi = t / GNT, tl = t % GNT;
    const int c = (G == 1) ? tl % W : (tl & 7);
    const int slot = (G == 1) ? tl / W : (tl >> 5) + 4 * ((tl & 31) >> 3);
    T* const gred = red + gi * CF::RED;
    const double sc = a.use_scale ? a.scale : 1.0;
    // The boundary terms at xs and xe of a tile's rows off the y and z
    // boundaries (one (row, side) per thread of the row's group) are one
    // global value each (a face entry of f or a Neumann array) times a
    // coefficient: the value of tile i + 1 is loaded while tile i is
    // transformed, so its latency never stalls the group's barrier.  A single
    // term is exactly v + coef * value, as bc_terms applies it.
    struct BcNext {
        int row = -1, l = 0;
        double coef = 0.0;
        const double* p = nullptr;
    };
    auto bc_next = [&](int i) {
        BcNext q;
        if (!a.has_bc || i >= nloc) return q;
        const BcArgs& b = a.bc;
        int ub, v, nl;
        tile_of(i, ub, v, nl);
        if (v == b.zs || v == b.ze || tl >= 2 * group_lines(nl, gi)) return q;
        const int r = tl >> 1, j = ub + gi * W + r;   // r: line of the group
        if (j == b.ys || j == b.ye || ((tl & 1) && b.xe == b.xs)) return q;
        const long long row_f = (long long)v * (b.nx + 1) * (b.ny + 1) + (long long)j * (b.nx + 1);
        const long long row_face = (long long)v * (b.ny + 1) + j;
        if (!(tl & 1)) {   // i == xs
            if (b.xbc == 1 || b.xbc == 2) { q.p = b.f + row_f; q.coef = -b.dx2; }
            else if (b.xbc == 3 || b.xbc == 4) { q.p = b.bcl + row_face; q.coef = 2.0 * b.dx; }
            q.l = b.xs;
        } else {           // i == xe
            if (b.xbc == 1 || b.xbc == 4) { q.p = b.f + row_f + b.nx; q.coef = -b.dx2; }
            else if (b.xbc == 2 || b.xbc == 3) { q.p = b.bcr + row_face; q.coef = -2.0 * b.dx; }
            q.l = b.xe;
        }
        if (q.p) q.row = r;
        return q;
    };
    BcNext bnext = bc_next(0);
    double bnext_val = bnext.p ? __ldg(bnext.p) : 0.0;
    for (int i = 0; i < nloc; ++i) {
        const int s = i % kStages;
        int ub, v, nl;
        tile_of(i, ub, v, nl);
        const int ug = ub + gi * W;              // first line of the group
        const int gl = group_lines(nl, gi);      // its lines in this tile
        const bool bzrow = a.has_bc && (v == a.bc.zs || v == a.bc.ze);
        const BcNext bcur = bnext;
        const double bcur_val = bnext_val;
        bnext = bc_next(i + 1);
        bnext_val = bnext.p ? __ldg(bnext.p) : 0.0;
        if (!mbar_wait(full + s, (uint32_t)((i / kStages) & 1), abort, wait_limit)) {
            if (t == 0) atomicOr(flags, kFlagConsumer);
        }
        T* buf = region_of(s, gi);
        const int off = (LDM == kLdSpan) ? span_at(in_row0(ug, v)).off : 0;
        // entry l of line r (of the group) of the loaded real view
        auto at = [&](int l, int r) -> T& {
            if constexpr (LDM == kLdSpan) return buf[off + r * (int)a.in_su + l];
            else return buf[swz<BS>(l, r)];
        };
        bool fix = false;
        // entries of the kind's input window outside the load window are 0
        // (only those entries are visited: one or two per line)
        {
            const int nlo = a.ld_lo > LO ? a.ld_lo - LO : 0;
            const int nhi = HI > a.ld_hi ? HI - a.ld_hi : 0;
            if (nlo + nhi > 0) {
                for (int e = tl; e < W * (nlo + nhi); e += GNT) {
                    const int r = e % W, q = e / W;
                    at(q < nlo ? LO + q : a.ld_hi + 1 + (q - nlo), r) = T(0);
                }
                fix = true;
            }
        }
        if (a.has_bc) {
            // boundary terms: every entry of a row on a y or z boundary (read
            // here), else the prefetched term at xs or xe
            const BcArgs& b = a.bc;
            for (int r = 0; r < gl; ++r) {
                const int j = ug + r;
                if (!(bzrow || j == b.ys || j == b.ye)) continue;
                for (int l = a.ld_lo + tl; l <= a.ld_hi; l += GNT) at(l, r) = (T)bc_terms((double)at(l, r), b, l, j, v);
            }
            if (bcur.row >= 0) at(bcur.l, bcur.row) = (T)((double)at(bcur.l, bcur.row) + bcur.coef * bcur_val);
            fix = true;
        }
        if (fix) CF::sync();
        T* outp = nullptr;
        int offo = 0;
        if constexpr (STM == kStRows) {
            outp = out_row0(ug, v);
            offo = span_at(outp).off;
        }
        auto run = [&](const auto& X) {
            if constexpr (STM == kStTensor) {
                SwzSink<T, BS> sink{buf, c};
                transform_lines_v<T, CF, KIND>(X, buf, gred, c, slot, tb, sink);
            } else {
                RowSink<T> sink{buf + offo + c * (int)a.out_su, sc};
                transform_lines_v<T, CF, KIND>(X, buf, gred, c, slot, tb, sink);
            }
        };
        if constexpr (LDM == kLdSpan) run(RowView<T>{buf + off + c * (int)a.in_su});
        else run(CF::reader(static_cast<const T*>(buf), c));
        if constexpr (STM == kStRows) {
            // the 8-byte ends of the rows' windows that the aligned bulk
            // stores leave out: (row, side) per thread of the row's group
            const bool whole = a.st_lo == 0 && a.st_hi == a.out_su - 1;
            const int nrow = whole ? 1 : gl;
            for (int e = tl; e < 2 * nrow; e += GNT) {
                const int r = e >> 1;
                const int rl = (whole && (e & 1)) ? gl - 1 : r;           // row of the end
                const int l = (e & 1) ? a.st_hi : a.st_lo;
                T* q = outp + (long long)rl * a.out_su + l;
                const uintptr_t qa = reinterpret_cast<uintptr_t>(q);
                // left end: not on a 16-byte boundary; right end: its end not on one
                const bool edge = (e & 1) ? ((qa + sizeof(T)) & 15) != 0 : (qa & 15) != 0;
                if (edge && gl > 0) *q = buf[offo + rl * (int)a.out_su + l];
            }
        }
        // make this thread's writes visible to the bulk / tensor stores, then release
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive(ready + s);
    }
}

}  // namespace xtma
}  // namespace chz
