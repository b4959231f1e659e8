// Warp-local form of the TMA-pipelined contiguous (x) pass, FP64.
//
// Tiles and copies are those of xtma_pass: 16 lines (rows) of one plane per
// tile, three stages filled by one producer thread; an input on a
// 16-byte-aligned array arrives by 16 x 16 tensor boxes in the 128-byte
// swizzled layout, an input on the solver's f (rows of N + 1 values, 8-byte
// aligned) as one bulk span, row-major.  What differs is who transforms a
// line and where its results go:
//
//  * the P = M/16 threads of a line are consecutive lanes of ONE warp (32/P
//    lines per warp), so every exchange of the line transform stays inside
//    the warp: __syncwarp in place of CTA barriers, and the warps of a CTA run
//    through their lines independently (one warp's FP64 stages overlap
//    another's shared-memory exchanges and a third's stores);
//  * the complex exchange view of a line lies in the line's own storage
//    (swizzled: entries 2m, 2m + 1 of line c are one 16-byte chunk of row c;
//    row-major: from the line's first 16-byte boundary), so no line's
//    exchange touches another line's input;
//  * the outputs leave from registers: each thread stores its output entries
//    straight to global memory, inside the pass's output window (16-byte
//    stores of entry pairs where the row is 16-byte aligned), so there is no
//    output staging and no store copy, and a stage goes back to the producer
//    as soon as its lines have been read.
#pragma once
#include "chz_xtma.cuh"

namespace chz {
namespace xtma {

// The exchanges of a line transform write bins 16 j + k from lane j and read
// bins j + 16 k into lane j (and the partners M - m): in a line's own
// storage both strides would put every lane on one bank.  Bin m is therefore
// kept at slot m ^ ((m >> 4) & 7) of the line's 16-byte slots -- the low three
// bits (the bank group of a 16-byte slot in a 128-byte row) mixed with bits
// 4..6 -- which stays inside the line and spreads either access pattern over
// all eight bank groups.
__device__ __forceinline__ int zslot(int m) { return m ^ ((m >> 4) & 7); }

// Exchange view of line c of a swizzled tile: 16-byte slot q of the line is
// the chunk of its entries 2q, 2q + 1.
template <typename T>
struct SwzZ {
    C2<T>* base;  // tile as complex values + 8 c
    int c7;       // c mod 8
    __device__ __forceinline__ C2<T>& operator[](int m) const {
        const int q = zslot(m);
        return base[((q >> 3) << 7) + ((q & 7) ^ c7)];
    }
};

// Exchange view of a row-major line: 16-byte slots from the line's first
// 16-byte boundary (the line holds at least 2M + 1 entries, so M slots fit).
template <typename T>
struct RowZ {
    C2<T>* base;
    __device__ __forceinline__ C2<T>& operator[](int m) const { return base[zslot(m)]; }
};

// Butterfly j of stage S taken by lane `slot` as its b-th: j = slot + P b (the
// reads j + nb k of the lanes of a line are then consecutive for every b).
template <int M, int S>
struct WBfly {
    using BF = fast::Bfly<M, S>;
    static constexpr int r = BF::r, Ns = BF::Ns, B = BF::B, nb = BF::nb, P = M / fast::kR;
    __device__ static __forceinline__ int j(int slot, int b) { return slot + P * b; }
    __device__ static __forceinline__ int in_idx(int slot, int b, int k) { return j(slot, b) + k * nb; }
    __device__ static __forceinline__ int out_idx(int slot, int b, int k) {
        const int jj = j(slot, b);
        const int p = jj & (Ns - 1);
        return (jj - p) * r + p + k * Ns;
    }
};

// Stage twiddles and radix-r butterflies for the WBfly assignment.  The
// lanes of a line run different butterflies, so the last stage (Ns = 16)
// reads its twiddles w^(p k) from tw2[(k - 1) * 16 + p], a table the kernel
// lays out once: for each k the 16 lanes read 16 consecutive entries (from
// twM their stride p k would put up to 16 lanes on one bank).
template <typename T, int M, int S>
__device__ __forceinline__ void stage_compute_w(C2<T>* v, int slot, const C2<T>* __restrict__ tw2) {
    using BF = WBfly<M, S>;
    constexpr int r = BF::r;
    static_assert(BF::Ns == 1 || BF::Ns == 16, "stages of M = 128 and 256");
#pragma unroll
    for (int b = 0; b < BF::B; ++b) {
        if constexpr (BF::Ns > 1) {
            const int p = BF::j(slot, b) & (BF::Ns - 1);
#pragma unroll
            for (int k = 1; k < r; ++k) v[b * r + k] = cmul<T>(v[b * r + k], ldtw<T>(tw2 + (k - 1) * 16 + p));
        }
        fast::dft_r<T, r>(v + b * r);
    }
}

// Shared-memory carve-up of the warp-local pass: xtma_pass's, with the
// last-stage twiddle table in place of the DCT-I partial sums and one
// barrier per stage.
template <typename T, int M>
struct XWSmem {
    using BASE = XSmem<T, M>;
    static constexpr int R1 = WBfly<M, XCfg<M>::NST - 1>::r;
    static constexpr size_t stage = BASE::stage;
    static constexpr size_t twM = BASE::twM, twN = BASE::twN, tw4N = BASE::tw4N, inv4sin = BASE::inv4sin;
    static constexpr size_t tw2 = BASE::red;
    static constexpr size_t bars = (tw2 + sizeof(C2<T>) * (R1 - 1) * 16 + 15) & ~size_t(15);
    static constexpr size_t abort = bars + kStages * sizeof(uint64_t);
    static constexpr size_t total = abort + 16 + 1024;  // + alignment slack
};

// One real transform of one line by its P lanes: the real input is read
// through X, the line's storage is then reused through Z for the exchanges,
// and the outputs go to `sink` as they are formed.  The same pre steps,
// radix-16 stages and post steps as fast::transform_lines_v; the DCT-I sum of
// odd entries is reduced over the line's lanes by shuffles.
template <typename T, int M, int KIND, typename V, typename ZV, typename SINK>
__device__ __forceinline__ void line_transform_w(const V& X, const ZV& Z, int slot, const LineTables<T>& tb,
                                                 const C2<T>* __restrict__ tw2, const SINK& sink) {
    constexpr int R = fast::kR;
    constexpr int P = M / R;
    constexpr int N = 2 * M;
    constexpr int NST = fast::Cfg<M>::NST;
    constexpr bool FWD = (KIND == kR2C || KIND == kDCT2 || KIND == kDST2);
    C2<T> v[R];

    T acc = T(0);
    if constexpr (KIND == kDCT1) {
#pragma unroll
        for (int q = 0; q < M / P; ++q) {
            if constexpr (V::kPair) acc += X.pair(2 * (slot + q * P)).y;
            else acc += X(2 * (slot + q * P) + 1);
        }
    }
    {
        using BF = WBfly<M, 0>;
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = fast::pre_value<T, KIND, M>(X, BF::in_idx(slot, 0, k), tb);
    }
    if constexpr (KIND == kDCT1) {
#pragma unroll
        for (int o = P / 2; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    }
    __syncwarp();   // the real view is read: the storage now holds the exchange view
    stage_compute_w<T, M, 0>(v, slot, tw2);

#define CHZ_WSTAGE(S)                                                                                    \
    if constexpr (NST > S) {                                                                             \
        using PB = WBfly<M, S - 1>;                                                                       \
        _Pragma("unroll") for (int b = 0; b < PB::B; ++b)                                                \
            _Pragma("unroll") for (int k = 0; k < PB::r; ++k) Z[PB::out_idx(slot, b, k)] = v[b * PB::r + k]; \
        __syncwarp();                                                                                    \
        using BF = WBfly<M, S>;                                                                           \
        _Pragma("unroll") for (int b = 0; b < BF::B; ++b)                                                \
            _Pragma("unroll") for (int k = 0; k < BF::r; ++k) v[b * BF::r + k] = Z[BF::in_idx(slot, b, k)]; \
        __syncwarp();                                                                                    \
        stage_compute_w<T, M, S>(v, slot, tw2);                                                   \
    }
    CHZ_WSTAGE(1)
    CHZ_WSTAGE(2)
#undef CHZ_WSTAGE

    using LB = WBfly<M, NST - 1>;
    if constexpr (FWD || KIND == kDCT1 || KIND == kDST1) {
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) Z[LB::out_idx(slot, b, k)] = v[b * LB::r + k];
        __syncwarp();
    }
    if constexpr (FWD) {
        // V[m] = 1/2 (Z[m] + conj Z[M-m]) - i/2 w^m (Z[m] - conj Z[M-m])
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) {
                const int m = LB::out_idx(slot, b, k);
                const C2<T> zk = v[b * LB::r + k];
                const C2<T> zm = Z[(M - m) & (M - 1)];
                const C2<T> wk = ldtw<T>(tb.twN + m);
                const C2<T> e = cadd<T>(zk, cconj<T>(zm));
                const C2<T> o = cmul<T>(wk, csub<T>(zk, cconj<T>(zm)));
                const C2<T> V = mk<T>(T(0.5) * (e.x + o.y), T(0.5) * (e.y - o.x));
                const C2<T> vM = mk<T>(zk.x - zk.y, T(0));   // used at m = 0
                if constexpr (KIND == kR2C) {
                    sink.put_pair(2 * m, V.x, m == 0 ? T(0) : V.y);
                    if (m == 0) sink.put_pair(N, vM.x, T(0));
                } else {
                    const C2<T> a = cmul<T>(ldtw<T>(tb.tw4N + m), V);
                    if constexpr (KIND == kDCT2) {
                        sink.put(m, a.x);
                        if (m > 0) sink.put(N - m, -a.y);
                    } else {  // DST2
                        sink.put(N - m, a.x);
                        if (m > 0) sink.put(m, -a.y);
                        else sink.put(0, T(0));
                    }
                    if (m == 0) {
                        const C2<T> aM = cmul<T>(ldtw<T>(tb.tw4N + M), vM);
                        sink.put(M, aM.x);
                    }
                }
            }
    } else if constexpr (KIND == kDCT1 || KIND == kDST1) {
        // v[n] = Re conj(Z[n/2]) (n even), Im conj(Z[n/2]) (n odd); pairs (k, N-k)
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) {
                const int m = LB::out_idx(slot, b, k);
                const C2<T> z = v[b * LB::r + k];
                const T ve = z.x, vo = -z.y;  // v[2m], v[2m+1]
                T oe;
                if (m == 0) {
                    if constexpr (KIND == kDCT1) {
                        const T h = T(0.5) * ve;
                        oe = h + acc;
                        sink.put(N, h - acc);
                    } else {
                        oe = T(0);
                    }
                } else {
                    const T pe = Z[M - m].x;  // v[N-2m]
                    const T is4 = ldr<T>(tb.inv4sin + (2 * m <= M ? 2 * m : N - 2 * m));
                    if constexpr (KIND == kDCT1) oe = ((ve + pe) * T(0.5) - (ve - pe) * is4) * T(0.5);
                    else oe = ((ve + pe) * is4 + (ve - pe) * T(0.5)) * T(0.5);
                }
                const T po = -Z[M - m - 1].y;  // v[N-2m-1]
                const int ko = 2 * m + 1;
                const T is4o = ldr<T>(tb.inv4sin + (ko <= M ? ko : N - ko));
                T oo;
                if constexpr (KIND == kDCT1) oo = ((vo + po) * T(0.5) - (vo - po) * is4o) * T(0.5);
                else oo = ((vo + po) * is4o + (vo - po) * T(0.5)) * T(0.5);
                sink.put2(2 * m, oe, oo);
            }
    } else {
        // C2R, DCT3, DST3: outputs straight from the thread's own values
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) {
                const int m = LB::out_idx(slot, b, k);
                const C2<T> z = v[b * LB::r + k];
                const T v0 = z.x, v1 = -z.y;
                const int e0 = 2 * m, e1 = 2 * m + 1;
                if constexpr (KIND == kC2R) {
                    sink.put2(e0, v0, v1);
                } else if constexpr (KIND == kDCT3) {
                    sink.put(e0 < M ? 2 * e0 : 2 * (N - 1 - e0) + 1, T(0.5) * v0);
                    sink.put(e1 < M ? 2 * e1 : 2 * (N - 1 - e1) + 1, T(0.5) * v1);
                } else {  // DST3
                    if (e0 < M) sink.put(2 * e0 + 1, T(0.5) * v0);
                    else sink.put(2 * (N - 1 - e0) + 2, T(-0.5) * v0);
                    if (e1 < M) sink.put(2 * e1 + 1, T(0.5) * v1);
                    else sink.put(2 * (N - 1 - e1) + 2, T(-0.5) * v1);
                    if (m == 0) sink.put(0, T(0));
                }
            }
    }
}

// LDM: kLdTensor -- the input moves by 16 x 16 tensor boxes (ldmap, swizzled
// layout); kLdSpan -- by one bulk copy of the tile's rows (row-major, rows of
// a.in_su >= N + 1 values).  The output rows (a.out_su values apart, 8-byte
// aligned) receive the window [a.st_lo, a.st_hi] of every line, scaled by
// a.scale when a.use_scale.
//
// There is no producer warp: thread 0 issues the first kStages loads, and the
// warp that is last to finish reading a stage (a shared-memory count per
// stage) issues the load that refills it.  The CTA is then NT threads, two
// warps per SM sub-partition, and the transform has up to 255 registers a
// thread (a ninth warp would put three warps on one sub-partition and cap
// them at 168).
template <typename T, int M, int KIND, int LDM>
__global__ void __launch_bounds__(XCfg<M>::NT, (M <= 128 ? 2 : 1))
xw_pass(const __grid_constant__ CUtensorMap ldmap, const T* in, T* out, PassArgs a, LineTables<T> tg, XGeom g,
        int ntx, int ntiles, int* flags, long long wait_limit) {
    using CF = XCfg<M>;
    using SL = XWSmem<T, M>;
    constexpr int W = CF::W, NT = CF::NT, N = CF::N, P = CF::P;
    constexpr int LO = fast::InWin<KIND, N>::lo, HI = fast::InWin<KIND, N>::hi;
    extern __shared__ __align__(128) unsigned char smem_dyn[];
    const int t = threadIdx.x;
    if ((int)blockIdx.x >= ntiles) return;
    // the 128-byte swizzle needs 1024-byte-aligned boxes (1 KB of slack is allocated)
    unsigned char* smem_raw = smem_dyn + ((1024u - (saddr(smem_dyn) & 1023u)) & 1023u);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + SL::bars);
    volatile int* abort = reinterpret_cast<volatile int*>(smem_raw + SL::abort);
    __shared__ int s_read[kStages];   // warps done reading each stage, over all its uses
    constexpr int NW = NT / 32;

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
    // last-stage twiddles by (k, butterfly): w^(p k) of the M-point transform
    C2<T>* tw2 = reinterpret_cast<C2<T>*>(smem_raw + SL::tw2);
    for (int i = t; i < (SL::R1 - 1) * 16; i += blockDim.x) {
        const int k = i / 16 + 1, p = i % 16;
        tw2[i] = tg.twM[p * k * (M / (16 * SL::R1))];
    }
    if (t == 0) {
        *abort = 0;
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full + s, 1);
            s_read[s] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    const int nloc = (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;
    auto stage_of = [&](int s) { return reinterpret_cast<T*>(smem_raw + (size_t)s * SL::stage); };
    // tile i of this CTA: first line ub, plane v, lines nl
    auto tile_of = [&](int i, int& ub, int& v, int& nl) {
        const int tile = (int)blockIdx.x + i * (int)gridDim.x;
        ub = a.u0 + (tile % ntx) * W;
        v = a.v0 + tile / ntx;
        nl = min(W, a.u0 + a.nu - ub);
    };
    auto in_row0 = [&](int ub, int v) { return in + (long long)v * a.in_sv + (long long)ub * a.in_su; };

    auto issue_load = [&](int i) {
        const int s = i % kStages;
        int ub, v, nl;
        tile_of(i, ub, v, nl);
        T* dst = stage_of(s);
        if constexpr (LDM == kLdTensor) {
            mbar_expect_tx(full + s, (uint32_t)(g.ld_nblk * 256 * sizeof(T)));
            for (int q = 0; q < g.ld_nblk; ++q) {
                const int blk = g.ld_blk0 + q;
                tma_load(dst + blk * 256, &ldmap, blk * 16, ub, v - g.v_off, full + s);
            }
        } else {
            // rows ub .. ub + nl - 1, whole, as one span widened to 16 bytes
            const T* p0 = in_row0(ub, v);
            const Span sp = span_at(p0);
            const uintptr_t end = (reinterpret_cast<uintptr_t>(p0 + (long long)nl * a.in_su) + 15) & ~uintptr_t(15);
            const uint32_t bytes = (uint32_t)(end - sp.a0);
            mbar_expect_tx(full + s, bytes);
            bulk_load(dst, reinterpret_cast<const void*>(sp.a0), bytes, full + s);
        }
    };
    if (t == 0) {
        if constexpr (LDM == kLdTensor)
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&ldmap)) : "memory");
        const int pre = nloc < kStages ? nloc : kStages;
        for (int i = 0; i < pre; ++i) issue_load(i);
    }

    // ---------------- compute: line c of every tile, by P lanes of one warp ----------------
    const int lane = t & 31;
    const int c = (t >> 5) * (32 / P) + lane / P;
    const int slot = lane % P;
    const T sc = (T)(a.use_scale ? a.scale : 1.0);
    // Boundary terms at xs and xe of a line off the y and z boundaries: one
    // global value times a coefficient, loaded one tile ahead by the line's
    // lanes 0 (xs) and 1 (xe).
    struct BcNext {
        int l = -1;
        double coef = 0.0;
        const double* p = nullptr;
    };
    // (a pass with a tensor input carries no boundary terms: the launch
    // sends those to the CTA-wide form)
    auto bc_next = [&](int i) {
        BcNext q;
        if (LDM != kLdSpan || !a.has_bc || i >= nloc || slot > 1) return q;
        const BcArgs& b = a.bc;
        int ub, v, nl;
        tile_of(i, ub, v, nl);
        if (v == b.zs || v == b.ze || c >= nl) return q;
        const int j = ub + c;
        if (j == b.ys || j == b.ye || (slot == 1 && b.xe == b.xs)) return q;
        const long long row_f = (long long)v * (b.nx + 1) * (b.ny + 1) + (long long)j * (b.nx + 1);
        const long long row_face = (long long)v * (b.ny + 1) + j;
        if (slot == 0) {   // i == xs
            if (b.xbc == 1 || b.xbc == 2) { q.p = b.f + row_f; q.coef = -b.dx2; }
            else if (b.xbc == 3 || b.xbc == 4) { q.p = b.bcl + row_face; q.coef = 2.0 * b.dx; }
            q.l = b.xs;
        } else {           // i == xe
            if (b.xbc == 1 || b.xbc == 4) { q.p = b.f + row_f + b.nx; q.coef = -b.dx2; }
            else if (b.xbc == 2 || b.xbc == 3) { q.p = b.bcr + row_face; q.coef = -2.0 * b.dx; }
            q.l = b.xe;
        }
        if (!q.p) q.l = -1;
        return q;
    };
    BcNext bnext = bc_next(0);
    double bnext_val = bnext.p ? __ldg(bnext.p) : 0.0;
    const int nlo = a.ld_lo > LO ? a.ld_lo - LO : 0;
    const int nhi = HI > a.ld_hi ? HI - a.ld_hi : 0;
    for (int i = 0; i < nloc; ++i) {
        const int s = i % kStages;
        int ub, v, nl;
        tile_of(i, ub, v, nl);
        const BcNext bcur = bnext;
        const double bcur_val = bnext_val;
        bnext = bc_next(i + 1);
        bnext_val = bnext.p ? __ldg(bnext.p) : 0.0;
        if (!mbar_wait(full + s, (uint32_t)((i / kStages) & 1), abort, wait_limit)) {
            if (t == 0) atomicOr(flags, kFlagConsumer);
        }
        T* buf = stage_of(s);
        const bool on = c < nl;
        const int e = (LDM == kLdSpan) ? span_at(in_row0(ub, v)).off + c * (int)a.in_su : 0;
        // entry l of this line in the loaded real view
        auto at = [&](int l) -> T& {
            if constexpr (LDM == kLdSpan) return buf[e + l];
            else return buf[swz(l, c)];
        };
        // entries of the kind's input window outside the load window are 0
        for (int q = slot; q < nlo + nhi; q += P) at(q < nlo ? LO + q : a.ld_hi + 1 + (q - nlo)) = T(0);
        if (LDM == kLdSpan && a.has_bc) {
            // boundary terms: every entry of a row on a y or z boundary (read
            // here), else the prefetched term at xs or xe
            const BcArgs& b = a.bc;
            const int j = ub + c;
            if (on && (v == b.zs || v == b.ze || j == b.ys || j == b.ye))
                for (int l = a.ld_lo + slot; l <= a.ld_hi; l += P) at(l) = (T)bc_terms((double)at(l), b, l, j, v);
            if (bcur.l >= 0) at(bcur.l) = (T)((double)at(bcur.l) + bcur.coef * bcur_val);
        }
        __syncwarp();
        T* orow = out + (long long)v * a.out_sv + (long long)(ub + c) * a.out_su;
        const GSink<T> sink{orow, a.st_lo, a.st_hi, sc, (reinterpret_cast<uintptr_t>(orow) & 15) == 0, on};
        if constexpr (LDM == kLdSpan) {
            line_transform_w<T, M, KIND>(RowView<T>{buf + e}, RowZ<T>{reinterpret_cast<C2<T>*>(buf + e + (e & 1))},
                                         slot, tb, tw2, sink);
        } else {
            line_transform_w<T, M, KIND>(SwzView<T>{buf + (c << 4), c & 7},
                                         SwzZ<T>{reinterpret_cast<C2<T>*>(buf) + (c << 3), c & 7}, slot, tb, tw2,
                                         sink);
        }
        // the stage is read: the last warp to finish it refills it with tile
        // i + kStages (every warp counts once per use of the stage)
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            const int prev = atomicAdd(&s_read[s], 1);
            if (prev == (i / kStages + 1) * NW - 1 && i + kStages < nloc) {
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                issue_load(i + kStages);
            }
        }
    }
    // no copy into this CTA's shared memory may be in flight when it exits
    // (after a normal run every phase is already complete)
    if (t == 0) tma::drain_loads(full, nloc, kStages, wait_limit, flags);
}

}  // namespace xtma
}  // namespace chz
