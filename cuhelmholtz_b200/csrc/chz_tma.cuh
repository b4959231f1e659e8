// TMA-pipelined line pass for the strided axes (y and z passes).
//
// A tile is W adjacent x columns (128 bytes: 16 FP64 or 32 FP32 values) of
// the lines of one plane; a line runs along y or z.  One producer thread
// moves whole tiles with cp.async.bulk.tensor: loads land in one of S stage
// buffers (row l of the tile at shared row l, so the kind's input window is
// addressed directly; rows the pass does not load are filled with zeros by
// the copy engine, which also zero-fills columns past the last line), and
// finished tiles leave by bulk tensor stores clipped to the output window.
// The compute warps run the register-resident radix-16 line transform of
// chz_fast.cuh on the stage buffer in place, synchronised by a named barrier
// that leaves the producer warp out, so loads run up to S - 1 tiles ahead of
// the compute and stores drain behind it.
//
// Every entry of a 128-byte row is read or written by the W threads of one
// slot at once, so all shared accesses of the real view are bank-conflict
// free; the complex exchange view Z[m * W + c] is two rows per entry.  The
// fused z pass of the solver at N = 512 (forward real DFT, division, inverse)
// keeps the spectrum in registers between the two transforms
// (r2c_div_c2r_regs).
//
// Waits are bounded: a wait that runs out sets a flag that the host reads
// (chz_stream_status, chz_debug_flags) and the thread carries on, so the
// kernel always ends; before it ends the producer waits (bounded as well) for
// the last load of every stage, so no copy into the CTA's shared memory is in
// flight when it exits.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "chz_fast.cuh"

namespace chz {
namespace tma {

using fast::LineCfg;
using fast::OutSink;
using fast::transform_lines;

template <typename T>
struct TileW {
    static constexpr int W = 128 / (int)sizeof(T);
};

template <typename T, int M>
using TCfg = LineCfg<M, TileW<T>::W, TileW<T>::W, 1>;

// The DCT/DST tables (tw4N, inv4sin) are staged in shared memory only for
// passes that use them.
template <int KIND, int KIND2>
struct UsesDctTables {
    static constexpr bool dft(int k) { return k == kR2C || k == kC2R; }
    static constexpr bool value = !dft(KIND) || (KIND2 >= 0 && !dft(KIND2));
};

constexpr int kStages = 3;

// Stage buffers of the strided pass: three for the power-of-two lengths; two
// for the mixed ones, so that two CTAs fit an SM at N = 320.
template <int M>
constexpr int tma_stages() { return (M & (M - 1)) == 0 ? kStages : 2; }

// Host-computed geometry of one pass.
struct TmaGeom {
    int rows_buf;     // rows of one stage buffer
    int ld_row0;      // shared row of the first loaded row
    int ld_coord0;    // its line coordinate in the load map
    int ld_nch;       // boxes per tile load
    int ld_box;       // rows per load box
    int st_row0;      // shared row of the first stored row
    int st_nch;       // boxes per tile store
    int st_box;       // rows per store box
    int l_mid;        // 1: map dims (u, l, v); 0: (u, v, l)
    unsigned tx_bytes;  // bytes one tile load delivers
    int col0;         // u of map column 0
    int v_off;        // v of the maps' first plane (the maps start at the first plane the pass reads)
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(b)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(saddr(b)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete.  Gives up after
// `limit` SM clock cycles (the host sets it: about a second by default), or
// at once when another thread of the CTA has given up (*abort), so a CTA
// whose copies never arrive still ends quickly.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort, long long limit) {
    const uint32_t a = saddr(b);
    const long long t0 = clock64();
    while (true) {
        if (mbar_try(a, parity)) return true;
        if (*abort || clock64() - t0 > limit) {
            *abort = 1;
            return false;
        }
    }
}

// The producer's last wait before the CTA ends: the phase of the last load
// issued into a stage, waited for whether or not the CTA has given up, so no
// copy into this CTA's shared memory is still in flight when it exits (after
// a normal run the phase is already complete).  Bounded by `limit` too.
__device__ __forceinline__ bool mbar_drain(uint64_t* b, uint32_t parity, long long limit) {
    const uint32_t a = saddr(b);
    const long long t0 = clock64();
    while (!mbar_try(a, parity)) {
        if (clock64() - t0 > limit) return false;
    }
    return true;
}

// The producer's drain: for every stage that received loads, the phase of
// the last load issued into it (tile i of this CTA loads stage i % kStages).
__device__ __forceinline__ void drain_loads(uint64_t* full, int nloc, int stages, long long limit, int* flags) {
    for (int s = 0; s < stages && s < nloc; ++s) {
        const int last = s + ((nloc - 1 - s) / stages) * stages;
        if (!mbar_drain(full + s, (uint32_t)((last / stages) & 1), limit)) atomicOr(flags, kFlagDrain);
    }
}

__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store(const CUtensorMap* map, int c0, int c1, int c2, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(saddr(src))
                 : "memory");
}

// The fused forward / division / inverse pass of N = 512 and N = 256 lines
// (M = 256: radix 16 x 16; M = 128: radix 16 x 8) with the spectrum kept in
// registers.  With P = M / 16 threads a line, after the forward stages thread
// `slot` holds bins m = slot + P k (k = 0..15) -- for M = 128 the last stage
// takes butterflies slot and slot + 8 to make it so -- which are exactly the
// inverse's first-stage inputs.  The split, the division and the inverse's
// pre step need each bin with its partner M - m, held by slot P - slot.  Slots
// are paired in warps (paired_slot): warp w >= 1 holds w and P - w, warp 0
// the self-paired 0 and P / 2.  Each pair (m, M - m) is finished once: a thread
// of warps 1.. takes the partner's bin of its k < 8 by shuffle, produces the
// inverse inputs of both bins, keeps its own and hands the partner its, so
// the spectrum never returns to shared memory.
template <typename T, int M, int WT, int KIND, int KIND2>
struct RegSpectrum {
    static constexpr bool value = (M == 256 || M == 128) && WT == 16 && KIND == kR2C && KIND2 == kC2R;
};

template <int P>
__device__ __forceinline__ int paired_slot(int t) {
    const int w = t >> 5, h = (t >> 4) & 1;
    return w == 0 ? (P / 2) * h : (h ? P - w : w);
}

// Pair (m, M - m) of the fused R2C / division / C2R pass, from Z[m] = zk,
// Z[M - m] = zm: the R2C split gives X[m] and X[M - m] (w^(M-m) = -conj w^m),
// each is divided by its eigenvalue, and the C2R pre step gives the inverse
// inputs at m (o1) and M - m (o2, the conjugate sums of o1's).  m = 0 pairs
// bin 0 with the Nyquist bin M (o2 is then not an input).
template <typename T, int N, typename DSINK>
__device__ __forceinline__ void split_div_pre(int m, C2<T> zk, C2<T> zm, C2<T>& o1, C2<T>& o2,
                                              const LineTables<T>& tb, const DSINK& dv) {
    const C2<T> wk = ldtw<T>(tb.twN + m);
    if (m != 0 && 2 * m >= dv.dlo && 2 * m + 1 <= dv.dhi && N - 2 * m >= dv.dlo && N - 2 * m + 1 <= dv.dhi) {
        // The split, the two divisions and the pre step compose into one
        // real-linear map of (zk, zm).  With s = zk + conj zm,
        // t = zk - conj zm, w = w^m = wr + i wi, dm, dp the reciprocal
        // eigenvalues of bins m and M - m: X[m] = (s - i w t) / 2,
        // X[M - m] = conj(s + i w t) / 2, and the pre step of the divided
        // pair gives (|w| = 1)
        //   o1 = ((dm + dp) + (dm - dp) wi) conj zk - i (dm - dp) wr zm
        //   o2 = ((dm + dp) - (dm - dp) wi) conj zm - i (dm - dp) wr zk.
        const T dm = (T)dv.eig(2 * m), dp = (T)dv.eig(N - 2 * m);
        const T sum = dm + dp, dif = dm - dp;
        const T c1 = sum + dif * wk.y, c2 = sum - dif * wk.y, g = dif * wk.x;
        o1 = mk<T>(c1 * zk.x + g * zm.y, -(c1 * zk.y + g * zm.x));
        o2 = mk<T>(c2 * zm.x + g * zk.y, -(c2 * zm.y + g * zk.x));
        return;
    }
    const C2<T> e = cadd<T>(zk, cconj<T>(zm));
    const C2<T> od = cmul<T>(wk, csub<T>(zk, cconj<T>(zm)));
    C2<T> a = mk<T>(T(0.5) * (e.x + od.y), T(0.5) * (e.y - od.x));    // X[m]
    C2<T> b = mk<T>(T(0.5) * (e.x - od.y), T(-0.5) * (e.y + od.x));   // X[M - m]
    int lb = N - 2 * m;
    if (m == 0) {
        a = mk<T>(zk.x + zk.y, T(0));
        b = mk<T>(zk.x - zk.y, T(0));
        lb = N;
    }
    dv.div_pair(2 * m, a);
    dv.div_pair(lb, b);
    const C2<T> e2 = cadd<T>(a, cconj<T>(b));
    const C2<T> o2c = cmul<T>(cconj<T>(wk), csub<T>(a, cconj<T>(b)));
    o1 = cconj<T>(cadd<T>(e2, cmul_i<T>(o2c)));
    o2 = cconj<T>(cadd<T>(cconj<T>(e2), cmul_i<T>(cconj<T>(o2c))));
}

template <typename T, typename CF, typename DSINK>
__device__ __forceinline__ void r2c_div_c2r_regs(T* buf, int c, int slot, bool partner_in_warp,
                                                 const LineTables<T>& tb, const DSINK& dv) {
    constexpr int M = CF::M, N = CF::N, PR = CF::PR, P = CF::P;
    static_assert((M == 256 || M == 128) && CF::W == 16, "M = 256 or 128, 16-line tiles");
    using B0 = fast::Bfly<M, 0>;
    using B1 = fast::Bfly<M, 1>;
    constexpr int R = fast::kR;
    const auto X = CF::reader(static_cast<const T*>(buf), c);
    C2<T>* Z = reinterpret_cast<C2<T>*>(buf);
    C2<T> v[R];

    // forward: stage 0 with the pre step in the reads, exchange, stage 1
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = fast::pre_value<T, kR2C, M>(X, B0::in_idx(slot, 0, k), tb);
    CF::sync();
    fast::stage_compute<T, M, 0>(v, slot, tb.twM);
#pragma unroll
    for (int k = 0; k < R; ++k) Z[CF::zi(B0::out_idx(slot, 0, k), c)] = v[k];
    CF::sync();
    // u[k] = Z[slot + P k] after the last forward stage
    C2<T> u[R];
    if constexpr (M == 256) {
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = Z[CF::zi(B1::in_idx(slot, 0, k), c)];
        CF::sync();
        fast::stage_compute<T, M, 1>(v, slot, tb.twM);
#pragma unroll
        for (int k = 0; k < R; ++k) u[k] = v[k];
    } else {
        // radix 8 (Ns = 16, nb = 16) on butterflies j = slot + 8 b: inputs
        // j + 16 k, twiddles w^(j k), outputs j + 16 k = slot + 8 (b + 2 k)
        static_assert(B1::r == 8 && B1::Ns == 16 && B1::nb == 16, "M = 128: last stage radix 8");
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int k = 0; k < 8; ++k) v[b * 8 + k] = Z[CF::zi(slot + 8 * b + 16 * k, c)];
        CF::sync();
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int j = slot + 8 * b;
#pragma unroll
            for (int k = 1; k < 8; ++k) v[b * 8 + k] = cmul<T>(v[b * 8 + k], ldtw<T>(tb.twM + j * k));
            fast::dft_r<T, 8>(v + b * 8);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) u[k] = v[(k & 1) * 8 + (k >> 1)];
    }

    auto pair = [&](int m, C2<T> zk, C2<T> zm, C2<T>& o1, C2<T>& o2) {
        split_div_pre<T, N>(m, zk, zm, o1, o2, tb, dv);
    };

    // Iteration k finishes bin k with its partner: lane ^ 16's u[15 - k]
    // (warps 1..), own u[15 - k] (slot P / 2), own u[(16 - k) mod 16] (slot 0).
    // Warps 1.. touch only u[0..7] here, so the partner's shuffles of u[8..15]
    // always see the forward values.
    C2<T> send[R / 2];
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
        C2<T> q;
        q.x = __shfl_xor_sync(0xffffffffu, u[R - 1 - k].x, 16);
        q.y = __shfl_xor_sync(0xffffffffu, u[R - 1 - k].y, 16);
        const int i2 = (slot == 0) ? ((R - k) & (R - 1)) : (R - 1 - k);   // own partner index (warp 0)
        const C2<T> own = (slot == 0) ? u[(R - k) & (R - 1)] : u[R - 1 - k];
        C2<T> o1, o2;
        pair(slot + P * k, u[k], partner_in_warp ? q : own, o1, o2);
        u[k] = o1;
        send[k] = o2;
        if (!partner_in_warp && k > 0) {
            // warp 0: the partner bin is this thread's own (index i2 > k)
#pragma unroll
            for (int j = R / 2; j < R; ++j)
                if (j == i2) u[j] = o2;
        } else if (!partner_in_warp && slot == P / 2) {
            u[R - 1] = o2;   // k = 0 of slot P / 2: partner index 15
        }
    }
    if (slot == 0) {   // bin M / 2 pairs with itself
        C2<T> o1, o2;
        pair(M / 2, u[R / 2], u[R / 2], o1, o2);
        u[R / 2] = o1;
    }
    // hand each partner its bins: my send[k] is the partner's u[15 - k]
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
        C2<T> r;
        r.x = __shfl_xor_sync(0xffffffffu, send[k].x, 16);
        r.y = __shfl_xor_sync(0xffffffffu, send[k].y, 16);
        if (partner_in_warp) u[R - 1 - k] = r;
    }

    // inverse: stage 0 (inputs slot + P k = u[k]), exchange, stage 1, real
    // outputs x[2m] = Re, x[2m+1] = -Im
    fast::stage_compute<T, M, 0>(u, slot, tb.twM);
#pragma unroll
    for (int k = 0; k < R; ++k) Z[CF::zi(B0::out_idx(slot, 0, k), c)] = u[k];
    CF::sync();
#pragma unroll
    for (int b = 0; b < B1::B; ++b)
#pragma unroll
        for (int k = 0; k < B1::r; ++k) u[b * B1::r + k] = Z[CF::zi(B1::in_idx(slot, b, k), c)];
    CF::sync();
    fast::stage_compute<T, M, 1>(u, slot, tb.twM);
#pragma unroll
    for (int b = 0; b < B1::B; ++b)
#pragma unroll
        for (int k = 0; k < B1::r; ++k) {
            const int m = B1::out_idx(slot, b, k);
            buf[(2 * m) * PR + c] = u[b * B1::r + k].x;
            buf[(2 * m + 1) * PR + c] = -u[b * B1::r + k].y;
        }
}

// The fused pass of N = 512 and 256 lines with 32-line tiles (FP32): one warp holds
// one slot of all 32 lines, so a bin's partner M - m (held by slot P - slot)
// is in another warp and the pair exchange goes through shared memory -- but
// only the half of the spectrum the partners need: after the forward stages
// (thread `slot` holds bins slot + P k, k = 0..15) every thread publishes its
// bins k = 8..15, reads the partner bin of each of its k < 8, finishes both
// bins of the pair, keeps its own and writes the partner's into the partner's
// published slot, from which the partner reads its k = 8..15 back.  Slot 0
// pairs with itself (bin 0 with the Nyquist bin, bin M / 2 alone), slot P / 2
// too; the same reads and writes serve them.  The spectrum never makes the
// full round trip of the unfused post / pre steps.
template <typename T, int M, int WT, int KIND, int KIND2>
struct SmemSpectrum {
    static constexpr bool value = (M == 256 || M == 128) && WT == 32 && KIND == kR2C && KIND2 == kC2R;
};

template <typename T, typename CF, typename DSINK>
__device__ __forceinline__ void r2c_div_c2r_smem(T* buf, int c, int slot, const LineTables<T>& tb,
                                                 const DSINK& dv) {
    constexpr int M = CF::M, N = CF::N, PR = CF::PR, P = CF::P;
    static_assert((M == 256 || M == 128) && CF::W == 32, "M = 256 or 128, 32-line tiles");
    using B0 = fast::Bfly<M, 0>;
    using B1 = fast::Bfly<M, 1>;
    constexpr int R = fast::kR;
    const auto X = CF::reader(static_cast<const T*>(buf), c);
    C2<T>* Z = reinterpret_cast<C2<T>*>(buf);
    C2<T> u[R];

    // forward: stage 0 with the pre step in the reads, exchange, stage 1
#pragma unroll
    for (int k = 0; k < R; ++k) u[k] = fast::pre_value<T, kR2C, M>(X, B0::in_idx(slot, 0, k), tb);
    CF::sync();
    fast::stage_compute<T, M, 0>(u, slot, tb.twM);
#pragma unroll
    for (int k = 0; k < R; ++k) Z[CF::zi(B0::out_idx(slot, 0, k), c)] = u[k];
    CF::sync();
    if constexpr (M == 256) {
#pragma unroll
        for (int k = 0; k < R; ++k) u[k] = Z[CF::zi(B1::in_idx(slot, 0, k), c)];
        CF::sync();
        fast::stage_compute<T, M, 1>(u, slot, tb.twM);
    } else {
        // radix 8 on butterflies j = slot + 8 b (as r2c_div_c2r_regs), so that
        // this thread's outputs are bins slot + 8 k
        static_assert(B1::r == 8 && B1::Ns == 16 && B1::nb == 16, "M = 128: last stage radix 8");
        C2<T> v[R];
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int k = 0; k < 8; ++k) v[b * 8 + k] = Z[CF::zi(slot + 8 * b + 16 * k, c)];
        CF::sync();
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int j = slot + 8 * b;
#pragma unroll
            for (int k = 1; k < 8; ++k) v[b * 8 + k] = cmul<T>(v[b * 8 + k], ldtw<T>(tb.twM + j * k));
            fast::dft_r<T, 8>(v + b * 8);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) u[k] = v[(k & 1) * 8 + (k >> 1)];
    }
    // u[k] = bin slot + P k; publish the upper half
#pragma unroll
    for (int k = R / 2; k < R; ++k) Z[CF::zi(slot + P * k, c)] = u[k];
    CF::sync();
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
        const int m = slot + P * k;
        const C2<T> zm = (m == 0) ? u[0] : Z[CF::zi(M - m, c)];
        C2<T> o1, o2;
        split_div_pre<T, N>(m, u[k], zm, o1, o2, tb, dv);
        u[k] = o1;
        if (m != 0) Z[CF::zi(M - m, c)] = o2;
    }
    if (slot == 0) {   // bin M / 2 pairs with itself
        C2<T> o1, o2;
        split_div_pre<T, N>(M / 2, u[R / 2], u[R / 2], o1, o2, tb, dv);
        Z[CF::zi(M / 2, c)] = o1;
    }
    CF::sync();
#pragma unroll
    for (int k = R / 2; k < R; ++k) u[k] = Z[CF::zi(slot + P * k, c)];
    CF::sync();

    // inverse: stage 0 (inputs slot + P k = u[k]), exchange, stage 1, real
    // outputs x[2m] = Re, x[2m+1] = -Im
    fast::stage_compute<T, M, 0>(u, slot, tb.twM);
#pragma unroll
    for (int k = 0; k < R; ++k) Z[CF::zi(B0::out_idx(slot, 0, k), c)] = u[k];
    CF::sync();
#pragma unroll
    for (int b = 0; b < B1::B; ++b)
#pragma unroll
        for (int k = 0; k < B1::r; ++k) u[b * B1::r + k] = Z[CF::zi(B1::in_idx(slot, b, k), c)];
    CF::sync();
    fast::stage_compute<T, M, 1>(u, slot, tb.twM);
#pragma unroll
    for (int b = 0; b < B1::B; ++b)
#pragma unroll
        for (int k = 0; k < B1::r; ++k) {
            const int m = B1::out_idx(slot, b, k);
            buf[(2 * m) * PR + c] = u[b * B1::r + k].x;
            buf[(2 * m + 1) * PR + c] = -u[b * B1::r + k].y;
        }
}

// Shared-memory carve-up (byte offsets).
template <typename T, int M, bool FUSED, bool DCTTAB = true>
struct TmaSmem {
    using CF = TCfg<T, M>;
    static constexpr int NS = tma_stages<M>();
    __host__ __device__ static constexpr size_t al(size_t b, size_t a) { return (b + a - 1) / a * a; }
    __host__ __device__ static size_t stage_bytes(int rows_buf) { return (size_t)rows_buf * CF::W * sizeof(T); }
    __host__ __device__ static size_t twM(int rows_buf) { return al(NS * stage_bytes(rows_buf), 128); }
    __host__ __device__ static size_t twN(int rows_buf) { return twM(rows_buf) + sizeof(C2<T>) * M; }
    __host__ __device__ static size_t tw4N(int rows_buf) { return twN(rows_buf) + sizeof(C2<T>) * (M + 1); }
    __host__ __device__ static size_t inv4sin(int rows_buf) {
        return tw4N(rows_buf) + (DCTTAB ? sizeof(C2<T>) * (M + 1) : 0);
    }
    __host__ __device__ static size_t ez(int rows_buf) {
        return al(inv4sin(rows_buf) + (DCTTAB ? sizeof(T) * (M + 1) : 0), 16);
    }
    __host__ __device__ static size_t red(int rows_buf) {
        return al(ez(rows_buf) + (FUSED ? sizeof(double) * (2 * M + 2) : 0), 16);
    }
    __host__ __device__ static size_t bars(int rows_buf) { return al(red(rows_buf) + sizeof(T) * CF::RED, 16); }
    __host__ __device__ static size_t abort(int rows_buf) { return bars(rows_buf) + 2 * NS * sizeof(uint64_t); }
    __host__ __device__ static size_t total(int rows_buf) { return abort(rows_buf) + 16; }
};

// CTAs per SM asked of the compiler: one at N = 512 (the pipeline's shared
// memory allows no more), four at N = 128 (three warps a CTA, 50 KB), two
// elsewhere.  Registers are allocated per SM sub-partition: two CTAs of five
// warps (or four of three) put three warps on some sub-partitions, so a
// thread may hold at most 168 (3 x 32 x 168 <= 16384), which these block
// counts ask of the compiler.
// The FP32 pass at N = 320 (nine warps, 20 values a thread) keeps one CTA
// per SM: two would leave it 113 registers and spill.
template <typename T, int M>
constexpr int tma_min_ctas() {
    return M >= 256 ? 1 : (M <= 64 ? 4 : ((sizeof(T) == 4 && M == 160) ? 1 : 2));
}

template <typename T, int M, int KIND, int KIND2>
__global__ void __launch_bounds__(TCfg<T, M>::NT + 32, tma_min_ctas<T, M>())
tma_pass(const __grid_constant__ CUtensorMap ldmap, const __grid_constant__ CUtensorMap stmap, PassArgs a,
         LineTables<T> tg, TmaGeom g, int ntx, int ntiles, int* flags, long long wait_limit) {
    using CF = TCfg<T, M>;
    constexpr bool DCTTAB = UsesDctTables<KIND, KIND2>::value;
    using SL = TmaSmem<T, M, (KIND2 >= 0), DCTTAB>;
    constexpr int W = CF::W, PR = CF::PR, NT = CF::NT, N = CF::N;
    constexpr int NS = SL::NS;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int t = threadIdx.x;
    if ((int)blockIdx.x >= ntiles) return;
    if (saddr(smem_raw) & 127) {  // uniform over the CTA: nothing has started
        if (t == 0) atomicOr(flags, kFlagAlign);
        return;
    }
    const int rb = g.rows_buf;
    const size_t sbytes = SL::stage_bytes(rb);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + SL::bars(rb));
    uint64_t* ready = full + NS;
    volatile int* abort = reinterpret_cast<volatile int*>(smem_raw + SL::abort(rb));
    T* red = reinterpret_cast<T*>(smem_raw + SL::red(rb));

    LineTables<T> tb = tg;
    {
        C2<T>* sM = reinterpret_cast<C2<T>*>(smem_raw + SL::twM(rb));
        C2<T>* sN = reinterpret_cast<C2<T>*>(smem_raw + SL::twN(rb));
        C2<T>* s4 = reinterpret_cast<C2<T>*>(smem_raw + SL::tw4N(rb));
        T* sI = reinterpret_cast<T*>(smem_raw + SL::inv4sin(rb));
        for (int i = t; i < M; i += blockDim.x) sM[i] = tg.twM[i];
        for (int i = t; i <= M; i += blockDim.x) {
            sN[i] = tg.twN[i];
            if constexpr (DCTTAB) {
                s4[i] = tg.tw4N[i];
                sI[i] = tg.inv4sin[i];
            }
        }
        tb.twM = sM;
        tb.twN = sN;
        if constexpr (DCTTAB) {
            tb.tw4N = s4;
            tb.inv4sin = sI;
        }
    }
    double* ez_s = reinterpret_cast<double*>(smem_raw + SL::ez(rb));
    if constexpr (KIND2 >= 0) {
        for (int i = t; i < N + 2; i += blockDim.x) ez_s[i] = a.dv.ez[i];
    }
    if (t == 0) {
        *abort = 0;
        for (int s = 0; s < NS; ++s) {
            mbar_init(full + s, 1);
            mbar_init(ready + s, NT);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    const int nloc = (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1;

    if (t >= NT) {
        // ---------------- producer ----------------
        if (t != NT) return;
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&ldmap)) : "memory");
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&stmap)) : "memory");
        auto issue_load = [&](int i) {
            const int s = i % NS;
            const int tile = (int)blockIdx.x + i * (int)gridDim.x;
            const int cx = (tile % ntx) * W;
            const int v = a.v0 + tile / ntx - g.v_off;   // map coordinate
            unsigned char* dst = smem_raw + (size_t)s * sbytes;
            mbar_expect_tx(full + s, g.tx_bytes);
            for (int q = 0; q < g.ld_nch; ++q) {
                const int l = g.ld_coord0 + q * g.ld_box;
                void* d = dst + (size_t)(g.ld_row0 + q * g.ld_box) * W * sizeof(T);
                if (g.l_mid) tma_load(d, &ldmap, cx, l, v, full + s);
                else tma_load(d, &ldmap, cx, v, l, full + s);
            }
        };
        const int pre = nloc < NS ? nloc : NS;
        for (int i = 0; i < pre; ++i) issue_load(i);
        for (int i = 0; i < nloc; ++i) {
            const int s = i % NS;
            if (!mbar_wait(ready + s, (uint32_t)((i / NS) & 1), abort, wait_limit))
                atomicOr(flags, kFlagProducer);
            const int tile = (int)blockIdx.x + i * (int)gridDim.x;
            const int cx = (tile % ntx) * W;
            const int v = a.v0 + tile / ntx - g.v_off;   // map coordinate
            const unsigned char* src = smem_raw + (size_t)s * sbytes;
            for (int q = 0; q < g.st_nch; ++q) {
                const int l = q * g.st_box;
                const void* sp = src + (size_t)(g.st_row0 + q * g.st_box) * W * sizeof(T);
                if (g.l_mid) tma_store(&stmap, cx, l, v, sp);
                else tma_store(&stmap, cx, v, l, sp);
            }
            asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
            if (i + NS < nloc) {
                // the buffer is refilled once the store has read it
                asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
                issue_load(i + NS);
            }
        }
        asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
        drain_loads(full, nloc, NS, wait_limit, flags);
        return;
    }

    // ---------------- compute ----------------
    constexpr bool REGSPEC = RegSpectrum<T, M, W, KIND, KIND2>::value;
    const int c = t % W;
    const int slot = REGSPEC ? paired_slot<CF::P>(t) : t / W;
    for (int i = 0; i < nloc; ++i) {
        const int s = i % NS;
        if (!mbar_wait(full + s, (uint32_t)((i / NS) & 1), abort, wait_limit)) {
            if (t == 0) atomicOr(flags, kFlagConsumer);
        }
        T* buf = reinterpret_cast<T*>(smem_raw + (size_t)s * sbytes);
        const int tile = (int)blockIdx.x + i * (int)gridDim.x;
        const int v = a.v0 + tile / ntx;
        if constexpr (KIND2 >= 0) {
            OutSink<T, PR, true> s1;
            s1.Rv = buf;
            s1.c = c;
            int col = g.col0 + (tile % ntx) * W + c;
            col = max(a.u0, min(col, a.u0 + a.nu - 1));
            s1.exy = __ldg(a.dv.ex + col) + __ldg(a.dv.ey + v);
            s1.lam = a.dv.lambda;
            s1.ez = ez_s;
            s1.dlo = a.dv.lo;
            s1.dhi = a.dv.hi;
            s1.zmax = (a.dv.perturb && col <= a.dv.xz_hi && v <= a.dv.yz_hi) ? a.dv.zz_hi : -1;
            if constexpr (REGSPEC) {
                r2c_div_c2r_regs<T, CF>(buf, c, slot, (t >> 5) != 0, tb, s1);
            } else if constexpr (SmemSpectrum<T, M, W, KIND, KIND2>::value) {
                r2c_div_c2r_smem<T, CF>(buf, c, slot, tb, s1);
            } else {
                transform_lines<T, CF, KIND>(buf, red, c, slot, tb, s1);
                OutSink<T, PR, false> s2;
                s2.Rv = buf;
                s2.c = c;
                transform_lines<T, CF, KIND2>(buf, red, c, slot, tb, s2);
            }
        } else {
            OutSink<T, PR, false> sk;
            sk.Rv = buf;
            sk.c = c;
            transform_lines<T, CF, KIND>(buf, red, c, slot, tb, sk);
        }
        // make this thread's writes visible to the bulk store, then release
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_arrive(ready + s);
    }
}

}  // namespace tma
}  // namespace chz
