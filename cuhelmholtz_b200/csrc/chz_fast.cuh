// Register-resident line-pass kernel for half lengths M = N/2 with a
// compile-time radix plan: the powers of two 16 .. 512 (N = 32 .. 1024) and a
// set of mixed lengths (M = 12 .. 192 with factors 3, 5, 7).
//
// * Each line is transformed by P = M/V threads; every thread keeps V complex
//   values in registers (V = 16 for the powers of two: radix-16 butterflies,
//   radix 2/4/8 for the last factor; V = 10 .. 20 for the mixed lengths, whose
//   radices -- 10, 12, 14, 18, 20 and 2, 4 -- are computed in registers as
//   nested small DFTs) between shared-memory exchanges (Stockham order).  The
//   kind's pre step is fused into the first stage's reads, the post step reads
//   only the partner values each output needs, and in the fused solver pass
//   the eigenvalue division is applied while the forward post step writes.
// * The transform kind (and the inverse kind of a fused pass) are template
//   parameters, so every index, window bound and branch is resolved at
//   compile time.
// * CTAs are persistent: each stages its line tables in shared memory once and
//   loops over tiles of W lines; a tile is loaded with cp.async (every copy in
//   flight at once) and several CTAs per SM overlap one another's loads, FFT
//   work and stores.
// One tile buffer of (N+2) x (W+1) values holds, in turn, the real input view,
// the complex FFT view and the real output view; phases are separated by
// barriers.
#pragma once
#include <type_traits>
#include <utility>

#include "chz_device.cuh"
#include "chz_internal.h"

namespace chz {
namespace fast {

constexpr int kNT = 128;  // threads per CTA
constexpr int kR = 16;    // complex values per thread of the power-of-two plans

// Radix plan of one half length M: V complex values per thread and the radix
// of each Stockham stage (every radix divides V, their product is M).  Powers
// of two: radix 16 stages, then the remaining factor 2, 4 or 8.
template <int M>
struct Plan {
    static_assert(M >= 16 && (M & (M - 1)) == 0, "no radix plan for this length");
    static constexpr int V = kR;
    static constexpr int A16 = (M >= 256) ? 2 : 1;
    static constexpr int R0 = M / (A16 == 2 ? 256 : 16);
    static constexpr int NST = A16 + (R0 > 1 ? 1 : 0);
    __host__ __device__ static constexpr int radix(int s) { return s < A16 ? 16 : R0; }
};
template <int V_, int R0_, int R1_ = 1, int R2_ = 1, int R3_ = 1>
struct MixedPlan {
    static constexpr int V = V_;
    static constexpr int NST = 1 + (R1_ > 1) + (R2_ > 1) + (R3_ > 1);
    __host__ __device__ static constexpr int radix(int s) {
        return s == 0 ? R0_ : s == 1 ? R1_ : s == 2 ? R2_ : R3_;
    }
};
// The mixed lengths: P = M / V threads a line divides the 128 threads of a CTA.
template <> struct Plan<12> : MixedPlan<12, 12> {};
template <> struct Plan<20> : MixedPlan<10, 10, 2> {};
template <> struct Plan<24> : MixedPlan<12, 12, 2> {};
template <> struct Plan<28> : MixedPlan<14, 14, 2> {};
template <> struct Plan<40> : MixedPlan<10, 10, 2, 2> {};
template <> struct Plan<48> : MixedPlan<12, 12, 4> {};
template <> struct Plan<56> : MixedPlan<14, 14, 2, 2> {};
template <> struct Plan<72> : MixedPlan<18, 18, 2, 2> {};
template <> struct Plan<80> : MixedPlan<20, 20, 4> {};
template <> struct Plan<96> : MixedPlan<12, 12, 4, 2> {};
template <> struct Plan<160> : MixedPlan<20, 20, 4, 2> {};
template <> struct Plan<192> : MixedPlan<12, 12, 4, 4> {};

// Geometry of a tile of W lines transformed by P = M/V threads each: the real
// view of entry l of line c is buf[l * PR + c], the complex view of entry m is
// Z[m * W + c] (rows permuted with ZPERM, below).  BAR = 0 synchronises the
// CTA with __syncthreads; BAR > 0 uses named barrier BAR over the NT compute
// threads only.
template <int M_, int W_, int PR_, int BAR_, bool ZPERM = false>
struct LineCfg {
    static constexpr int M = M_;
    static constexpr int V = Plan<M>::V;  // values per thread
    static constexpr int P = M / V;       // threads per line
    static constexpr int W = W_;          // lines per tile
    static constexpr int NT = P * W;      // compute threads
    static constexpr int N = 2 * M;
    static constexpr int L = N + 2;       // padded line
    static constexpr int PR = PR_;        // real-view pitch
    static constexpr int BAR = BAR_;
    static constexpr int NST = Plan<M>::NST;
    static constexpr int BUF = ((L * PR) + 3) & ~3;   // elements per tile buffer (>= 2*M*W)
    static constexpr int RED = P * W;      // DCT1 odd-sum partials
    __device__ static __forceinline__ void sync() {
        if constexpr (BAR == 0) __syncthreads();
        else asm volatile("bar.sync %0, %1;\n" ::"n"(BAR), "n"(NT) : "memory");
    }
    // real view of line c: reader(buf, c)(l) = buf[l * PR + c]; complex view Z[zi(m, c)]
    template <typename T>
    __device__ static __forceinline__ StridedView<T> reader(const T* buf, int c) {
        return StridedView<T>{buf, PR, c};
    }
    // ZPERM (8 lines, FP32): a row m of the exchange view is then half a bank
    // cycle (8 x 8 bytes), and the four slot groups of a warp (slots w + 4 j in
    // the contiguous passes) access rows of one parity, so they would share 16
    // banks.  Rows m and m ^ 1 trade places when bits 2 and 6 of m differ: a
    // permutation of the rows that puts two of the groups on each half for the
    // stage exchanges (rows 16 slot + k written, slot + 16 k read) and the
    // partner reads.  Measured faster only where the pass waits on shared
    // memory (the accumulating FP32 x inverse: 0.686 -> 0.603 ms a launch under
    // ncu); the issue-bound FP32 x forward from FP64 input slowed down with it
    // (0.628 -> 0.795 ms), so only the former uses it.
    __device__ static __forceinline__ int zi(int m, int c) {
        if constexpr (ZPERM && W == 8) return (m ^ (((m >> 2) ^ (m >> 6)) & 1)) * W + c;
        else return m * W + c;
    }
};

// The persistent cp.async kernel: 128 threads, odd pitch W + 1 (conflict-free
// transposed access).
template <int M>
using Cfg = LineCfg<M, kNT / (M / Plan<M>::V), kNT / (M / Plan<M>::V) + 1, 0>;
// The same with the exchange rows permuted (the accumulating FP32 x inverse).
template <int M>
using CfgPerm = LineCfg<M, kNT / (M / Plan<M>::V), kNT / (M / Plan<M>::V) + 1, 0, true>;

#define CHZ_C1 0.92387953251128675613
#define CHZ_S1 0.38268343236508977173

template <typename T>
__device__ __forceinline__ C2<T> cmulc(C2<T> a, T wr, T wi) {
    return mk<T>(a.x * wr - a.y * wi, a.x * wi + a.y * wr);
}

// forward radix-16 DFT (4 x 4 with internal twiddles) on v[0..15]
template <typename T>
__device__ __forceinline__ void dft16(C2<T>* v) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<T>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    const T c1 = T(CHZ_C1), s1 = T(CHZ_S1), r = T(CHZ_SQRT_HALF);
    // v[n2 + 4 k1] *= w16^(n2 k1)
    v[5] = cmulc<T>(v[5], c1, -s1);    // t = 1
    v[6] = cmulc<T>(v[6], r, -r);      // t = 2
    v[7] = cmulc<T>(v[7], s1, -c1);    // t = 3
    v[9] = cmulc<T>(v[9], r, -r);      // t = 2
    v[10] = cmul_negi<T>(v[10]);       // t = 4
    v[11] = cmulc<T>(v[11], -r, -r);   // t = 6
    v[13] = cmulc<T>(v[13], s1, -c1);  // t = 3
    v[14] = cmulc<T>(v[14], -r, -r);   // t = 6
    v[15] = cmulc<T>(v[15], -c1, s1);  // t = 9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<T>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[4 k1 + k2] = X[k1 + 4 k2]: transpose 4 x 4
    C2<T> t[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
}

template <typename T, int r>
__device__ __forceinline__ void dft_r(C2<T>* v) {
    if constexpr (r == 16) dft16<T>(v);
    else if constexpr (r == 8) Dft<T, 8>::run(v, nullptr, 0);
    else if constexpr (r == 4) Dft<T, 4>::run(v, nullptr, 0);
    else if constexpr (r == 2) Dft<T, 2>::run(v, nullptr, 0);
}

// a * w_R^t (w_R = exp(-2 pi i / R)) with t a compile-time exponent: the
// eighth roots of unity in closed form, every other factor from the M-point
// table (w_R^t = twM[t M / R]; R divides M).
template <typename T, int R, int t, int M>
__device__ __forceinline__ C2<T> rot(C2<T> a, const C2<T>* __restrict__ twM) {
    constexpr int u = t % R;
    if constexpr (u == 0) return a;
    else if constexpr (4 * u == R) return cmul_negi<T>(a);
    else if constexpr (2 * u == R) return mk<T>(-a.x, -a.y);
    else if constexpr (4 * u == 3 * R) return cmul_i<T>(a);
    else if constexpr (8 * u == R) {
        const T r = T(CHZ_SQRT_HALF);
        return mk<T>(r * (a.x + a.y), r * (a.y - a.x));
    } else if constexpr (8 * u == 3 * R) {
        const T r = T(CHZ_SQRT_HALF);
        return mk<T>(r * (a.y - a.x), -r * (a.x + a.y));
    } else {
        return cmul<T>(a, ldtw<T>(twM + u * (M / R)));
    }
}

template <typename T, int R, int M>
__device__ __forceinline__ void dft_plan(C2<T>* v, const C2<T>* __restrict__ twM);

// Radix R = R1 R2 in registers (Cooley-Tukey): with n = R2 n1 + n2 and
// k = k1 + R1 k2, X[k] = sum_n2 w_R2^(n2 k2) w_R^(n2 k1) sum_n1 w_R1^(n1 k1) v[n].
// Column n2: the R1-point DFT of v[R2 n1 + n2], twiddled into a[k1 R2 + n2]
// (the exponents n2 k1 are template arguments, so the trivial ones fold).
template <typename T, int R1, int R2, int M, int n2, int... k1>
__device__ __forceinline__ void ct_twiddle(const C2<T>* u, C2<T>* a, const C2<T>* __restrict__ twM,
                                           std::integer_sequence<int, k1...>) {
    ((a[k1 * R2 + n2] = rot<T, R1 * R2, n2 * k1, M>(u[k1], twM)), ...);
}
template <typename T, int R1, int R2, int M, int n2>
__device__ __forceinline__ void ct_column(const C2<T>* v, C2<T>* a, const C2<T>* __restrict__ twM) {
    C2<T> u[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) u[n1] = v[R2 * n1 + n2];
    dft_plan<T, R1, M>(u, twM);
    ct_twiddle<T, R1, R2, M, n2>(u, a, twM, std::make_integer_sequence<int, R1>{});
}
template <typename T, int R1, int R2, int M, int... n2>
__device__ __forceinline__ void ct_columns(const C2<T>* v, C2<T>* a, const C2<T>* __restrict__ twM,
                                           std::integer_sequence<int, n2...>) {
    (ct_column<T, R1, R2, M, n2>(v, a, twM), ...);
}
template <typename T, int R1, int R2, int M>
__device__ __forceinline__ void dft_ct(C2<T>* v, const C2<T>* __restrict__ twM) {
    C2<T> a[R1 * R2];
    ct_columns<T, R1, R2, M>(v, a, twM, std::make_integer_sequence<int, R2>{});
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        C2<T> u[R2];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) u[n2] = a[k1 * R2 + n2];
        dft_plan<T, R2, M>(u, twM);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = u[k2];
    }
}

// Forward radix-R DFT of v[0..R-1] for any radix of a plan of length M.
template <typename T, int R, int M>
__device__ __forceinline__ void dft_plan(C2<T>* v, const C2<T>* __restrict__ twM) {
    if constexpr (R == 16 || R == 8 || R == 4 || R == 2) dft_r<T, R>(v);
    else if constexpr (R == 3) Dft<T, 3>::run(v, nullptr, 0);
    else if constexpr (R == 5 || R == 7 || R == 11 || R == 13) Dft<T, R>::run(v, twM, M);
    else if constexpr (R == 9) dft_ct<T, 3, 3, M>(v, twM);
    else if constexpr (R == 10) dft_ct<T, 2, 5, M>(v, twM);
    else if constexpr (R == 12) dft_ct<T, 4, 3, M>(v, twM);
    else if constexpr (R == 14) dft_ct<T, 2, 7, M>(v, twM);
    else if constexpr (R == 18) dft_ct<T, 2, 9, M>(v, twM);
    else if constexpr (R == 20) dft_ct<T, 4, 5, M>(v, twM);
    else static_assert(R == 16, "radix without a register DFT");
}

// Radix and Ns (product of the previous radices) of stage S.
template <int M, int S>
struct StageOf {
    __host__ __device__ static constexpr int ns() {
        int p = 1;
        for (int i = 0; i < S; ++i) p *= Plan<M>::radix(i);
        return p;
    }
    static constexpr int r = Plan<M>::radix(S);
    static constexpr int Ns = ns();
};

// Stockham butterfly bookkeeping for slot `slot`, butterfly b of stage S.
template <int M, int S>
struct Bfly {
    static constexpr int r = StageOf<M, S>::r;
    static constexpr int Ns = StageOf<M, S>::Ns;
    static constexpr int B = Plan<M>::V / r;
    static constexpr int nb = M / r;
    static_assert(B * r == Plan<M>::V, "every radix divides the values per thread");
    __device__ static __forceinline__ int j(int slot, int b) { return slot * B + b; }
    __device__ static __forceinline__ int in_idx(int slot, int b, int k) { return j(slot, b) + k * nb; }
    __device__ static __forceinline__ int out_idx(int slot, int b, int k) {
        const int jj = j(slot, b);
        const int p = jj % Ns;
        return (jj - p) * r + p + k * Ns;
    }
};

// Multiply by the stage twiddles and run the radix-r butterflies.
template <typename T, int M, int S>
__device__ __forceinline__ void stage_compute(C2<T>* v, int slot, const C2<T>* __restrict__ twM) {
    using BF = Bfly<M, S>;
    constexpr int r = BF::r;
#pragma unroll
    for (int b = 0; b < BF::B; ++b) {
        if constexpr (BF::Ns > 1) {
            const int p = BF::j(slot, b) % BF::Ns;
            constexpr int tstep = M / (BF::Ns * r);
#pragma unroll
            for (int k = 1; k < r; ++k) v[b * r + k] = cmul<T>(v[b * r + k], ldtw<T>(twM + p * k * tstep));
        }
        dft_plan<T, r, M>(v + b * r, twM);
    }
}

// Complex value A[n] fed to the FFT, from the real view (pre step); the kind
// is a compile-time constant so the gathers fold to fixed offsets.
template <typename T, int KIND, int M, typename V>
__device__ __forceinline__ C2<T> pre_value(const V& X, int n, const LineTables<T>& tb) {
    constexpr int N = 2 * M;
    if constexpr (KIND == kR2C && V::kPair) {
        return X.pair(2 * n);
    } else if constexpr (KIND == kR2C || KIND == kDCT2 || KIND == kDST2) {
        return mk<T>(fwd_gather_v<T>(KIND, X, 2 * n, N, M), fwd_gather_v<T>(KIND, X, 2 * n + 1, N, M));
    } else {
        const C2<T> vk = inv_spectrum_v<T>(KIND, X, n, N, M, tb);
        const C2<T> vm = inv_spectrum_v<T>(KIND, X, M - n, N, M, tb);
        const C2<T> wk = ldtw<T>(tb.twN + n);
        const C2<T> e = cadd<T>(vk, cconj<T>(vm));
        const C2<T> o = cmul<T>(cconj<T>(wk), csub<T>(vk, cconj<T>(vm)));
        return cconj<T>(cadd<T>(e, cmul_i<T>(o)));
    }
}

// Sink for real outputs of the post step; with DIV, values on the spectral
// window are divided by the Helmholtz eigenvalue as they are written.
template <typename T, int PR, bool DIV>
struct OutSink {
    T* Rv;
    int c;
    double exy, lam;  // ex[i] + ey[j], lambda
    const double* ez;
    int dlo, dhi;     // spectral window along the line
    int zmax;         // entries l <= zmax are zeroed (zero mode), else -1
    // 1 / (lambda_x + lambda_y + lambda_z[l] + lambda), 0 for the zero mode
    __device__ __forceinline__ double eig(int l) const {
        const double r = recip((exy + ez[l]) + lam);
        return l <= zmax ? 0.0 : r;
    }
    __device__ __forceinline__ void put(int l, T val) const {
        if constexpr (DIV) {
            if (l >= dlo && l <= dhi) val = (T)((double)val * eig(l));
        }
        Rv[l * PR + c] = val;
    }
    // Entries l, l + 1 of one complex bin of a periodic axis, which share the
    // eigenvalue (one reciprocal for both).
    __device__ __forceinline__ void put_pair(int l, T re, T im) const {
        if constexpr (DIV) {
            if (l >= dlo && l + 1 <= dhi) {
                const double e = eig(l);
                re = (T)((double)re * e);
                im = (T)((double)im * e);
            } else {
                put(l, re);
                put(l + 1, im);
                return;
            }
        }
        Rv[l * PR + c] = re;
        Rv[(l + 1) * PR + c] = im;
    }
    // Two adjacent entries, each with its own eigenvalue.
    __device__ __forceinline__ void put2(int l, T a, T b) const {
        put(l, a);
        put(l + 1, b);
    }
    // put_pair's division applied to a bin held in registers.
    __device__ __forceinline__ void div_pair(int l, C2<T>& v) const {
        if (l >= dlo && l + 1 <= dhi) {
            const double e = eig(l);
            v.x = (T)((double)v.x * e);
            v.y = (T)((double)v.y * e);
        } else {
            if (l >= dlo && l <= dhi) v.x = (T)((double)v.x * eig(l));
            if (l + 1 >= dlo && l + 1 <= dhi) v.y = (T)((double)v.y * eig(l + 1));
        }
    }
    __device__ static __forceinline__ double recip(double d) { return recip_nr(d); }
};

// One complete real transform of the W lines held in `buf`: the real input of
// line c is read through the view X (entry l: X(l)), the complex exchange view
// Z[m * W + c] reuses `buf` once every input is in registers, and the real
// output goes to `sink`.
template <typename T, typename CF, int KIND, typename V, typename SINK>
__device__ __forceinline__ void transform_lines_v(const V& X, T* buf, T* red, int c, int slot,
                                                  const LineTables<T>& tb, const SINK& sink) {
    constexpr int M = CF::M;
    constexpr int W = CF::W, N = CF::N, P = CF::P;
    constexpr bool FWD = (KIND == kR2C || KIND == kDCT2 || KIND == kDST2);
    constexpr int VPT = CF::V;
    C2<T>* Z = reinterpret_cast<C2<T>*>(buf);
    C2<T> v[VPT];

    // DCT1: partial sums of the odd entries x[1], x[3], ..., x[N-1] -- the
    // entries x[2n + 1] the pre step reads for this thread's inputs n, so the
    // partial sum is published only after those reads (no store between them
    // lets the compiler load each entry once)
    T acc = T(0), S = T(0);
    if constexpr (KIND == kDCT1) {
#pragma unroll
        for (int q = 0; q < M / P; ++q) {
            if constexpr (V::kPair) acc += X.pair(2 * (slot + q * P)).y;   // the pre step's own pair reads
            else acc += X(2 * (slot + q * P) + 1);
        }
    }

    // ---- stage 0: pre step fused into the reads ----
    {
        using BF = Bfly<M, 0>;
#pragma unroll
        for (int k = 0; k < VPT; ++k) v[k] = pre_value<T, KIND, M>(X, BF::in_idx(slot, 0, k), tb);
        if constexpr (KIND == kDCT1) red[slot * W + c] = acc;
        CF::sync();
        // DCT1: the line's odd-entry sum, by the thread of slot 0, while the
        // other warps run stage 0 (the partials stay until the next pre step)
        if constexpr (KIND == kDCT1) {
            if (slot == 0) {
#pragma unroll
                for (int q = 0; q < P; ++q) S += red[q * W + c];
            }
        }
        stage_compute<T, M, 0>(v, slot, tb.twM);
    }

    // ---- middle and last stages: write previous results, read this stage's inputs ----
#define CHZ_STAGE(S)                                                                          \
    if constexpr (CF::NST > S) {                                                              \
        using PB = Bfly<M, S - 1>;                                                            \
        _Pragma("unroll") for (int b = 0; b < PB::B; ++b)                                     \
            _Pragma("unroll") for (int k = 0; k < PB::r; ++k)                                 \
                Z[CF::zi(PB::out_idx(slot, b, k), c)] = v[b * PB::r + k];                        \
        CF::sync();                                                                      \
        using BF = Bfly<M, S>;                                                                \
        _Pragma("unroll") for (int b = 0; b < BF::B; ++b)                                     \
            _Pragma("unroll") for (int k = 0; k < BF::r; ++k)                                 \
                v[b * BF::r + k] = Z[CF::zi(BF::in_idx(slot, b, k), c)];                         \
        CF::sync();                                                                      \
        stage_compute<T, M, S>(v, slot, tb.twM);                                              \
    }
    static_assert(CF::NST <= 4, "at most four stages");
    CHZ_STAGE(1)
    CHZ_STAGE(2)
    CHZ_STAGE(3)
#undef CHZ_STAGE

    // ---- post step ----
    using LB = Bfly<M, CF::NST - 1>;
    if constexpr (FWD || KIND == kDCT1 || KIND == kDST1) {
        // publish Z, then read the partner entries
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) Z[CF::zi(LB::out_idx(slot, b, k), c)] = v[b * LB::r + k];
        CF::sync();
    }
    if constexpr (FWD) {
        // split: V[m] = 1/2 (Z[m] + conj Z[M-m]) - i/2 w^m (Z[m] - conj Z[M-m])
        C2<T> vM = mk<T>(T(0), T(0));
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) {
                const int m = LB::out_idx(slot, b, k);
                const C2<T> zk = v[b * LB::r + k];
                const C2<T> zm = Z[CF::zi(m == 0 ? 0 : M - m, c)];
                const C2<T> wk = ldtw<T>(tb.twN + m);
                const C2<T> e = cadd<T>(zk, cconj<T>(zm));
                const C2<T> o = cmul<T>(wk, csub<T>(zk, cconj<T>(zm)));
                v[b * LB::r + k] = mk<T>(T(0.5) * (e.x + o.y), T(0.5) * (e.y - o.x));
                if (m == 0) vM = mk<T>(zk.x - zk.y, T(0));
            }
        CF::sync();
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) {
                const int m = LB::out_idx(slot, b, k);
                const C2<T> V = v[b * LB::r + k];
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
        T outs[2 * VPT];
        T extra = T(0);  // out[N] (DCT1, m = 0)
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
                        oe = h + S;
                        extra = h - S;
                    } else {
                        oe = T(0);
                    }
                } else {
                    const T pe = Z[CF::zi(M - m, c)].x;  // v[N-2m]
                    const T is4 = ldr<T>(tb.inv4sin + (2 * m <= M ? 2 * m : N - 2 * m));
                    if constexpr (KIND == kDCT1) oe = ((ve + pe) * T(0.5) - (ve - pe) * is4) * T(0.5);
                    else oe = ((ve + pe) * is4 + (ve - pe) * T(0.5)) * T(0.5);
                }
                const T po = -Z[CF::zi(M - m - 1, c)].y;  // v[N-2m-1]
                const int ko = 2 * m + 1;
                const T is4o = ldr<T>(tb.inv4sin + (ko <= M ? ko : N - ko));
                T oo;
                if constexpr (KIND == kDCT1) oo = ((vo + po) * T(0.5) - (vo - po) * is4o) * T(0.5);
                else oo = ((vo + po) * is4o + (vo - po) * T(0.5)) * T(0.5);
                outs[2 * (b * LB::r + k)] = oe;
                outs[2 * (b * LB::r + k) + 1] = oo;
            }
        CF::sync();
#pragma unroll
        for (int b = 0; b < LB::B; ++b)
#pragma unroll
            for (int k = 0; k < LB::r; ++k) {
                const int m = LB::out_idx(slot, b, k);
                sink.put2(2 * m, outs[2 * (b * LB::r + k)], outs[2 * (b * LB::r + k) + 1]);
                if constexpr (KIND == kDCT1) {
                    if (m == 0) sink.put(N, extra);
                }
            }
    } else {
        // C2R, DCT3, DST3: outputs come straight from the thread's own values
        // (every thread passed the barrier after its last shared reads)
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
    CF::sync();
}

// The same with the configuration's own real view of `buf`.
template <typename T, typename CF, int KIND, typename SINK>
__device__ __forceinline__ void transform_lines(T* buf, T* red, int c, int slot, const LineTables<T>& tb,
                                                const SINK& sink) {
    transform_lines_v<T, CF, KIND>(CF::reader(static_cast<const T*>(buf), c), buf, red, c, slot, tb, sink);
}

template <int KIND, int N>
struct InWin {
    static constexpr int lo = (KIND == kDST1 || KIND == kDST2) ? 1 : 0;
    static constexpr int hi = (KIND == kDST1) ? N - 1
                            : (KIND == kDST2 || KIND == kDST3 || KIND == kDCT1) ? N
                            : (KIND == kC2R) ? N + 1 : N - 1;
};

template <typename TI>
__device__ __forceinline__ double ldin(const TI* p) { return (double)__ldg(p); }

// Issues the loads of one tile (cp.async when no conversion is needed) into
// `buf` and commits them as one group.
template <typename T, typename TI, int M, bool CONTIG, int KIND>
__device__ __forceinline__ void load_tile(T* buf, const TI* __restrict__ in, const PassArgs& a, int ub, int nl,
                                          int v, int t, int c, int slot) {
    using CF = Cfg<M>;
    constexpr int W = CF::W, PR = CF::PR, N = CF::N, P = CF::P;
    constexpr int LO = InWin<KIND, N>::lo, HI = InWin<KIND, N>::hi;
    const long long vb = (long long)v * a.in_sv;
    if constexpr (CONTIG) {
#pragma unroll 1
        for (int cc = 0; cc < W; ++cc) {
            const bool ok = cc < nl;
            const TI* row = in + vb + (long long)(ok ? ub + cc : ub) * a.in_su;
#pragma unroll
            for (int l = LO + t; l <= HI; l += kNT) {
                const bool valid = ok && l >= a.ld_lo && l <= a.ld_hi;
                if constexpr (sizeof(TI) == sizeof(T)) {
                    cp_async_elem<sizeof(T)>(&buf[l * PR + cc], valid ? row + l : in, valid);
                } else {
                    buf[l * PR + cc] = valid ? (T)ldin<TI>(row + l) : T(0);
                }
            }
        }
    } else {
        const bool ok = c < nl;
        const TI* p = in + vb + (long long)(ok ? ub + c : ub) * a.in_su + (long long)(LO + slot) * a.in_sl;
        const long long step = (long long)P * a.in_sl;
#pragma unroll
        for (int l = LO + slot; l <= HI; l += P) {
            const bool valid = ok && l >= a.ld_lo && l <= a.ld_hi;
            if constexpr (sizeof(TI) == sizeof(T)) {
                cp_async_elem<sizeof(T)>(&buf[l * PR + c], valid ? p : in, valid);
            } else {
                buf[l * PR + c] = valid ? (T)ldin<TI>(p) : T(0);
            }
            p += step;
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

// Contiguous FP32 passes with an FP64 output (the refinement's x inverse):
// the rows an accumulated output adds to are staged in shared memory by
// cp.async while the tile is transformed.
template <typename T, typename TO, bool CONTIG>
constexpr bool acc_staged() { return CONTIG && sizeof(T) == 4 && sizeof(TO) == 8; }

// Shared-memory footprint of one CTA (bytes): tile buffer, DCT1 partials,
// the line tables, for the fused pass the z eigenvalue table and, with ACC,
// the staged rows of an accumulated output (W rows of N + 2 FP64 values).
template <typename T, int M, bool FUSED, bool ACC = false>
struct SmemLayout {
    using CF = Cfg<M>;
    static constexpr size_t buf = 0;
    static constexpr size_t red = buf + sizeof(T) * CF::BUF;
    static constexpr size_t twM = (red + sizeof(T) * CF::RED + 15) & ~size_t(15);
    static constexpr size_t twN = twM + sizeof(C2<T>) * M;
    static constexpr size_t tw4N = twN + sizeof(C2<T>) * (M + 1);
    static constexpr size_t inv4sin = tw4N + sizeof(C2<T>) * (M + 1);
    static constexpr size_t ez = (inv4sin + sizeof(T) * (M + 1) + 15) & ~size_t(15);
    static constexpr size_t accb = (ez + (FUSED ? sizeof(double) * (2 * M + 2) : 0) + 15) & ~size_t(15);
    static constexpr size_t total = accb + (ACC ? sizeof(double) * CF::W * (2 * M + 2) : 0);
};

// Four CTAs per SM (128 registers a thread); three for plans of more than 16
// values a thread.
template <int M>
constexpr int fast_min_ctas() { return Plan<M>::V > kR ? 3 : 4; }

// One tile of a pass: load (cp.async), boundary terms, the line transforms
// (with the division of a fused pass) and the store.  `a` may live in the
// kernel's parameters or in shared memory (the batched kernel).
template <typename T, typename TI, typename TO, int M, bool CONTIG, int KIND, int KIND2>
__device__ __forceinline__ void fast_tile(const TI* in, TO* out, const PassArgs& a, const LineTables<T>& tb,
                                          const double* ez_s, T* buf, T* red, int tile, int ntx, int t, int c,
                                          int slot, double* accb = nullptr) {
    using CF = std::conditional_t<acc_staged<T, TO, CONTIG>(), CfgPerm<M>, Cfg<M>>;
    constexpr int W = CF::W, PR = CF::PR, P = CF::P, N = CF::N;
    constexpr bool ACCS = acc_staged<T, TO, CONTIG>();
    const int tx = tile % ntx;
    const int v = a.v0 + tile / ntx;
    const int ub = a.u0 + tx * W;
    const int nl = min(W, a.u0 + a.nu - ub);
    load_tile<T, TI, M, CONTIG, KIND>(buf, in, a, ub, nl, v, t, c, slot);
    // the rows an accumulated output adds to: a second copy group, waited
    // for only before the store, so its latency overlaps the transform
    bool staged = false;
    if constexpr (ACCS) {
        if (a.acc) {
            const long long vb = (long long)v * a.out_sv;
            for (int cc = 0; cc < nl; ++cc) {
                const double* arow = a.acc + vb + (long long)(ub + cc) * a.out_su;
                for (int l = a.st_lo + t; l <= a.st_hi; l += kNT)
                    cp_async_elem<8>(accb + cc * (N + 2) + l, arow + l, true);
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
            staged = true;
        }
    }
    if (staged) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();

    if (CONTIG && a.has_bc) {
        // boundary terms: every entry of a y/z boundary row; elsewhere the
        // entries at xs and xe (one thread applies all terms of an entry)
        const BcArgs& b = a.bc;
        const bool zrow = (v == b.zs || v == b.ze);
        // rows on a y or z boundary: every entry
        for (int cc = 0; cc < nl; ++cc) {
            const int j = ub + cc;
            if (zrow || j == b.ys || j == b.ye) {
                for (int l = a.ld_lo + t; l <= a.ld_hi; l += kNT)
                    buf[l * PR + cc] = (T)bc_terms((double)buf[l * PR + cc], b, l, j, v);
            }
        }
        // other rows: the entries at xs and xe, one (row, side) per thread
        for (int q = t; q < 2 * nl; q += kNT) {
            const int cc = q >> 1;
            const int j = ub + cc;
            if (zrow || j == b.ys || j == b.ye) continue;
            if ((q & 1) && b.xe == b.xs) continue;
            const int l = (q & 1) ? b.xe : b.xs;
            buf[l * PR + cc] = (T)bc_terms((double)buf[l * PR + cc], b, l, j, v);
        }
        __syncthreads();
    }

    if constexpr (KIND2 >= 0) {
        OutSink<T, PR, true> s1;
        s1.Rv = buf;
        s1.c = c;
        const int i = min(ub + c, a.u0 + a.nu - 1);
        s1.exy = __ldg(a.dv.ex + i) + __ldg(a.dv.ey + v);
        s1.lam = a.dv.lambda;
        s1.ez = ez_s;
        s1.dlo = a.dv.lo;
        s1.dhi = a.dv.hi;
        s1.zmax = (a.dv.perturb && i <= a.dv.xz_hi && v <= a.dv.yz_hi) ? a.dv.zz_hi : -1;
        transform_lines<T, CF, KIND>(buf, red, c, slot, tb, s1);
        OutSink<T, PR, false> s2;
        s2.Rv = buf;
        s2.c = c;
        transform_lines<T, CF, KIND2>(buf, red, c, slot, tb, s2);
    } else {
        OutSink<T, PR, false> s;
        s.Rv = buf;
        s.c = c;
        transform_lines<T, CF, KIND>(buf, red, c, slot, tb, s);
    }

    // ---- store the output window ----
    {
        const int lo = a.st_lo, hi = a.st_hi;
        const long long vb = (long long)v * a.out_sv;
        const double sc = a.use_scale ? a.scale : 1.0;
        if constexpr (CONTIG) {
            // accumulated output (the refinement's update u += c): all of
            // a thread's u values are loaded before any store, so the
            // loads overlap instead of one latency per row
            constexpr int NI = (N + 2 + kNT - 1) / kNT;
            bool done = false;
            if constexpr (ACCS) {
                if (staged) {
                    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
                    __syncthreads();
                    for (int cc = 0; cc < nl; ++cc) {
                        TO* row = out + vb + (long long)(ub + cc) * a.out_su;
                        const double* ar = accb + cc * (N + 2);
                        for (int l = lo + t; l <= hi; l += kNT) row[l] = (TO)(ar[l] + (double)buf[l * PR + cc] * sc);
                    }
                    done = true;
                }
            }
            if constexpr (W * NI <= 48) {
                if (a.acc && !done) {
                    double av[W][NI];
#pragma unroll
                    for (int cc = 0; cc < W; ++cc) {
                        const double* arow = a.acc + vb + (long long)(ub + cc) * a.out_su;
#pragma unroll
                        for (int it = 0; it < NI; ++it) {
                            const int l = lo + t + it * kNT;
                            av[cc][it] = (cc < nl && l <= hi) ? __ldg(arow + l) : 0.0;
                        }
                    }
#pragma unroll
                    for (int cc = 0; cc < W; ++cc) {
                        TO* row = out + vb + (long long)(ub + cc) * a.out_su;
#pragma unroll
                        for (int it = 0; it < NI; ++it) {
                            const int l = lo + t + it * kNT;
                            if (cc < nl && l <= hi) row[l] = (TO)(av[cc][it] + (double)buf[l * PR + cc] * sc);
                        }
                    }
                    done = true;
                }
            }
#pragma unroll 1
            for (int cc = 0; cc < (done ? 0 : nl); ++cc) {
                const long long ro = vb + (long long)(ub + cc) * a.out_su;
                TO* row = out + ro;
                if (a.acc) {
                    const double* arow = a.acc + ro;
                    for (int l = lo + t; l <= hi; l += kNT) row[l] = (TO)(arow[l] + (double)buf[l * PR + cc] * sc);
                } else {
                    for (int l = lo + t; l <= hi; l += kNT) row[l] = (TO)((double)buf[l * PR + cc] * sc);
                }
            }
        } else if (c < nl) {
            const long long o = vb + (long long)(ub + c) * a.out_su + (long long)(lo + slot) * a.out_sl;
            TO* p = out + o;
            const double* q = a.acc ? a.acc + o : nullptr;
            const long long step = (long long)P * a.out_sl;
            for (int l = lo + slot; l <= hi; l += P) {
                const double x = (double)buf[l * PR + c] * sc;
                *p = (TO)(q ? *q + x : x);
                p += step;
                if (q) q += step;
            }
        }
    }
    __syncthreads();
}

template <typename T, typename TI, typename TO, int M, bool CONTIG, int KIND, int KIND2>
__global__ void __launch_bounds__(kNT, fast_min_ctas<M>())
fast_pass(const TI* in, TO* out, PassArgs a, LineTables<T> tg, int ntx, int ntiles) {
    using CF = Cfg<M>;
    constexpr bool ACCS = acc_staged<T, TO, CONTIG>();
    using SL = SmemLayout<T, M, (KIND2 >= 0), ACCS>;
    constexpr int W = CF::W, PR = CF::PR, P = CF::P, N = CF::N;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw + SL::buf);
    T* red = reinterpret_cast<T*>(smem_raw + SL::red);
    double* accb = ACCS ? reinterpret_cast<double*>(smem_raw + SL::accb) : nullptr;

    const int t = threadIdx.x;
    const int c = t % W;
    // slots of a warp: with 8 lines a tile (N = 512) the contiguous passes give
    // warp w the slots w, w + 4, w + 8, w + 12 -- their real-view rows then
    // start 0 / 8 (or 0 / 4 / 8 / 12) 8-byte words apart mod 16 at pitch 9, so
    // the 32 accesses of an instruction hit each bank pair exactly twice (four
    // consecutive slots collide 4-way); elsewhere consecutive slots
    constexpr bool spread = CONTIG && W == 8;
    const int slot = spread ? (t >> 5) + (kNT / 32) * ((t & 31) / W) : t / W;
    if ((int)blockIdx.x >= ntiles) return;

    // stage the line tables in shared memory once (the CTA is persistent)
    LineTables<T> tb = tg;
    {
        C2<T>* sM = reinterpret_cast<C2<T>*>(smem_raw + SL::twM);
        C2<T>* sN = reinterpret_cast<C2<T>*>(smem_raw + SL::twN);
        C2<T>* s4 = reinterpret_cast<C2<T>*>(smem_raw + SL::tw4N);
        T* sI = reinterpret_cast<T*>(smem_raw + SL::inv4sin);
        for (int i = t; i < M; i += kNT) sM[i] = tg.twM[i];
        for (int i = t; i <= M; i += kNT) {
            sN[i] = tg.twN[i];
            s4[i] = tg.tw4N[i];
            sI[i] = tg.inv4sin[i];
        }
        tb.twM = sM;
        tb.twN = sN;
        tb.tw4N = s4;
        tb.inv4sin = sI;
    }
    double* ez_s = reinterpret_cast<double*>(smem_raw + SL::ez);
    if constexpr (KIND2 >= 0) {
        for (int i = t; i < N + 2; i += kNT) ez_s[i] = a.dv.ez[i];
    }

    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        fast_tile<T, TI, TO, M, CONTIG, KIND, KIND2>(in, out, a, tb, ez_s, buf, red, tile, ntx, t, c, slot, accb);
}

// One group of a batched pass (FP64): the members share the length and the
// kinds, so the line tables are staged once; each CTA takes a contiguous range
// of the group's tiles and, when the member changes, copies that member's pass
// descriptor into shared memory (its f and face pointers patched from the
// call's pointer table) and stages its z eigenvalue terms (fused pass).
template <int M, bool CONTIG, int KIND, int KIND2>
__global__ void __launch_bounds__(kNT, fast_min_ctas<M>())
fast_batch_pass(FastBatchArgs g, LineTables<double> tg) {
    using T = double;
    using CF = Cfg<M>;
    using SL = SmemLayout<T, M, (KIND2 >= 0)>;
    constexpr int W = CF::W, N = CF::N;
    constexpr size_t kArgs = (SL::total + 15) & ~size_t(15);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ const double* s_in;
    __shared__ double* s_out;
    __shared__ int s_ntx, s_first;
    T* buf = reinterpret_cast<T*>(smem_raw + SL::buf);
    T* red = reinterpret_cast<T*>(smem_raw + SL::red);
    PassArgs* as = reinterpret_cast<PassArgs*>(smem_raw + kArgs);

    const int t = threadIdx.x;
    const int c = t % W;
    constexpr bool spread = CONTIG && W == 8;
    const int slot = spread ? (t >> 5) + (kNT / 32) * ((t & 31) / W) : t / W;
    const int per = (g.ntiles + (int)gridDim.x - 1) / (int)gridDim.x;
    const int t0 = (int)blockIdx.x * per;
    const int t1 = min(g.ntiles, t0 + per);
    if (t0 >= t1) return;

    LineTables<T> tb = tg;
    {
        C2<T>* sM = reinterpret_cast<C2<T>*>(smem_raw + SL::twM);
        C2<T>* sN = reinterpret_cast<C2<T>*>(smem_raw + SL::twN);
        C2<T>* s4 = reinterpret_cast<C2<T>*>(smem_raw + SL::tw4N);
        T* sI = reinterpret_cast<T*>(smem_raw + SL::inv4sin);
        for (int i = t; i < M; i += kNT) sM[i] = tg.twM[i];
        for (int i = t; i <= M; i += kNT) {
            sN[i] = tg.twN[i];
            s4[i] = tg.tw4N[i];
            sI[i] = tg.inv4sin[i];
        }
        tb.twM = sM;
        tb.twN = sN;
        tb.tw4N = s4;
        tb.inv4sin = sI;
    }
    double* ez_s = reinterpret_cast<double*>(smem_raw + SL::ez);

    int cur = -1, cur_end = 0;
    for (int tile = t0; tile < t1; ++tile) {
        if (tile >= cur_end) {
            // the member owning this tile (binary search over the prefix)
            int lo = 0, hi = g.count - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(g.start + mid) <= tile) lo = mid;
                else hi = mid - 1;
            }
            cur = lo;
            cur_end = __ldg(g.start + cur + 1);
            __syncthreads();   // every thread is done with the previous member's descriptor
            const BatchMember* mb = g.members + cur;
            const long long* src = reinterpret_cast<const long long*>(&mb->a);
            long long* dst = reinterpret_cast<long long*>(as);
            static_assert(sizeof(PassArgs) % 8 == 0, "descriptor copied in 8-byte words");
            for (int i = t; i < (int)(sizeof(PassArgs) / 8); i += kNT) dst[i] = __ldg(src + i);
            __syncthreads();
            if (t == 0) {
                const BatchPtrs& pp = g.ptrs[mb->prob];
                if (as->has_bc) {
                    as->bc.f = pp.f;
                    as->bc.bcl = pp.face[0];
                    as->bc.bcr = pp.face[1];
                    as->bc.bcb = pp.face[2];
                    as->bc.bct = pp.face[3];
                    as->bc.bcf = pp.face[4];
                    as->bc.bce = pp.face[5];
                }
                s_in = mb->in_user ? pp.f : g.ws + mb->ws_off;
                s_out = mb->out_user ? pp.f : g.ws + mb->ws_off;
                s_ntx = mb->ntx;
                s_first = __ldg(g.start + cur);
            }
            if constexpr (KIND2 >= 0) {
                const double* ez = mb->a.dv.ez;
                for (int i = t; i < N + 2; i += kNT) ez_s[i] = __ldg(ez + i);
            }
            __syncthreads();
        }
        fast_tile<T, T, T, M, CONTIG, KIND, KIND2>(s_in, s_out, *as, tb, ez_s, buf, red, tile - s_first, s_ntx, t,
                                                   c, slot);
    }
}

// Shared memory of the batched kernel: the persistent kernel's plus one pass
// descriptor.
template <int M, bool FUSED>
constexpr size_t batch_smem_bytes() {
    return ((SmemLayout<double, M, FUSED>::total + 15) & ~size_t(15)) + sizeof(PassArgs);
}

}  // namespace fast
}  // namespace chz
