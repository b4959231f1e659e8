// Device building blocks for the line-pass kernels: complex helpers, the
// shared-memory Stockham FFT stages, and the per-kind pre/post steps that turn
// one complex FFT of length M = N/2 into each of the eight real transforms of
// the reference's transform_kind (cudasymmfft/global.h:6-15).
//
// Data model inside a CTA ("line tile"): W lines of one axis.  A line is the
// padded row of L = N+2 entries.  Two shared-memory buffers are used:
//   real view     R[l * PR + c]   l = 0..N+1, c = 0..W-1 (pitch PR >= W)
//   complex view  Z[m * W + c]    m = 0..M-1
// Threads are mapped column-fastest (c = idx % W), so every step reads and
// writes contiguous runs of W entries: bank-conflict free for W >= 8.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace chz {

template <typename T> struct CplxOf;
template <> struct CplxOf<double> { using type = double2; };
template <> struct CplxOf<float> { using type = float2; };
template <typename T> using C2 = typename CplxOf<T>::type;

template <typename T>
__device__ __forceinline__ C2<T> mk(T re, T im) { C2<T> r; r.x = re; r.y = im; return r; }
template <typename T>
__device__ __forceinline__ C2<T> cadd(C2<T> a, C2<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T>
__device__ __forceinline__ C2<T> csub(C2<T> a, C2<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T>
__device__ __forceinline__ C2<T> cmul(C2<T> a, C2<T> b) {
    return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ C2<T> cconj(C2<T> a) { return mk<T>(a.x, -a.y); }
// a * (-i)
template <typename T>
__device__ __forceinline__ C2<T> cmul_negi(C2<T> a) { return mk<T>(a.y, -a.x); }
// a * (+i)
template <typename T>
__device__ __forceinline__ C2<T> cmul_i(C2<T> a) { return mk<T>(-a.y, a.x); }

// 1/d: the hardware's approximate FP64 reciprocal (about 23 good bits)
// refined by two Newton-Raphson steps r <- r + r (1 - d r), each of which
// squares the relative error (2^-23 -> 2^-46 -> below double rounding).
__device__ __forceinline__ double recip_nr(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// Table reads: plain loads, so the same code reads tables in global memory
// (generic kernel) or staged in shared memory (register-resident kernels).
template <typename T>
__device__ __forceinline__ C2<T> ldtw(const C2<T>* p) { return *p; }
template <typename T>
__device__ __forceinline__ T ldr(const T* p) { return *p; }

// Asynchronous global -> shared copy of one element (cp.async, no register
// staging, so a thread keeps all its copies in flight).  valid == false
// writes zero and reads nothing; `src` must still be a mapped address.
template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* smem_dst, const void* src, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    const int n = valid ? BYTES : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(src), "n"(BYTES), "r"(n)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// sqrt(1/2), sqrt(3)/2 to 20 significant digits
#define CHZ_SQRT_HALF 0.70710678118654752440
#define CHZ_SQRT3_HALF 0.86602540378443864676

// ---------------------------------------------------------------------------
// Forward radix-R DFTs (exponent sign -1) on a register array.
// Radices 2, 3, 4, 8 are written out; 5, 7, 11, 13 use the M-point twiddle
// table (omega_R^t = twM[t * (M/R)]).
// ---------------------------------------------------------------------------
template <typename T, int R> struct Dft;

template <typename T> struct Dft<T, 2> {
    __device__ __forceinline__ static void run(C2<T>* v, const C2<T>*, int) {
        C2<T> a = v[0], b = v[1];
        v[0] = cadd<T>(a, b);
        v[1] = csub<T>(a, b);
    }
};

template <typename T> struct Dft<T, 3> {
    __device__ __forceinline__ static void run(C2<T>* v, const C2<T>*, int) {
        const T s = T(CHZ_SQRT3_HALF);
        C2<T> t1 = cadd<T>(v[1], v[2]);
        C2<T> t2 = mk<T>(v[0].x - T(0.5) * t1.x, v[0].y - T(0.5) * t1.y);
        C2<T> d = csub<T>(v[1], v[2]);
        C2<T> t3 = mk<T>(s * d.x, s * d.y);
        v[0] = cadd<T>(v[0], t1);
        v[1] = cadd<T>(t2, cmul_negi<T>(t3));
        v[2] = cadd<T>(t2, cmul_i<T>(t3));
    }
};

template <typename T>
__device__ __forceinline__ void dft4(C2<T>& a0, C2<T>& a1, C2<T>& a2, C2<T>& a3) {
    C2<T> s02 = cadd<T>(a0, a2), d02 = csub<T>(a0, a2);
    C2<T> s13 = cadd<T>(a1, a3), d13 = csub<T>(a1, a3);
    a0 = cadd<T>(s02, s13);
    a2 = csub<T>(s02, s13);
    a1 = cadd<T>(d02, cmul_negi<T>(d13));
    a3 = cadd<T>(d02, cmul_i<T>(d13));
}

template <typename T> struct Dft<T, 4> {
    __device__ __forceinline__ static void run(C2<T>* v, const C2<T>*, int) {
        dft4<T>(v[0], v[1], v[2], v[3]);
    }
};

template <typename T> struct Dft<T, 8> {
    __device__ __forceinline__ static void run(C2<T>* v, const C2<T>*, int) {
        C2<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        C2<T> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<T>(e0, e1, e2, e3);
        dft4<T>(o0, o1, o2, o3);
        const T r = T(CHZ_SQRT_HALF);
        // o_k *= exp(-i pi k / 4)
        o1 = mk<T>(r * (o1.x + o1.y), r * (o1.y - o1.x));
        o2 = cmul_negi<T>(o2);
        o3 = mk<T>(r * (o3.y - o3.x), -r * (o3.x + o3.y));
        v[0] = cadd<T>(e0, o0); v[4] = csub<T>(e0, o0);
        v[1] = cadd<T>(e1, o1); v[5] = csub<T>(e1, o1);
        v[2] = cadd<T>(e2, o2); v[6] = csub<T>(e2, o2);
        v[3] = cadd<T>(e3, o3); v[7] = csub<T>(e3, o3);
    }
};

// Odd prime radices: pairs (q, R-q) share work.  With s_q = v[q] + v[R-q],
// d_q = v[q] - v[R-q] (q = 1..h, h = (R-1)/2) and omega^t = c_t - i s_t:
//   X[0]   = v[0] + sum_q s_q
//   X[p]   = v[0] + sum_q c_{pq} s_q  - i sum_q s_{pq} d_q
//   X[R-p] = v[0] + sum_q c_{pq} s_q  + i sum_q s_{pq} d_q
// Constants come from the M-point table: omega_R^t = twM[t * (M/R)].
template <typename T, int R> struct DftOddSym {
    __device__ __forceinline__ static void run(C2<T>* v, const C2<T>* twM, int M) {
        constexpr int h = (R - 1) / 2;
        const int step = M / R;
        C2<T> sq[h], dq[h];
        C2<T> x0 = v[0];
#pragma unroll
        for (int q = 1; q <= h; ++q) {
            sq[q - 1] = cadd<T>(v[q], v[R - q]);
            dq[q - 1] = csub<T>(v[q], v[R - q]);
            x0 = cadd<T>(x0, sq[q - 1]);
        }
        const C2<T> v0 = v[0];
        v[0] = x0;
#pragma unroll
        for (int p = 1; p <= h; ++p) {
            C2<T> a = v0;
            C2<T> b = mk<T>(T(0), T(0));
#pragma unroll
            for (int q = 1; q <= h; ++q) {
                const C2<T> w = ldtw<T>(twM + ((p * q) % R) * step);  // (cos, -sin)
                a.x += w.x * sq[q - 1].x;
                a.y += w.x * sq[q - 1].y;
                b.x -= w.y * dq[q - 1].x;
                b.y -= w.y * dq[q - 1].y;
            }
            // X[p] = a - i b, X[R-p] = a + i b
            v[p] = mk<T>(a.x + b.y, a.y - b.x);
            v[R - p] = mk<T>(a.x - b.y, a.y + b.x);
        }
    }
};
template <typename T> struct Dft<T, 5> : DftOddSym<T, 5> {};
template <typename T> struct Dft<T, 7> : DftOddSym<T, 7> {};
template <typename T> struct Dft<T, 11> : DftOddSym<T, 11> {};
template <typename T> struct Dft<T, 13> : DftOddSym<T, 13> {};

// One Stockham autosort stage (forward): src -> dst, natural order in and out
// after all stages.  Ns = product of the radices of the previous stages.
template <typename T, int R>
__device__ __forceinline__ void fft_stage(const C2<T>* __restrict__ src, C2<T>* __restrict__ dst,
                                          int M, int Ns, int log2W, const C2<T>* __restrict__ twM,
                                          int tid, int nthr) {
    const int W = 1 << log2W;
    const int nb = M / R;
    const int total = nb << log2W;
    const int tstep = M / (Ns * R);
    // idx advances by nthr (a multiple of W): c stays, j advances by jstep,
    // and p = j mod Ns is carried along instead of divided out per butterfly
    const int c = tid & (W - 1);
    const int jstep = nthr >> log2W;
    const int pstep = jstep % Ns;
    int p = (tid >> log2W) % Ns;
    for (int idx = tid; idx < total; idx += nthr) {
        const int j = idx >> log2W;
        C2<T> v[R];
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] = src[((j + k * nb) << log2W) + c];
        if (Ns > 1) {
#pragma unroll
            for (int k = 1; k < R; ++k) v[k] = cmul<T>(v[k], ldtw<T>(twM + p * k * tstep));
        }
        Dft<T, R>::run(v, twM, M);
        const int base = (j - p) * R + p;
#pragma unroll
        for (int k = 0; k < R; ++k) dst[((base + k * Ns) << log2W) + c] = v[k];
        p += pstep;
        if (p >= Ns) p -= Ns;
    }
}

constexpr int kMaxStages = 12;

// Radix schedule of one FFT length: stage s uses radix (code >> 4s) & 15.
struct RadixPlan {
    int nst;
    unsigned long long code;
    __host__ __device__ int radix(int s) const { return (int)((code >> (4 * s)) & 15ull); }
};

// Radix sets a kernel variant dispatches over (fewer cases, fewer registers).
enum RadixSet : int { kRadixPow2 = 0, kRadixSmall = 1, kRadixAll = 2 };

__host__ __device__ inline int radix_set_of(const RadixPlan& rp) {
    int set = kRadixPow2;
    for (int s = 0; s < rp.nst; ++s) {
        const int r = rp.radix(s);
        if (r == 3 || r == 5) set = set < kRadixSmall ? kRadixSmall : set;
        if (r == 7 || r == 11 || r == 13) set = kRadixAll;
    }
    return set;
}

// Runs all stages; the input is in buf0; returns 0 when the result is in buf0
// and 1 when it is in buf1.  Ends with a __syncthreads().
template <typename T, int RSET>
__device__ __forceinline__ int fft_run(C2<T>* buf0, C2<T>* buf1, int M, int log2W,
                                       const RadixPlan& rp, const C2<T>* __restrict__ twM,
                                       int tid, int nthr) {
    C2<T>* src = buf0;
    C2<T>* dst = buf1;
    int cur = 0;
    int Ns = 1;
    for (int s = 0; s < rp.nst; ++s) {
        const int R = rp.radix(s);
        switch (R) {
            case 2: fft_stage<T, 2>(src, dst, M, Ns, log2W, twM, tid, nthr); break;
            case 4: fft_stage<T, 4>(src, dst, M, Ns, log2W, twM, tid, nthr); break;
            case 8: fft_stage<T, 8>(src, dst, M, Ns, log2W, twM, tid, nthr); break;
            default:
                if (RSET >= kRadixSmall) {
                    if (R == 3) fft_stage<T, 3>(src, dst, M, Ns, log2W, twM, tid, nthr);
                    else if (R == 5) fft_stage<T, 5>(src, dst, M, Ns, log2W, twM, tid, nthr);
                }
                if (RSET >= kRadixAll) {
                    if (R == 7) fft_stage<T, 7>(src, dst, M, Ns, log2W, twM, tid, nthr);
                    else if (R == 11) fft_stage<T, 11>(src, dst, M, Ns, log2W, twM, tid, nthr);
                    else if (R == 13) fft_stage<T, 13>(src, dst, M, Ns, log2W, twM, tid, nthr);
                }
                break;
        }
        Ns *= R;
        C2<T>* t = src;
        src = dst;
        dst = t;
        cur ^= 1;
        __syncthreads();
    }
    return cur;
}

// ---------------------------------------------------------------------------
// Transform kinds (values of the reference's transform_kind enum)
// ---------------------------------------------------------------------------
enum Kind : int { kDCT1 = 0, kDCT2, kDCT3, kDST1, kDST2, kDST3, kR2C, kC2R };

// Kinds computed as "pack -> forward FFT -> split": a forward real DFT of a
// reordered copy of the line.
__host__ __device__ __forceinline__ bool kind_is_forward_type(int k) {
    return k == kR2C || k == kDCT2 || k == kDST2;
}

// Per-length tables (host-computed in double precision, stored in T):
//   twM[t]     = exp(-2 pi i t / M),        t = 0..M-1
//   twN[k]     = exp(-2 pi i k / N),        k = 0..M
//   tw4N[k]    = exp(-i pi k / (2N)),       k = 0..M
//   inv4sin[k] = 1 / (4 sin(pi k / N)),     k = 1..M (entry 0 unused)
template <typename T>
struct LineTables {
    const C2<T>* twM;
    const C2<T>* twN;
    const C2<T>* tw4N;
    const T* inv4sin;
    int N;
    int M;
    RadixPlan rp;
};

// Input window [lo, hi] each kind reads along its line.
__host__ __device__ __forceinline__ void kind_in_window(int kind, int N, int& lo, int& hi) {
    switch (kind) {
        case kDST1: lo = 1; hi = N - 1; break;
        case kDST2: lo = 1; hi = N; break;
        case kDST3: lo = 0; hi = N; break;
        case kDCT1: lo = 0; hi = N; break;
        case kDCT2: lo = 0; hi = N - 1; break;
        case kDCT3: lo = 0; hi = N - 1; break;
        case kR2C: lo = 0; hi = N - 1; break;
        default: lo = 0; hi = N + 1; break;  // kC2R
    }
}

// Output window [lo, hi] (index 0 of the DST kinds holds an explicit zero).
__host__ __device__ __forceinline__ void kind_out_window(int kind, int N, int& lo, int& hi) {
    switch (kind) {
        case kDST1: lo = 0; hi = N - 1; break;
        case kDST2: lo = 0; hi = N; break;
        case kDST3: lo = 0; hi = N; break;
        case kDCT1: lo = 0; hi = N; break;
        case kDCT2: lo = 0; hi = N - 1; break;
        case kDCT3: lo = 0; hi = N - 1; break;
        case kR2C: lo = 0; hi = N + 1; break;
        default: lo = 0; hi = N - 1; break;  // kC2R
    }
}

// ---------------------------------------------------------------------------
// Pre step: real view R -> complex view Z (the FFT input).
//
// Forward-type kinds pack a reordered copy v of the line as Z[n] = v[2n] + i v[2n+1]:
//   R2C : v[j] = x[j]
//   DCT2: v[j] = x[2j] (j < M),   v[j] = x[2N-1-2j] (j >= M)        (Makhoul order)
//   DST2: v[j] = x[2j+1] (j < M), v[j] = -x[2N-2j] (j >= M)
//         (DST2 of x[1..N] is DCT2 of (-1)^n x[n+1] read backwards)
// Inverse-type kinds build a half spectrum V[0..M] and merge it for an
// inverse real DFT: Z[k] = conj((V[k] + conj V[M-k]) + i conj(w^k)(V[k] - conj V[M-k])),
// w = exp(-2 pi i / N); the outer conj turns the forward FFT into the inverse.
//   C2R : V[k] = x[2k] + i x[2k+1]       (Im V[0] = Im V[M] = 0)
//   DCT3: V[k] = exp(i pi k/2N) (x[k] - i x[N-k]),  x[N] := 0
//   DST3: V[0] = x[0] + x[N], V[k] = exp(i pi k/2N) (x[N-k] - i x[k])
//   DCT1: V[m] = x[2m] + i (x[2m-1] - x[2m+1]), V[0] = x[0], V[M] = x[N]
//   DST1: V[m] = (x[2m+1] - x[2m-1]) - i x[2m], V[0] = 2 x[1], V[M] = -2 x[N-1]
// ---------------------------------------------------------------------------
// Real view of one line: entry l at R[l * PR + c].
template <typename T>
struct StridedView {
    const T* __restrict__ R;
    int PR, c;
    static constexpr bool kPair = false;   // entries l, l + 1 are not adjacent
    __device__ __forceinline__ T operator()(int l) const { return R[l * PR + c]; }
    __device__ __forceinline__ C2<T> pair(int l) const { return mk<T>(R[l * PR + c], R[(l + 1) * PR + c]); }
};

template <typename T>
__device__ __forceinline__ C2<T> inv_spectrum(int kind, const T* __restrict__ R, int PR, int c,
                                              int k, int N, int M, const LineTables<T>& tb);

// The same on any real-view accessor V (entry l of the line: V(l)).  A view
// whose entries 2j, 2j + 1 share one aligned 16-byte word (V::kPair) is read a
// pair at a time where the kind takes both (one shared-memory access instead
// of two; the DCT-I / DST-I differences read pair j - 1 as well).
template <typename T, typename V>
__device__ __forceinline__ C2<T> inv_spectrum_v(int kind, const V& X, int k, int N, int M,
                                                const LineTables<T>& tb) {
    if constexpr (V::kPair) {
        if (kind == kC2R && k != 0 && k != M) return X.pair(2 * k);
        // the odd neighbour x[2k - 1] alone (8 bytes): its pair partner
        // x[2k - 2] is not needed
        if (kind == kDCT1 && k != 0 && k != M) {
            const C2<T> p1 = X.pair(2 * k);
            return mk<T>(p1.x, X(2 * k - 1) - p1.y);
        }
        if (kind == kDST1 && k != 0 && k != M) {
            const C2<T> p1 = X.pair(2 * k);
            return mk<T>(p1.y - X(2 * k - 1), -p1.x);
        }
    }
    switch (kind) {
        case kC2R: {
            if (k == 0 || k == M) return mk<T>(X(2 * k), T(0));
            return mk<T>(X(2 * k), X(2 * k + 1));
        }
        case kDCT3: {
            const T a = X(k);
            const T b = (k == 0) ? T(0) : X(N - k);
            const C2<T> w = cconj<T>(ldtw<T>(tb.tw4N + k));  // exp(+i pi k / 2N)
            C2<T> v = cmul<T>(w, mk<T>(a, -b));
            if (k == M) v.y = T(0);
            return v;
        }
        case kDST3: {
            if (k == 0) return mk<T>(X(0) + X(N), T(0));
            const T a = X(N - k);
            const T b = X(k);
            const C2<T> w = cconj<T>(ldtw<T>(tb.tw4N + k));
            C2<T> v = cmul<T>(w, mk<T>(a, -b));
            if (k == M) v.y = T(0);
            return v;
        }
        case kDCT1: {
            if (k == 0) return mk<T>(X(0), T(0));
            if (k == M) return mk<T>(X(N), T(0));
            return mk<T>(X(2 * k), X(2 * k - 1) - X(2 * k + 1));
        }
        default: {  // kDST1
            if (k == 0) return mk<T>(T(2) * X(1), T(0));
            if (k == M) return mk<T>(T(-2) * X(N - 1), T(0));
            return mk<T>(X(2 * k + 1) - X(2 * k - 1), -X(2 * k));
        }
    }
}

template <typename T>
__device__ __forceinline__ C2<T> inv_spectrum(int kind, const T* __restrict__ R, int PR, int c,
                                              int k, int N, int M, const LineTables<T>& tb) {
    return inv_spectrum_v<T>(kind, StridedView<T>{R, PR, c}, k, N, M, tb);
}

template <typename T, typename V>
__device__ __forceinline__ T fwd_gather_v(int kind, const V& X, int j, int N, int M) {
    switch (kind) {
        case kR2C: return X(j);
        case kDCT2: return (j < M) ? X(2 * j) : X(2 * N - 1 - 2 * j);
        default:  // kDST2
            return (j < M) ? X(2 * j + 1) : -X(2 * N - 2 * j);
    }
}

template <typename T>
__device__ __forceinline__ T fwd_gather(int kind, const T* __restrict__ R, int PR, int c, int j,
                                        int N, int M) {
    return fwd_gather_v<T>(kind, StridedView<T>{R, PR, c}, j, N, M);
}

template <typename T>
__device__ __forceinline__ void pre_step(int kind, const T* __restrict__ R, int PR, C2<T>* __restrict__ Z,
                                         int log2W, const LineTables<T>& tb, int tid, int nthr) {
    const int W = 1 << log2W;
    const int N = tb.N, M = tb.M;
    if (kind_is_forward_type(kind)) {
        const int total = M << log2W;
        for (int idx = tid; idx < total; idx += nthr) {
            const int c = idx & (W - 1);
            const int n = idx >> log2W;
            const T a = fwd_gather<T>(kind, R, PR, c, 2 * n, N, M);
            const T b = fwd_gather<T>(kind, R, PR, c, 2 * n + 1, N, M);
            Z[idx] = mk<T>(a, b);
        }
    } else {
        const int half = M / 2;
        const int total = (half + 1) << log2W;
        for (int idx = tid; idx < total; idx += nthr) {
            const int c = idx & (W - 1);
            const int k = idx >> log2W;
            const int km = M - k;
            const C2<T> vk = inv_spectrum<T>(kind, R, PR, c, k, N, M, tb);
            const C2<T> vm = inv_spectrum<T>(kind, R, PR, c, km, N, M, tb);
            // Z[k] = (V[k] + conj V[M-k]) + i conj(w^k) (V[k] - conj V[M-k])
            const C2<T> wk = ldtw<T>(tb.twN + k);
            {
                const C2<T> e = cadd<T>(vk, cconj<T>(vm));
                const C2<T> o = cmul<T>(cconj<T>(wk), csub<T>(vk, cconj<T>(vm)));
                Z[(k << log2W) + c] = cconj<T>(cadd<T>(e, cmul_i<T>(o)));
            }
            if (km != k && km < M) {
                // Z[M-k] = (V[M-k] + conj V[k]) + i conj(w^(M-k)) (V[M-k] - conj V[k]),
                // conj(w^(M-k)) = -w^k
                const C2<T> e = cadd<T>(vm, cconj<T>(vk));
                const C2<T> o = cmul<T>(mk<T>(-wk.x, -wk.y), csub<T>(vm, cconj<T>(vk)));
                Z[(km << log2W) + c] = cconj<T>(cadd<T>(e, cmul_i<T>(o)));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Post step: complex FFT result Z -> real view R (the output line).
// `odd_sum[c]` holds sum_j x[2j+1] of line c (DCT1 only).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void post_step(int kind, const C2<T>* __restrict__ Z, T* __restrict__ R, int PR,
                                          int log2W, const LineTables<T>& tb, const T* odd_sum,
                                          int tid, int nthr) {
    const int W = 1 << log2W;
    const int N = tb.N, M = tb.M;
#define Y(l) R[(l) * PR + c]
    if (kind_is_forward_type(kind)) {
        // split: V[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 w^k (Z[k] - conj Z[M-k])
        const int half = M / 2;
        const int total = (half + 1) << log2W;
        for (int idx = tid; idx < total; idx += nthr) {
            const int c = idx & (W - 1);
            const int k = idx >> log2W;
            const int km = M - k;
            const C2<T> zk = Z[(k << log2W) + c];
            const C2<T> zm = (k == 0) ? zk : Z[(km << log2W) + c];
            const C2<T> wk = ldtw<T>(tb.twN + k);
            C2<T> vk, vm;
            {
                const C2<T> e = cadd<T>(zk, cconj<T>(zm));
                const C2<T> o = cmul<T>(wk, csub<T>(zk, cconj<T>(zm)));
                vk = mk<T>(T(0.5) * (e.x + o.y), T(0.5) * (e.y - o.x));
            }
            {
                // w^(M-k) = -conj(w^k)
                const C2<T> e = cadd<T>(zm, cconj<T>(zk));
                const C2<T> o = cmul<T>(mk<T>(-wk.x, wk.y), csub<T>(zm, cconj<T>(zk)));
                vm = mk<T>(T(0.5) * (e.x + o.y), T(0.5) * (e.y - o.x));
            }
            if (kind == kR2C) {
                Y(2 * k) = vk.x;
                Y(2 * k + 1) = (k == 0) ? T(0) : vk.y;
                if (km != k) {
                    Y(2 * km) = vm.x;
                    Y(2 * km + 1) = (km == M) ? T(0) : vm.y;
                }
            } else {
                // DCT2: D[k] = Re(e^{-i pi k/2N} V[k]); D[N-k] = -Im(...) for 0 < k < M.
                const C2<T> ak = cmul<T>(ldtw<T>(tb.tw4N + k), vk);
                const C2<T> am = cmul<T>(ldtw<T>(tb.tw4N + km), vm);
                if (kind == kDCT2) {
                    Y(k) = ak.x;
                    if (k > 0 && k < M) Y(N - k) = -ak.y;
                    if (km != k) {
                        Y(km) = am.x;
                        if (km > 0 && km < M) Y(N - km) = -am.y;
                    }
                } else {  // DST2: out[m] = D[N-m], out[0] = 0
                    Y(N - k) = ak.x;
                    if (k > 0 && k < M) Y(k) = -ak.y;
                    if (km != k) {
                        Y(N - km) = am.x;
                        if (km > 0 && km < M) Y(km) = -am.y;
                    }
                    if (k == 0) Y(0) = T(0);
                }
            }
        }
    } else if (kind == kDCT1 || kind == kDST1) {
        // v[n] = Re a[n/2] (n even) or Im a[n/2] (n odd), a = conj(Z)
        const int total = (M + 1) << log2W;
        for (int idx = tid; idx < total; idx += nthr) {
            const int c = idx & (W - 1);
            const int k = idx >> log2W;
            auto vat = [&](int n) -> T {
                const C2<T> a = Z[((n >> 1) << log2W) + c];
                return (n & 1) ? -a.y : a.x;
            };
            if (k == 0) {
                if (kind == kDCT1) {
                    const T h = T(0.5) * vat(0);
                    Y(0) = h + odd_sum[c];
                    Y(N) = h - odd_sum[c];
                } else {
                    Y(0) = T(0);
                }
                continue;
            }
            const T s = vat(k);
            const T sn = vat(N - k);
            const T is4 = ldr<T>(tb.inv4sin + k);
            if (kind == kDCT1) {
                const T ta = (s + sn) * T(0.5);
                const T tbv = (s - sn) * is4;
                Y(k) = (ta - tbv) * T(0.5);
                if (N - k != k) Y(N - k) = (ta + tbv) * T(0.5);
            } else {
                const T ta = (s + sn) * is4;
                const T tbv = (s - sn) * T(0.5);
                Y(k) = (ta + tbv) * T(0.5);
                if (N - k != k) Y(N - k) = (ta - tbv) * T(0.5);
            }
        }
    } else {
        // C2R, DCT3, DST3: a = conj(Z); v[2n] = Re a[n], v[2n+1] = Im a[n]
        const int total = M << log2W;
        for (int idx = tid; idx < total; idx += nthr) {
            const int c = idx & (W - 1);
            const int n = idx >> log2W;
            const C2<T> zc = Z[idx];
            const T v0 = zc.x, v1 = -zc.y;  // v[2n], v[2n+1]
            if (kind == kC2R) {
                Y(2 * n) = v0;
                Y(2 * n + 1) = v1;
            } else if (kind == kDCT3) {
                // y[2n'] = v[n']/2, y[2n'+1] = v[N-1-n']/2
                const int e0 = 2 * n, e1 = 2 * n + 1;
                // position of v[e] in the output
                Y(e0 < M ? 2 * e0 : 2 * (N - 1 - e0) + 1) = T(0.5) * v0;
                Y(e1 < M ? 2 * e1 : 2 * (N - 1 - e1) + 1) = T(0.5) * v1;
            } else {  // DST3: out[2n'+1] = v[n']/2, out[2n'+2] = -v[N-1-n']/2
                const int e0 = 2 * n, e1 = 2 * n + 1;
                if (e0 < M) Y(2 * e0 + 1) = T(0.5) * v0;
                else Y(2 * (N - 1 - e0) + 2) = T(-0.5) * v0;
                if (e1 < M) Y(2 * e1 + 1) = T(0.5) * v1;
                else Y(2 * (N - 1 - e1) + 2) = T(-0.5) * v1;
                if (n == 0) Y(0) = T(0);
            }
        }
    }
#undef Y
}

// Sum of the odd entries x[1], x[3], ..., x[N-1] of every line (DCT1), with a
// fixed summation order.  `red` holds nthr values; the result lands in
// odd_sum[0..W-1].  Ends with a __syncthreads().
template <typename T>
__device__ __forceinline__ void odd_sums(const T* __restrict__ R, int PR, int log2W, int N, T* red,
                                         T* odd_sum, int tid, int nthr) {
    const int W = 1 << log2W;
    const int parts = nthr >> log2W;  // threads per column
    const int M = N / 2;
    {
        const int c = tid & (W - 1);
        const int part = tid >> log2W;
        T acc = T(0);
        if (part < parts) {
            for (int j = part; j < M; j += parts) acc += R[(2 * j + 1) * PR + c];
        }
        red[tid] = acc;
    }
    __syncthreads();
    if (tid < W) {
        T acc = T(0);
        for (int p = 0; p < parts; ++p) acc += red[(p << log2W) + tid];
        odd_sum[tid] = acc;
    }
    __syncthreads();
}

}  // namespace chz
