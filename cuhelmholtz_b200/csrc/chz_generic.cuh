// Generic shared-memory line pass (any even N <= 2048, radices 2..13): the
// per-tile body shared by the single-problem kernel (chz_kernels.cu) and the
// batched kernel (chz_batch.cu).
#pragma once
#include "chz_device.cuh"
#include "chz_internal.h"

namespace chz {

constexpr int kThreads = 256;

template <typename TI>
__device__ __forceinline__ double ld_in(const TI* p) { return (double)__ldg(p); }

// Body of one tile (bx, by) of a line pass; shared by the single-problem
// kernel below and the batched kernels (one launch over many problems).
// CONTIG: 1 contiguous (x) pass, 0 strided (y, z) pass, kContigRuntime: the
// argument `contig_rt` says which (one body for both, as the persistent batch
// kernel runs both kinds of pass).
constexpr int kContigRuntime = 2;
template <typename T, typename TI, typename TO, int CONTIG, int RSET>
__device__ __forceinline__ void line_pass_tile(const TI* in, TO* out, const PassArgs& a, const LineTables<T>& tb,
                                               int buf_elems, int bx, int by, unsigned char* smem_raw,
                                               bool contig_rt = false) {
    const bool contig = (CONTIG == kContigRuntime) ? contig_rt : (CONTIG != 0);
    T* buf0 = reinterpret_cast<T*>(smem_raw);
    T* buf1 = buf0 + buf_elems;
    T* red = buf1 + buf_elems;
    T* odd = red + kThreads;

    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    const int log2W = a.log2W;
    const int W = 1 << log2W;
    const int PR = a.PR;
    const int N = tb.N;
    const int ub = a.u0 + bx * W;
    const int nl = min(W, a.u0 + a.nu - ub);
    const int v = a.v0 + by;

    // ---- load the input window of W lines into buf0 (real view) ----
    {
        int lo, hi;
        kind_in_window(a.kind, N, lo, hi);
        const int len = hi - lo + 1;
        const long long vbase = (long long)v * a.in_sv;
        if constexpr (sizeof(TI) == sizeof(T)) {
            if (contig) {
                const int total = len * W;
                for (int idx = tid; idx < total; idx += nthr) {
                    const int c = idx / len;
                    const int l = lo + (idx - c * len);
                    const bool valid = c < nl && l >= a.ld_lo && l <= a.ld_hi;
                    const TI* src = valid ? in + vbase + (long long)(ub + c) * a.in_su + l : in;
                    cp_async_elem<sizeof(T)>(&buf0[l * PR + c], src, valid);
                }
            } else {
                const int total = len << log2W;
                for (int idx = tid; idx < total; idx += nthr) {
                    const int c = idx & (W - 1);
                    const int l = lo + (idx >> log2W);
                    const bool valid = c < nl && l >= a.ld_lo && l <= a.ld_hi;
                    const TI* src = valid ? in + vbase + (long long)l * a.in_sl + (ub + c) * a.in_su : in;
                    cp_async_elem<sizeof(T)>(&buf0[l * PR + c], src, valid);
                }
            }
            cp_async_wait_all();
            __syncthreads();
            if (contig && a.has_bc) {
                const int ln = a.ld_hi - a.ld_lo + 1;
                const int total = ln * nl;
                for (int idx = tid; idx < total; idx += nthr) {
                    const int c = idx / ln;
                    const int l = a.ld_lo + (idx - c * ln);
                    buf0[l * PR + c] = (T)bc_terms((double)buf0[l * PR + c], a.bc, l, ub + c, v);
                }
                __syncthreads();
            }
        } else {
            if (contig) {
                const int total = len * W;
                for (int idx = tid; idx < total; idx += nthr) {
                    const int c = idx / len;
                    const int l = lo + (idx - c * len);
                    T val = T(0);
                    if (c < nl && l >= a.ld_lo && l <= a.ld_hi) {
                        double x = ld_in<TI>(in + vbase + (long long)(ub + c) * a.in_su + l);
                        if (a.has_bc) x = bc_terms(x, a.bc, l, ub + c, v);
                        val = (T)x;
                    }
                    buf0[l * PR + c] = val;
                }
            } else {
                const int total = len << log2W;
                for (int idx = tid; idx < total; idx += nthr) {
                    const int c = idx & (W - 1);
                    const int l = lo + (idx >> log2W);
                    T val = T(0);
                    if (c < nl && l >= a.ld_lo && l <= a.ld_hi)
                        val = (T)ld_in<TI>(in + vbase + (long long)l * a.in_sl + (ub + c) * a.in_su);
                    buf0[l * PR + c] = val;
                }
            }
            __syncthreads();
        }
    }

    T* rin = buf0;
    T* other = buf1;
    T* rout = nullptr;
    int kind = a.kind;
    const int reps = (a.kind2 >= 0) ? 2 : 1;
    for (int rep = 0; rep < reps; ++rep) {
        if (kind == kDCT1) odd_sums<T>(rin, PR, log2W, N, red, odd, tid, nthr);
        pre_step<T>(kind, rin, PR, reinterpret_cast<C2<T>*>(other), log2W, tb, tid, nthr);
        __syncthreads();
        const int res = fft_run<T, RSET>(reinterpret_cast<C2<T>*>(other), reinterpret_cast<C2<T>*>(rin),
                                   tb.M, log2W, tb.rp, tb.twM, tid, nthr);
        C2<T>* zres = reinterpret_cast<C2<T>*>(res == 0 ? other : rin);
        rout = (res == 0) ? rin : other;
        post_step<T>(kind, zres, rout, PR, log2W, tb, odd, tid, nthr);
        __syncthreads();
        if (rep == 0 && a.kind2 >= 0) {
            if (a.has_div) {
                // idx advances by nthr (a multiple of W): each thread keeps
                // one column c, so ex[i] + ey[j] is read once
                const DivArgs& d = a.dv;
                const int len = d.hi - d.lo + 1;
                const int total = len << log2W;
                const int c = tid & (W - 1);
                const int i = ub + c;  // x entry (u)
                const int j = v;       // y entry (v)
                if (c < nl) {
                    const double exy = __ldg(d.ex + i) + __ldg(d.ey + j);
                    const int zmax = (d.perturb && i <= d.xz_hi && j <= d.yz_hi) ? d.zz_hi : -1;
                    for (int idx = tid; idx < total; idx += nthr) {
                        const int l = d.lo + (idx >> log2W);
                        const double eig = l <= zmax ? 0.0 : recip_nr((exy + __ldg(d.ez + l)) + d.lambda);
                        T& r = rout[l * PR + c];
                        r = (T)((double)r * eig);
                    }
                }
                __syncthreads();
            }
            kind = a.kind2;
            T* nb = (rout == buf0) ? buf1 : buf0;
            rin = rout;
            other = nb;
        }
    }

    // ---- store the output window ----
    {
        const int lo = a.st_lo, hi = a.st_hi;
        const int len = hi - lo + 1;
        const long long vbase = (long long)v * a.out_sv;
        const double sc = a.scale;
        if (contig) {
            const int total = len * W;
            for (int idx = tid; idx < total; idx += nthr) {
                const int c = idx / len;
                const int l = lo + (idx - c * len);
                if (c < nl) {
                    double x = (double)rout[l * PR + c];
                    if (a.use_scale) x *= sc;
                    const long long o = vbase + (long long)(ub + c) * a.out_su + l;
                    if (a.acc) x += a.acc[o];
                    out[o] = (TO)x;
                }
            }
        } else {
            const int total = len << log2W;
            for (int idx = tid; idx < total; idx += nthr) {
                const int c = idx & (W - 1);
                const int l = lo + (idx >> log2W);
                if (c < nl) {
                    double x = (double)rout[l * PR + c];
                    if (a.use_scale) x *= sc;
                    const long long o = vbase + (long long)l * a.out_sl + (ub + c) * a.out_su;
                    if (a.acc) x += a.acc[o];
                    out[o] = (TO)x;
                }
            }
        }
    }
}

}  // namespace chz
