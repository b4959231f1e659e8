// Line-pass kernels for the 3-D mixed DFT/DST/DCT transform and the fused
// Helmholtz passes, hand-written for sm_100a.
//
// One kernel, `line_pass`, transforms lines of one axis of a 3-D array.  A CTA
// owns a tile of W lines: it loads the kind's input window of those lines into
// shared memory (rows of a contiguous axis, or W-wide column segments of a
// strided axis, which performs the axis transpose that the reference delegates
// to libcuTranspose, cudasymmfft/funcinterface.cu:120-195), runs pre step ->
// Stockham FFT of length N/2 -> post step in shared memory, optionally applies
// the eigenvalue division and a second (inverse) transform, and stores the
// output window.  Every pass is one HBM read and one HBM write of its lines.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "chz_internal.h"

#include "chz_generic.cuh"
#include "chz_fast.cuh"

namespace chz {

template <typename T, typename TI, typename TO, bool CONTIG, int RSET>
__global__ void __launch_bounds__(kThreads, RSET == kRadixAll ? 2 : 3)
line_pass(const TI* in, TO* out, PassArgs a, LineTables<T> tb, int buf_elems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    line_pass_tile<T, TI, TO, CONTIG, RSET>(in, out, a, tb, buf_elems, blockIdx.x, blockIdx.y, smem_raw);
}

// Periodic planes: every node with index N on a periodic axis takes the value
// at the wrapped position (the composition of _3d_bc0_store_{x,y,z}_,
// _cuda_helmholtz_.inl:58-68, 116-126, 173-183, run in x, y, z order).  The
// source node never lies on a periodic N plane, so the copies do not race;
// nodes on two planes are written twice with the same value.
__global__ void periodic_fixup(double* f, int nx, int ny, int nz, int px, int py, int pz) {
    const long long sfy = nx + 1;
    const long long sfz = (long long)(nx + 1) * (ny + 1);
    const long long nX = px ? (long long)(ny + 1) * (nz + 1) : 0;
    const long long nY = py ? (long long)(nx + 1) * (nz + 1) : 0;
    const long long nZ = pz ? (long long)(nx + 1) * (ny + 1) : 0;
    const long long total = nX + nY + nZ;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (e < nX) {
            k = (int)(e / (ny + 1));
            j = (int)(e - (long long)k * (ny + 1));
            i = nx;
        } else if (e < nX + nY) {
            const long long r = e - nX;
            k = (int)(r / (nx + 1));
            i = (int)(r - (long long)k * (nx + 1));
            j = ny;
        } else {
            const long long r = e - nX - nY;
            j = (int)(r / (nx + 1));
            i = (int)(r - (long long)j * (nx + 1));
            k = nz;
        }
        const int si = (px && i == nx) ? 0 : i;
        const int sj = (py && j == ny) ? 0 : j;
        const int sk = (pz && k == nz) ? 0 : k;
        f[k * sfz + j * sfy + i] = f[sk * sfz + sj * sfy + si];
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

std::atomic<int> g_force_generic{0};

int factor_radices(int M, RadixPlan* rp) {
    int m = M;
    int e2 = 0;
    int n = 0;
    unsigned long long code = 0;
    auto push = [&](int r) {
        if (n >= kMaxStages) return false;
        code |= (unsigned long long)r << (4 * n);
        ++n;
        return true;
    };
    while (m % 2 == 0) { m /= 2; ++e2; }
    while (e2 >= 3) { if (!push(8)) return -1; e2 -= 3; }
    if (e2 == 2 && !push(4)) return -1;
    if (e2 == 1 && !push(2)) return -1;
    const int odd[] = {3, 5, 7, 11, 13};
    for (int p : odd) {
        while (m % p == 0) {
            if (!push(p)) return -1;
            m /= p;
        }
    }
    if (m != 1) return -1;
    rp->nst = n;
    rp->code = code;
    return 0;
}

bool radix_plan_is_pow2(const RadixPlan& rp) {
    for (int s = 0; s < rp.nst; ++s) {
        const int r = rp.radix(s);
        if (r != 2 && r != 4 && r != 8) return false;
    }
    return true;
}

static int ilog2(int x) { int r = 0; while ((1 << (r + 1)) <= x) ++r; return r; }

LineGeom line_geometry(int N, int is_double, bool contig) {
    return line_geometry_target(N, is_double, contig, is_double ? 4096 : 8192, ~(size_t)0);
}

LineGeom line_geometry_target(int N, int is_double, bool contig, int target, size_t max_smem) {
    LineGeom g{};
    g.N = N;
    g.M = N / 2;
    int W = 1 << ilog2(std::max(1, target / N));
    W = std::max(2, std::min(64, W));
    const size_t esz0 = is_double ? 8 : 4;
    while (W > 2) {
        const size_t pr = contig ? W + 1 : W;
        const size_t be = ((std::max(((size_t)N + 2) * pr, (size_t)N * W) + 3) & ~(size_t)3);
        if ((2 * be + kThreads + W) * esz0 <= max_smem) break;
        W >>= 1;
    }
    g.W = W;
    g.log2W = ilog2(W);
    g.PR = contig ? W + 1 : W;
    const size_t L = (size_t)N + 2;
    const size_t real_elems = L * g.PR;
    const size_t cplx_elems = (size_t)2 * g.M * W;
    g.buf_elems = std::max(real_elems, cplx_elems);
    // keep each buffer a multiple of 4 elements (16-byte alignment of buf1)
    g.buf_elems = (g.buf_elems + 3) & ~(size_t)3;
    const size_t esz = is_double ? 8 : 4;
    g.smem_bytes = (2 * g.buf_elems + kThreads + W) * esz;
    g.threads = kThreads;
    return g;
}

namespace {

struct TablesCache {
    std::mutex mu;
    std::map<std::tuple<int, int, int>, DeviceLineTables> map;
};

TablesCache& tables_cache() {
    static TablesCache* c = new TablesCache();  // intentionally never destroyed
    return *c;
}

template <typename T>
int build_tables(int N, DeviceLineTables* t) {
    const int M = N / 2;
    std::vector<C2<T>> twM(M), twN(M + 1), tw4N(M + 1);
    std::vector<T> inv4sin(M + 1, T(0));
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < M; ++k) {
        // exact values on the axes keep the symmetric entries exact
        const double ang = -2.0 * pi * (double)k / (double)M;
        twM[k].x = (T)std::cos(ang);
        twM[k].y = (T)std::sin(ang);
        if (4 * k == M) { twM[k].x = T(0); twM[k].y = T(-1); }
        if (2 * k == M) { twM[k].x = T(-1); twM[k].y = T(0); }
        if (4 * k == 3 * M) { twM[k].x = T(0); twM[k].y = T(1); }
    }
    for (int k = 0; k <= M; ++k) {
        const double a = -2.0 * pi * (double)k / (double)N;
        twN[k].x = (T)std::cos(a);
        twN[k].y = (T)std::sin(a);
        if (4 * k == N) { twN[k].x = T(0); twN[k].y = T(-1); }
        if (k == M) { twN[k].x = T(-1); twN[k].y = T(0); }
        const double b = -pi * (double)k / (2.0 * (double)N);
        tw4N[k].x = (T)std::cos(b);
        tw4N[k].y = (T)std::sin(b);
        if (k >= 1) inv4sin[k] = (T)(1.0 / (4.0 * std::sin(pi * (double)k / (double)N)));
    }
    twM[0].x = T(1); twM[0].y = T(0);
    twN[0].x = T(1); twN[0].y = T(0);
    tw4N[0].x = T(1); tw4N[0].y = T(0);
    size_t bytes[4] = {sizeof(C2<T>) * M, sizeof(C2<T>) * (M + 1), sizeof(C2<T>) * (M + 1),
                       sizeof(T) * (M + 1)};
    const void* src[4] = {twM.data(), twN.data(), tw4N.data(), inv4sin.data()};
    void* dst[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < 4; ++i) {
        if (cudaMalloc(&dst[i], bytes[i]) != cudaSuccess) {
            for (int j = 0; j < i; ++j) cudaFree(dst[j]);
            return (int)cudaErrorMemoryAllocation;
        }
        if (cudaMemcpy(dst[i], src[i], bytes[i], cudaMemcpyHostToDevice) != cudaSuccess) {
            for (int j = 0; j <= i; ++j) cudaFree(dst[j]);
            return (int)cudaErrorUnknown;
        }
    }
    t->twM = dst[0];
    t->twN = dst[1];
    t->tw4N = dst[2];
    t->inv4sin = dst[3];
    return 0;
}

}  // namespace

int get_line_tables(int N, int is_double, int device, DeviceLineTables* out) {
    TablesCache& c = tables_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    auto key = std::make_tuple(N, is_double, device);
    auto it = c.map.find(key);
    if (it != c.map.end()) {
        *out = it->second;
        return 0;
    }
    DeviceLineTables t;
    t.N = N;
    t.M = N / 2;
    if (factor_radices(t.M, &t.rp) != 0) return -1;
    const int rc = is_double ? build_tables<double>(N, &t) : build_tables<float>(N, &t);
    if (rc != 0) return rc;
    c.map[key] = t;
    *out = t;
    return 0;
}

template <typename T>
static LineTables<T> to_tables(const DeviceLineTables& d) {
    LineTables<T> t;
    t.twM = reinterpret_cast<const C2<T>*>(d.twM);
    t.twN = reinterpret_cast<const C2<T>*>(d.twN);
    t.tw4N = reinterpret_cast<const C2<T>*>(d.tw4N);
    t.inv4sin = reinterpret_cast<const T*>(d.inv4sin);
    t.N = d.N;
    t.M = d.M;
    t.rp = d.rp;
    return t;
}

template <typename T, typename TI, typename TO, bool CONTIG>
static int launch_typed(const void* in, void* out, const PassArgs& a, const DeviceLineTables& tb,
                        const LineGeom& g, int nv, cudaStream_t stream, const char* label) {
    const int rset = radix_set_of(tb.rp);
    auto kern = rset == kRadixPow2    ? line_pass<T, TI, TO, CONTIG, kRadixPow2>
                : rset == kRadixSmall ? line_pass<T, TI, TO, CONTIG, kRadixSmall>
                                      : line_pass<T, TI, TO, CONTIG, kRadixAll>;
    // opt in to large dynamic shared memory (idempotent; cheap)
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g.smem_bytes);
    if (e != cudaSuccess) return (int)e;
    const int ntiles = (a.nu + g.W - 1) / g.W;
    if (ntiles <= 0 || nv <= 0) return 0;
    dim3 grid(ntiles, nv);
    trace_begin(stream, label);
    kern<<<grid, g.threads, g.smem_bytes, stream>>>(static_cast<const TI*>(in), static_cast<TO*>(out), a,
                                                    to_tables<T>(tb), (int)g.buf_elems);
    count_launch();
    trace_end(stream);
    return (int)cudaGetLastError();
}

// Power-of-two half lengths 16..512 use the register-resident kernels (FP64
// and FP32); the mixed lengths with a register radix plan use them in FP64,
// and in FP32 at N = 192, 320, 384 (the others: the generic kernel).
static bool fast_mixed_length(int M) {
    switch (M) {
        case 12: case 20: case 24: case 28: case 40: case 48: case 56: case 72: case 80: case 96: case 160:
        case 192:
            return true;
        default:
            return false;
    }
}
bool fast_path_supported(int M, bool is_double) {
    if (M >= 16 && M <= 512 && (M & (M - 1)) == 0) return true;
    if (!is_double) return M == 96 || M == 160 || M == 192;
    return fast_mixed_length(M);
}

namespace fast {
template <typename T, typename TI, typename TO, int M>
int launch_fast_kind(bool contig, int kind, int kind2, const void* in, void* out, const PassArgs& a,
                     const LineTables<T>& tb, int nv, cudaStream_t stream, const char* label);
template <int M>
int launch_fast_batch_kind(bool contig, int kind, int kind2, const FastBatchArgs& g, const LineTables<double>& tb,
                           cudaStream_t stream);

int device_sm_count() {
    static std::atomic<int> cached[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v == 0) {
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        if (v <= 0) v = 1;
        cached[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}
}  // namespace fast

template <typename T, typename TI, typename TO>
static int launch_fast_t(bool contig, const void* in, void* out, const PassArgs& a, const DeviceLineTables& tb,
                         int nv, cudaStream_t stream, const char* label) {
    const LineTables<T> t = to_tables<T>(tb);
#define CHZ_M(MM) \
    case MM: return fast::launch_fast_kind<T, TI, TO, MM>(contig, a.kind, a.kind2, in, out, a, t, nv, stream, label)
    switch (tb.M) {
        CHZ_M(16);
        CHZ_M(32);
        CHZ_M(64);
        CHZ_M(128);
        CHZ_M(256);
        CHZ_M(512);
        default: break;
    }
    if constexpr (std::is_same<T, float>::value) {
        switch (tb.M) {
            CHZ_M(96);
            CHZ_M(160);
            CHZ_M(192);
            default: return (int)cudaErrorInvalidValue;
        }
    } else {
        switch (tb.M) {
            CHZ_M(12);
            CHZ_M(20);
            CHZ_M(24);
            CHZ_M(28);
            CHZ_M(40);
            CHZ_M(48);
            CHZ_M(56);
            CHZ_M(72);
            CHZ_M(80);
            CHZ_M(96);
            CHZ_M(160);
            CHZ_M(192);
            default: break;
        }
    }
    return (int)cudaErrorInvalidValue;
#undef CHZ_M
}

#define CHZ_FAST_LENGTHS(X) \
    X(12) X(16) X(20) X(24) X(28) X(32) X(40) X(48) X(56) X(64) X(72) X(80) X(96) X(128) X(160) X(192) X(256) X(512)

int fast_lines_per_tile(int M) {
    switch (M) {
#define CHZ_W(MM) \
    case MM: return fast::Cfg<MM>::W;
        CHZ_FAST_LENGTHS(CHZ_W)
#undef CHZ_W
        default: return 0;
    }
}

int launch_fast_batch(bool contig, int kind, int kind2, const FastBatchArgs& g, const LineTables<double>& t,
                      cudaStream_t stream) {
    switch (t.M) {
#define CHZ_B(MM) \
    case MM: return fast::launch_fast_batch_kind<MM>(contig, kind, kind2, g, t, stream);
        CHZ_FAST_LENGTHS(CHZ_B)
#undef CHZ_B
        default: return (int)cudaErrorInvalidValue;
    }
}

namespace tma {
template <typename T, int M>
int launch_tma_kind(int kind, int kind2, const void* in, void* out, const PassArgs& a, const LineTables<T>& tb,
                    int nv, cudaStream_t stream, const char* label);
}  // namespace tma

// Strided passes of N = 128, 256, 512 with the same type in and out and no
// scale, accumulation or boundary terms go to the TMA-pipelined kernel; -1
// when it does not take the pass.
template <typename T>
static int try_tma(const void* in, void* out, const PassArgs& a, const DeviceLineTables& tb, int nv,
                   cudaStream_t stream, const char* label) {
    if (a.acc || a.use_scale || a.has_bc) return -1;
    const LineTables<T> t = to_tables<T>(tb);
    switch (tb.M) {
        case 64: return tma::launch_tma_kind<T, 64>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
        case 128: return tma::launch_tma_kind<T, 128>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
        case 256: return tma::launch_tma_kind<T, 256>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
        default: break;
    }
    switch (tb.M) {
        case 96: return tma::launch_tma_kind<T, 96>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
        case 160: return tma::launch_tma_kind<T, 160>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
        default: break;
    }
    return -1;
}

namespace xtma {
template <int M>
int launch_xtma_kind(int kind, int kind2, const void* in, void* out, const PassArgs& a,
                     const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label);
}  // namespace xtma

// FP64 contiguous passes of N = 256 and 512 go to the TMA-pipelined
// contiguous kernel (each side by tensor boxes on 16-byte-aligned rows, or by
// bulk spans / row stores on the solver's f); -1 when it does not take the
// pass.
static int try_xtma(const void* in, void* out, const PassArgs& a, const DeviceLineTables& tb, int nv,
                    cudaStream_t stream, const char* label) {
    if (a.acc || a.kind2 >= 0 || (tb.M != 256 && tb.M != 128)) return -1;
    const LineTables<double> t = to_tables<double>(tb);
    if (tb.M == 128) return xtma::launch_xtma_kind<128>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
    return xtma::launch_xtma_kind<256>(a.kind, a.kind2, in, out, a, t, nv, stream, label);
}

int launch_line_pass(int is_double, int in_type, int out_type, bool contig, const void* in,
                     void* out, const PassArgs& a, const DeviceLineTables& tb, const LineGeom& g,
                     int nv, cudaStream_t stream, const char* label) {
    const int family = g_force_generic.load(std::memory_order_relaxed);
    if (contig && family == 0 && is_double && in_type == kIoF64 && out_type == kIoF64) {
        const int rc = try_xtma(in, out, a, tb, nv, stream, label);
        if (rc != -1) return rc;
    }
    if (!contig && family == 0 && in_type == out_type) {
        const int rc = is_double ? try_tma<double>(in, out, a, tb, nv, stream, label)
                                 : try_tma<float>(in, out, a, tb, nv, stream, label);
        if (rc != -1) return rc;
    }
    if (fast_path_supported(tb.M, is_double != 0) && family != 1) {
        if (is_double) {
            if (in_type == kIoF64 && out_type == kIoF64)
                return launch_fast_t<double, double, double>(contig, in, out, a, tb, nv, stream, label);
        } else {
            if (in_type == kIoF32 && out_type == kIoF32)
                return launch_fast_t<float, float, float>(contig, in, out, a, tb, nv, stream, label);
            if (in_type == kIoF64 && out_type == kIoF32)
                return launch_fast_t<float, double, float>(contig, in, out, a, tb, nv, stream, label);
            if (in_type == kIoF32 && out_type == kIoF64)
                return launch_fast_t<float, float, double>(contig, in, out, a, tb, nv, stream, label);
        }
        return (int)cudaErrorInvalidValue;
    }
#define CHZ_DISPATCH(T, TI, TO)                                                              \
    return contig ? launch_typed<T, TI, TO, true>(in, out, a, tb, g, nv, stream, label)     \
                  : launch_typed<T, TI, TO, false>(in, out, a, tb, g, nv, stream, label)
    if (is_double) {
        if (in_type == kIoF64 && out_type == kIoF64) CHZ_DISPATCH(double, double, double);
    } else {
        if (in_type == kIoF64 && out_type == kIoF32) CHZ_DISPATCH(float, double, float);
        if (in_type == kIoF32 && out_type == kIoF32) CHZ_DISPATCH(float, float, float);
        if (in_type == kIoF32 && out_type == kIoF64) CHZ_DISPATCH(float, float, double);
    }
#undef CHZ_DISPATCH
    return (int)cudaErrorInvalidValue;
}

int launch_periodic_fixup(double* f, int nx, int ny, int nz, int xbc, int ybc, int zbc,
                          cudaStream_t stream) {
    if (xbc != 0 && ybc != 0 && zbc != 0) return 0;
    const long long total = (xbc == 0 ? (long long)(ny + 1) * (nz + 1) : 0) +
                            (ybc == 0 ? (long long)(nx + 1) * (nz + 1) : 0) +
                            (zbc == 0 ? (long long)(nx + 1) * (ny + 1) : 0);
    const int threads = 256;
    long long blocks = (total + threads - 1) / threads;
    blocks = std::min<long long>(blocks, 148LL * 16);
    trace_begin(stream, "periodic_fixup");
    periodic_fixup<<<(int)blocks, threads, 0, stream>>>(f, nx, ny, nz, xbc == 0, ybc == 0, zbc == 0);
    count_launch();
    trace_end(stream);
    return (int)cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launch tracing
// ---------------------------------------------------------------------------
namespace {
struct TraceRec {
    const char* label;
    cudaEvent_t start, stop;
};
struct TraceState {
    std::mutex mu;
    bool on = false;
    std::vector<TraceRec> recs;
    std::vector<cudaEvent_t> pending_start;
};
TraceState& trace_state() {
    static TraceState* t = new TraceState();
    return *t;
}
std::atomic<unsigned long long> g_launches{0};
thread_local cudaEvent_t t_open_start = nullptr;
thread_local const char* t_open_label = nullptr;
}  // namespace

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void trace_begin(cudaStream_t stream, const char* label) {
    TraceState& t = trace_state();
    if (!t.on) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, stream);
    t_open_start = e;
    t_open_label = label;
}

void trace_end(cudaStream_t stream) {
    TraceState& t = trace_state();
    if (!t.on || !t_open_start) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, stream);
    std::lock_guard<std::mutex> lk(t.mu);
    t.recs.push_back({t_open_label, t_open_start, e});
    t_open_start = nullptr;
}

}  // namespace chz

using namespace chz;

extern "C" {

// Starts (on != 0) or stops recording per-launch CUDA events.
int chz_trace_enable(int on) {
    TraceState& t = trace_state();
    std::lock_guard<std::mutex> lk(t.mu);
    t.on = on != 0;
    return 0;
}

// Waits for the recorded launches and writes "label count total_ms\n" lines
// (one per label, in first-seen order) into buf; clears the records.  Returns
// the number of launches collected, or -1 on a CUDA error.
int chz_trace_collect(char* buf, size_t len) {
    TraceState& t = trace_state();
    std::vector<TraceRec> recs;
    {
        std::lock_guard<std::mutex> lk(t.mu);
        recs.swap(t.recs);
    }
    std::vector<std::string> order;
    std::map<std::string, std::pair<int, double>> acc;
    int n = 0;
    for (auto& r : recs) {
        if (cudaEventSynchronize(r.stop) != cudaSuccess) return -1;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.start, r.stop);
        std::string key = r.label ? r.label : "?";
        if (!acc.count(key)) order.push_back(key);
        acc[key].first += 1;
        acc[key].second += ms;
        cudaEventDestroy(r.start);
        cudaEventDestroy(r.stop);
        ++n;
    }
    std::string out;
    for (auto& k : order) {
        char line[256];
        snprintf(line, sizeof(line), "%s %d %.6f\n", k.c_str(), acc[k].first, acc[k].second);
        out += line;
    }
    if (buf && len) {
        std::strncpy(buf, out.c_str(), len - 1);
        buf[len - 1] = 0;
    }
    return n;
}

// Selects the kernel family: 0 = register-resident kernels where supported
// (default), 1 = the generic shared-memory kernel for every length.  Returns
// the previous setting.
int chz_set_kernel_family(int family) {
    if (family < 0 || family > 2) return -1;
    return g_force_generic.exchange(family);
}

// Total kernel launches issued by this library in this process.
unsigned long long chz_launch_count(void) { return launch_count(); }

}  // extern "C"
