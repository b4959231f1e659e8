// Allocation-free FP64 Helmholtz solve: chz_helmholtz_solve_noalloc.
//
// Some callers cannot call cudaMalloc: code that runs where the device memory
// is owned by another allocator (a framework's caching pool, a fixed arena),
// processes under a hard memory budget, and code paths that must not block on
// the allocator.  This entry point needs no device allocation at all: its work
// array and its per-axis tables live in file-scope __device__ arrays of fixed
// size, which every GPU that loads the library holds until the process exits.
//
// Limits: (NX+2)(NY+2)(NZ+2) <= 2^23 doubles (64 MiB of scratch, e.g. 200^3 or
// 256 x 256 x 126) and N <= 1024 per axis; larger problems are rejected with
// CHZ_ERROR_UNSUPPORTED_SIZE before any device work.
//
// All calls share the arrays, which keep the last call's contents; calls that
// overlap on the GPU (different streams or host threads) race on them.  Each
// call rewrites every table entry and work-array entry it reads, so nothing
// needs to start at zero.  The first call on a device looks up the arrays'
// device addresses (cudaGetSymbolAddress, with that device current); make that
// first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace {

constexpr size_t kScratchElems = size_t(1) << 23;  // doubles (64 MiB)
constexpr int kMaxN = 1024;                        // cells per axis
constexpr int kMaxM = kMaxN / 2;
// per axis: twM 2M + twN 2(M+1) + tw4N 2(M+1) + inv4sin (M+1) + eigenvalues (N+2)
// (a multiple of 4 keeps every axis slice 32-byte aligned)
constexpr int kAxisElems = (2 * kMaxM + 2 * (kMaxM + 1) + 2 * (kMaxM + 1) + (kMaxM + 1) + (kMaxN + 2) + 4 + 3) & ~3;

static __device__ __align__(256) double g_scratch[kScratchElems];
static __device__ __align__(256) double g_tables[3 * kAxisElems];

struct Addrs {
    double* scratch = nullptr;
    double* tables = nullptr;
};
constexpr int kMaxDevices = 64;
std::mutex g_mu;
Addrs g_addrs[kMaxDevices];

// Device addresses of the arrays for the current device (looked up once).
int device_addresses(Addrs* out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail((int)e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(CHZ_ERROR_INVALID_VALUE, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    Addrs& a = g_addrs[dev];
    if (!a.scratch) {
        void* s = nullptr;
        void* t = nullptr;
        e = cudaGetSymbolAddress(&s, g_scratch);
        if (e != cudaSuccess) return cuda_fail((int)e, "cudaGetSymbolAddress(scratch)");
        e = cudaGetSymbolAddress(&t, g_tables);
        if (e != cudaSuccess) return cuda_fail((int)e, "cudaGetSymbolAddress(tables)");
        a.scratch = static_cast<double*>(s);
        a.tables = static_cast<double*>(t);
    }
    *out = a;
    return CHZ_SUCCESS;
}

// Offsets of one axis' tables inside its slice of the table array.
struct AxisLayout {
    int twM, twN, tw4N, inv4sin, eig;
};
AxisLayout layout_for(int N) {
    const int M = N / 2;
    AxisLayout l;
    l.twM = 0;
    l.twN = l.twM + 2 * M;
    l.tw4N = l.twN + 2 * (M + 1);
    l.inv4sin = l.tw4N + 2 * (M + 1);
    l.eig = l.inv4sin + (M + 1);
    // keep the double2 tables 16-byte aligned
    l.twN = (l.twN + 1) & ~1;
    l.tw4N = (l.tw4N + 1) & ~1;
    return l;
}

// Twiddle, pre/post and eigenvalue tables of one axis (the same values the
// cached path computes on the host, here from the device's sincospi/cos).
__global__ void fill_axis_tables(double* base, int N, AxisLayout l, int bc, double pidiv, double shift,
                                 double d2) {
    const int M = N / 2;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N + 2; t += gridDim.x * blockDim.x) {
        double s, c;
        if (t < M) {
            sincospi(-2.0 * t / M, &s, &c);
            base[l.twM + 2 * t] = c;
            base[l.twM + 2 * t + 1] = s;
        }
        if (t <= M) {
            sincospi(-2.0 * t / N, &s, &c);
            base[l.twN + 2 * t] = c;
            base[l.twN + 2 * t + 1] = s;
            sincospi(-(double)t / (2.0 * N), &s, &c);
            base[l.tw4N + 2 * t] = c;
            base[l.tw4N + 2 * t + 1] = s;
            base[l.inv4sin + t] = (t == 0) ? 0.0 : 1.0 / (4.0 * sinpi((double)t / N));
        }
        const int mode = (bc == 0) ? t / 2 : t;
        base[l.eig + t] = (2.0 * cos(mode * pidiv + shift) - 2.0) * d2;
    }
}

int axis_tables(const AxisSolve& a, double* base, DeviceLineTables* tb, const double** eig, cudaStream_t s) {
    const AxisLayout l = layout_for(a.n);
    if (l.eig + a.n + 2 > kAxisElems) return fail(CHZ_ERROR_UNSUPPORTED_SIZE, "axis tables exceed capacity");
    tb->N = a.n;
    tb->M = a.n / 2;
    if (factor_radices(tb->M, &tb->rp) != 0) return fail(CHZ_ERROR_UNSUPPORTED_SIZE, "size %d not supported", a.n);
    tb->twM = base + l.twM;
    tb->twN = base + l.twN;
    tb->tw4N = base + l.tw4N;
    tb->inv4sin = base + l.inv4sin;
    *eig = base + l.eig;
    fill_axis_tables<<<(a.n + 2 + 255) / 256, 256, 0, s>>>(base, a.n, l, a.bc, a.pidiv, a.shift, a.d2);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail((int)e, "table fill");
    return CHZ_SUCCESS;
}

}  // namespace
}  // namespace chz

using namespace chz;

extern "C" int chz_helmholtz_solve_noalloc(double left, double right, int nx, int xbc, const double* bcl,
                                           const double* bcr, double bottom, double top, int ny, int ybc,
                                           const double* bcb, const double* bct, double front, double back,
                                           int nz, int zbc, const double* bcf, const double* bce, double lambda,
                                           double* f, void* stream) {
    g_last_error[0] = 0;
    int rc;
    AxisSolve X, Y, Z;
    if ((rc = setup_axis(nx, xbc, left, right, &X)) || (rc = setup_axis(ny, ybc, bottom, top, &Y)) ||
        (rc = setup_axis(nz, zbc, front, back, &Z)))
        return rc;
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    if (nx > kMaxN || ny > kMaxN || nz > kMaxN)
        return fail(CHZ_ERROR_UNSUPPORTED_SIZE, "allocation-free solve: at most %d cells per axis", kMaxN);
    const size_t need = (size_t)(nx + 2) * (ny + 2) * (nz + 2);
    if (need > kScratchElems)
        return fail(CHZ_ERROR_UNSUPPORTED_SIZE,
                    "allocation-free solve: (NX+2)(NY+2)(NZ+2) = %zu exceeds the %zu-value scratch array", need,
                    kScratchElems);
    if (!f) return fail(CHZ_ERROR_INVALID_VALUE, "f is NULL");
    if ((rc = check_faces(X, bcl, bcr, "x")) || (rc = check_faces(Y, bcb, bct, "y")) ||
        (rc = check_faces(Z, bcf, bce, "z")))
        return rc;
    Addrs ad;
    if ((rc = device_addresses(&ad))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DeviceLineTables tx, ty, tz;
    const double *ex, *ey, *ez;
    if ((rc = axis_tables(X, ad.tables, &tx, &ex, s)) || (rc = axis_tables(Y, ad.tables + kAxisElems, &ty, &ey, s)) ||
        (rc = axis_tables(Z, ad.tables + 2 * kAxisElems, &tz, &ez, s)))
        return rc;
    return run_solve_passes(X, Y, Z, tx, ty, tz, ex, ey, ez, bcl, bcr, bcb, bct, bcf, bce, lambda, f, ad.scratch, s);
}
