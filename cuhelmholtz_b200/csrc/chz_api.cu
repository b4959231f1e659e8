// Host side: argument checking, pass planning and the exported entry points
// (the extern "C" ABI of include/cuhelmholtz_b200.h and the reference's
// C++-linkage drop-in signatures of include/funcinterface.h and
// include/cuda_helmholtz_solver.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "chz_internal.h"
#include "cuhelmholtz_b200.h"
#include "cuda_helmholtz_solver.h"
#include "funcinterface.h"

namespace chz {

thread_local char g_last_error[512] = "";

int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_fail(int err, const char* where) {
    return fail(CHZ_ERROR_CUDA, "%s: %s", where, cudaGetErrorString((cudaError_t)err));
}

constexpr int kMaxN = 2048;

int check_len(int n, const char* axis) {
    if (n < 4 || n > kMaxN || (n & 1))
        return fail(CHZ_ERROR_UNSUPPORTED_SIZE, "%s size %d: need an even size in [4, %d]", axis, n, kMaxN);
    RadixPlan rp;
    if (factor_radices(n / 2, &rp) != 0)
        return fail(CHZ_ERROR_UNSUPPORTED_SIZE, "%s size %d: N/2 has a prime factor above 13", axis, n);
    return CHZ_SUCCESS;
}

int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

int tables_for(int n, int is_double, DeviceLineTables* t) {
    const int rc = get_line_tables(n, is_double, current_device(), t);
    if (rc == -1) return fail(CHZ_ERROR_UNSUPPORTED_SIZE, "size %d not supported", n);
    if (rc == (int)cudaErrorMemoryAllocation) return fail(CHZ_ERROR_ALLOC, "table allocation failed");
    if (rc != 0) return cuda_fail(rc, "table upload");
    return CHZ_SUCCESS;
}

namespace {

struct Dims {
    int nx, ny, nz;
};

// --------------------------------------------------------------------------
// do_transform planning
// --------------------------------------------------------------------------

int transform_impl(const double* src, double* dst, int nx, int ny, int nz, int kx, int ky, int kz,
                   cudaStream_t s) {
    DeviceLineTables tx, ty, tz;
    int rc;
    if ((rc = tables_for(nx, 1, &tx)) || (rc = tables_for(ny, 1, &ty)) || (rc = tables_for(nz, 1, &tz)))
        return rc;
    const long long sy = nx + 2;
    const long long sz = (long long)(nx + 2) * (ny + 2);
    int xi0, xi1, yi0, yi1, zi0, zi1, xo0, xo1, yo0, yo1, zo0, zo1;
    kind_in_window(kx, nx, xi0, xi1);
    kind_in_window(ky, ny, yi0, yi1);
    kind_in_window(kz, nz, zi0, zi1);
    kind_out_window(kx, nx, xo0, xo1);
    kind_out_window(ky, ny, yo0, yo1);
    kind_out_window(kz, nz, zo0, zo1);

    // x pass: rows (y, z) over the y and z input windows
    {
        const LineGeom g = line_geometry(nx, 1, true);
        PassArgs a{};
        a.kind = kx; a.kind2 = -1;
        a.u0 = yi0; a.nu = yi1 - yi0 + 1; a.v0 = zi0;
        a.in_su = sy; a.in_sv = sz; a.in_sl = 1;
        a.ld_lo = xi0; a.ld_hi = xi1;
        a.out_su = sy; a.out_sv = sz; a.out_sl = 1;
        a.st_lo = xo0; a.st_hi = xo1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, true, src, dst, a, tx, g, zi1 - zi0 + 1, s, "transform_x");
        if (rc) return cuda_fail(rc, "x pass");
    }
    // y pass: columns x over the x output window, planes z over the z input window
    {
        const LineGeom g = line_geometry(ny, 1, false);
        PassArgs a{};
        a.kind = ky; a.kind2 = -1;
        a.u0 = xo0; a.nu = xo1 - xo0 + 1; a.v0 = zi0;
        a.in_su = 1; a.in_sv = sz; a.in_sl = sy;
        a.ld_lo = yi0; a.ld_hi = yi1;
        a.out_su = 1; a.out_sv = sz; a.out_sl = sy;
        a.st_lo = yo0; a.st_hi = yo1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, dst, dst, a, ty, g, zi1 - zi0 + 1, s, "transform_y");
        if (rc) return cuda_fail(rc, "y pass");
    }
    // z pass: columns x over the x output window, rows y over the y output window
    {
        const LineGeom g = line_geometry(nz, 1, false);
        PassArgs a{};
        a.kind = kz; a.kind2 = -1;
        a.u0 = xo0; a.nu = xo1 - xo0 + 1; a.v0 = yo0;
        a.in_su = 1; a.in_sv = sy; a.in_sl = sz;
        a.ld_lo = zi0; a.ld_hi = zi1;
        a.out_su = 1; a.out_sv = sy; a.out_sl = sz;
        a.st_lo = zo0; a.st_hi = zo1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, dst, dst, a, tz, g, yo1 - yo0 + 1, s, "transform_z");
        if (rc) return cuda_fail(rc, "z pass");
    }
    return CHZ_SUCCESS;
}

int check_kinds(int kx, int ky, int kz) {
    if (kx < 0 || kx > 7 || ky < 0 || ky > 7 || kz < 0 || kz > 7)
        return fail(CHZ_ERROR_INVALID_VALUE, "transform kind out of range 0..7");
    return CHZ_SUCCESS;
}

int do_transform_common(double* d_data, double* d_out, int nx, int ny, int nz, int kx, int ky, int kz,
                        void* stream, bool require_cube) {
    g_last_error[0] = 0;
    int rc;
    if (!d_data) return fail(CHZ_ERROR_INVALID_VALUE, "d_data is NULL");
    if ((rc = check_kinds(kx, ky, kz))) return rc;
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    const bool inplace = (d_out == nullptr || d_out == d_data);
    if (inplace && require_cube && !(nx == ny && nx == nz))
        return fail(CHZ_ERROR_NOT_CUBIC, "the matrix for inplace transform must be cubic!");
    double* dst = inplace ? d_data : d_out;
    return transform_impl(d_data, dst, nx, ny, nz, kx, ky, kz, static_cast<cudaStream_t>(stream));
}

// --------------------------------------------------------------------------
// Helmholtz solver planning
// --------------------------------------------------------------------------

}  // namespace

int setup_axis(int n, int bc, double lo, double hi, AxisSolve* a) {
    a->n = n;
    a->bc = bc;
    switch (bc) {
        case 0: a->s = 0; a->e = n - 1; a->kf = kR2C; a->ki = kC2R; break;
        case 1: a->s = 1; a->e = n - 1; a->kf = kDST1; a->ki = kDST1; break;
        case 2: a->s = 1; a->e = n; a->kf = kDST3; a->ki = kDST2; break;
        case 3: a->s = 0; a->e = n; a->kf = kDCT1; a->ki = kDCT1; break;
        case 4: a->s = 0; a->e = n - 1; a->kf = kDCT3; a->ki = kDCT2; break;
        default: return fail(CHZ_ERROR_INVALID_VALUE, "bad boundary condition %d", bc);
    }
    a->sp0 = a->s;
    a->sp1 = (bc == 0) ? n + 1 : a->e;
    a->d = n / (hi - lo);
    a->d2 = a->d * a->d;
    const double pi = 3.14159265358979323846;
    a->shift = 0.0;
    if (bc == 2) a->shift = -0.5 * pi / n;
    if (bc == 4) a->shift = 0.5 * pi / n;
    a->pidiv = pi / n;
    if (bc == 0) a->pidiv *= 2;
    if (!(std::isfinite(a->d)) || a->d == 0.0)
        return fail(CHZ_ERROR_INVALID_VALUE, "degenerate domain extent");
    return CHZ_SUCCESS;
}

namespace {

// Eigenvalue tables (2 cos(mode*pidiv + shift) - 2) * d^2 per padded entry,
// cached on the device by (n, bc, d2, device).
struct EigCache {
    std::mutex mu;
    std::map<std::tuple<int, int, unsigned long long, int>, double*> map;
};
EigCache& eig_cache() {
    static EigCache* c = new EigCache();
    return *c;
}

}  // namespace

int eig_table(const AxisSolve& a, const double** out) {
    EigCache& c = eig_cache();
    unsigned long long bits;
    std::memcpy(&bits, &a.d2, sizeof(bits));
    auto key = std::make_tuple(a.n, a.bc, bits, current_device());
    std::lock_guard<std::mutex> lk(c.mu);
    auto it = c.map.find(key);
    if (it != c.map.end()) {
        *out = it->second;
        return CHZ_SUCCESS;
    }
    std::vector<double> h(a.n + 2);
    for (int idx = 0; idx < a.n + 2; ++idx) {
        const int mode = (a.bc == 0) ? idx / 2 : idx;
        h[idx] = (2.0 * std::cos(mode * a.pidiv + a.shift) - 2.0) * a.d2;
    }
    double* d = nullptr;
    if (cudaMalloc(&d, sizeof(double) * h.size()) != cudaSuccess)
        return fail(CHZ_ERROR_ALLOC, "eigenvalue table allocation failed");
    if (cudaMemcpy(d, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return fail(CHZ_ERROR_CUDA, "eigenvalue table upload failed");
    }
    c.map[key] = d;
    *out = d;
    return CHZ_SUCCESS;
}

// `int ratio = NX/2 * NY/2 * NZ/2`, doubled per periodic axis (solver.cu:211-215)
double solver_scale(const AxisSolve& x, const AxisSolve& y, const AxisSolve& z) {
    long long r = x.n / 2;
    r = r * y.n / 2;
    r = r * z.n / 2;
    if (x.bc == 0) r *= 2;
    if (y.bc == 0) r *= 2;
    if (z.bc == 0) r *= 2;
    return 1.0 / (double)r;
}

size_t padded_elems(int nx, int ny, int nz) { return (size_t)(nx + 2) * (ny + 2) * (nz + 2); }

int check_faces(const AxisSolve& a, const double* lo, const double* hi, const char* name) {
    if ((a.bc == 3 || a.bc == 4) && !lo) return fail(CHZ_ERROR_INVALID_VALUE, "%s: lower Neumann face is NULL", name);
    if ((a.bc == 2 || a.bc == 3) && !hi) return fail(CHZ_ERROR_INVALID_VALUE, "%s: upper Neumann face is NULL", name);
    return CHZ_SUCCESS;
}

// Division of the 19-point variant (_nonpoisson_devide_19points_,
// _cuda_helmholtz_.inl:255-274, left commented out in the reference at
// cuda_helmholtz_solver.cu:325,338): on the spectral window, with
// c_a = cos(m_a pi / N_a),
//   value *= (1/2 + (c_i + c_j + c_k) / 6)
//          / ((2/3 (c_i c_j + c_i c_k + c_j c_k + c_i + c_j + c_k) - 4) h^-2 + lambda)
// -- the eigenvalues of the compact 19-point Laplacian and of its 7-point
// right-hand-side filter.  The mode (0,0,0) is set to 0 when its denominator
// is 0 (lambda = 0, Neumann on every axis), where the reference divides by 0.
__global__ void divide19(double* ws, long long wy, long long wz, int xs, int xe, int ys, int ys_n, int zs,
                         double pix, double piy, double piz, double d2, double lam, int zero_mode) {
    const int i = xs + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = ys + blockIdx.y;
    const int k = zs + blockIdx.z;
    if (i > xe || j >= ys + ys_n) return;
    const double ci = cos(i * pix), cj = cos(j * piy), ck = cos(k * piz);
    const double coef = (2.0 / 3.0 * (ci * cj + ci * ck + cj * ck + ci + cj + ck) - 4.0) * d2 + lam;
    const double filt = 0.5 + (ci + cj + ck) / 6.0;
    const long long o = k * wz + j * wy + i;
    ws[o] = (zero_mode && i == 0 && j == 0 && k == 0) ? 0.0 : ws[o] * filt / coef;
}

// The five line passes and the periodic planes of one FP64 solve, with the
// per-axis tables and the work array given by the caller.  stencil19: the
// z pass is split around the 19-point division (divide19) instead of fusing
// the 7-point one.
int run_solve_passes(const AxisSolve& X, const AxisSolve& Y, const AxisSolve& Z, const DeviceLineTables& tx,
                     const DeviceLineTables& ty, const DeviceLineTables& tz, const double* ex, const double* ey,
                     const double* ez, const double* bcl, const double* bcr, const double* bcb,
                     const double* bct, const double* bcf, const double* bce, double lambda, double* f,
                     double* ws, cudaStream_t s, bool stencil19) {
    int rc;
    const int nx = X.n, ny = Y.n, nz = Z.n;
    const long long fy = nx + 1, fz = (long long)(nx + 1) * (ny + 1);
    const long long wy = nx + 2, wz = (long long)(nx + 2) * (ny + 2);

    BcArgs bc{};
    bc.xbc = X.bc; bc.ybc = Y.bc; bc.zbc = Z.bc;
    bc.xs = X.s; bc.xe = X.e; bc.ys = Y.s; bc.ye = Y.e; bc.zs = Z.s; bc.ze = Z.e;
    bc.nx = nx; bc.ny = ny; bc.nz = nz;
    bc.dx = X.d; bc.dy = Y.d; bc.dz = Z.d;
    bc.dx2 = X.d2; bc.dy2 = Y.d2; bc.dz2 = Z.d2;
    bc.f = f;
    bc.bcl = bcl; bc.bcr = bcr; bc.bcb = bcb; bc.bct = bct; bc.bcf = bcf; bc.bce = bce;

    // pass 1: x forward, f -> ws, boundary terms fused into the load
    {
        const LineGeom g = line_geometry(nx, 1, true);
        PassArgs a{};
        a.kind = X.kf; a.kind2 = -1;
        a.u0 = Y.s; a.nu = Y.e - Y.s + 1; a.v0 = Z.s;
        a.in_su = fy; a.in_sv = fz; a.in_sl = 1;
        a.ld_lo = X.s; a.ld_hi = X.e;
        a.out_su = wy; a.out_sv = wz; a.out_sl = 1;
        a.st_lo = X.sp0; a.st_hi = X.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        a.has_bc = 1; a.bc = bc;
        rc = launch_line_pass(1, kIoF64, kIoF64, true, f, ws, a, tx, g, Z.e - Z.s + 1, s, "solve_x_fwd");
        if (rc) return cuda_fail(rc, "solver pass 1");
    }
    // pass 2: y forward, in place
    {
        const LineGeom g = line_geometry(ny, 1, false);
        PassArgs a{};
        a.kind = Y.kf; a.kind2 = -1;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = Z.s;
        a.in_su = 1; a.in_sv = wz; a.in_sl = wy;
        a.ld_lo = Y.s; a.ld_hi = Y.e;
        a.out_su = 1; a.out_sv = wz; a.out_sl = wy;
        a.st_lo = Y.sp0; a.st_hi = Y.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, ws, ws, a, ty, g, Z.e - Z.s + 1, s, "solve_y_fwd");
        if (rc) return cuda_fail(rc, "solver pass 2");
    }
    // pass 3: z forward, eigenvalue division, z inverse, in place
    if (stencil19) {
        const LineGeom g = line_geometry(nz, 1, false);
        PassArgs a{};
        a.kind = Z.kf; a.kind2 = -1;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = Y.sp0;
        a.in_su = 1; a.in_sv = wy; a.in_sl = wz;
        a.ld_lo = Z.s; a.ld_hi = Z.e;
        a.out_su = 1; a.out_sv = wy; a.out_sl = wz;
        a.st_lo = Z.sp0; a.st_hi = Z.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, ws, ws, a, tz, g, Y.sp1 - Y.sp0 + 1, s, "solve19_z_fwd");
        if (rc) return cuda_fail(rc, "solver pass 3 (forward)");
        const dim3 blk(128, 1, 1);
        const dim3 grd((X.sp1 - X.sp0 + 128) / 128, Y.sp1 - Y.sp0 + 1, Z.sp1 - Z.sp0 + 1);
        const bool zm = lambda == 0.0 && X.bc == 3 && Y.bc == 3 && Z.bc == 3;
        trace_begin(s, "solve19_divide");
        divide19<<<grd, blk, 0, s>>>(ws, wy, wz, X.sp0, X.sp1, Y.sp0, Y.sp1 - Y.sp0 + 1, Z.sp0, X.pidiv, Y.pidiv,
                                      Z.pidiv, X.d2, lambda, zm ? 1 : 0);
        count_launch();
        trace_end(s);
        if ((rc = (int)cudaGetLastError())) return cuda_fail(rc, "19-point division");
        a.kind = Z.ki;
        a.ld_lo = Z.sp0; a.ld_hi = Z.sp1;
        a.st_lo = Z.s; a.st_hi = Z.e;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, ws, ws, a, tz, g, Y.sp1 - Y.sp0 + 1, s, "solve19_z_inv");
        if (rc) return cuda_fail(rc, "solver pass 3 (inverse)");
    } else {
        const LineGeom g = line_geometry(nz, 1, false);
        PassArgs a{};
        a.kind = Z.kf; a.kind2 = Z.ki;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = Y.sp0;
        a.in_su = 1; a.in_sv = wy; a.in_sl = wz;
        a.ld_lo = Z.s; a.ld_hi = Z.e;
        a.out_su = 1; a.out_sv = wy; a.out_sl = wz;
        a.st_lo = Z.s; a.st_hi = Z.e;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        a.has_div = 1;
        a.dv.ex = ex; a.dv.ey = ey; a.dv.ez = ez;
        a.dv.lambda = lambda;
        a.dv.perturb = (lambda == 0.0 && (X.bc == 0 || X.bc == 3) && (Y.bc == 0 || Y.bc == 3) &&
                        (Z.bc == 0 || Z.bc == 3));
        a.dv.xz_hi = X.bc == 0 ? 1 : 0;
        a.dv.yz_hi = Y.bc == 0 ? 1 : 0;
        a.dv.zz_hi = Z.bc == 0 ? 1 : 0;
        a.dv.lo = Z.sp0; a.dv.hi = Z.sp1;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, ws, ws, a, tz, g, Y.sp1 - Y.sp0 + 1, s, "solve_z_fwd_div_inv");
        if (rc) return cuda_fail(rc, "solver pass 3");
    }
    // pass 4: y inverse, in place
    {
        const LineGeom g = line_geometry(ny, 1, false);
        PassArgs a{};
        a.kind = Y.ki; a.kind2 = -1;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = Z.s;
        a.in_su = 1; a.in_sv = wz; a.in_sl = wy;
        a.ld_lo = Y.sp0; a.ld_hi = Y.sp1;
        a.out_su = 1; a.out_sv = wz; a.out_sl = wy;
        a.st_lo = Y.s; a.st_hi = Y.e;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, ws, ws, a, ty, g, Z.e - Z.s + 1, s, "solve_y_inv");
        if (rc) return cuda_fail(rc, "solver pass 4");
    }
    // pass 5: x inverse, ws -> f, scaled by the reference's ratio
    {
        const LineGeom g = line_geometry(nx, 1, true);
        PassArgs a{};
        a.kind = X.ki; a.kind2 = -1;
        a.u0 = Y.s; a.nu = Y.e - Y.s + 1; a.v0 = Z.s;
        a.in_su = wy; a.in_sv = wz; a.in_sl = 1;
        a.ld_lo = X.sp0; a.ld_hi = X.sp1;
        a.out_su = fy; a.out_sv = fz; a.out_sl = 1;
        a.st_lo = X.s; a.st_hi = X.e;
        a.scale = solver_scale(X, Y, Z); a.use_scale = 1;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, true, ws, f, a, tx, g, Z.e - Z.s + 1, s, "solve_x_inv");
        if (rc) return cuda_fail(rc, "solver pass 5");
    }
    rc = launch_periodic_fixup(f, nx, ny, nz, X.bc, Y.bc, Z.bc, s);
    if (rc) return cuda_fail(rc, "periodic planes");
    return CHZ_SUCCESS;
}

namespace {

int solve_fp64(const AxisSolve& X, const AxisSolve& Y, const AxisSolve& Z, const double* bcl,
               const double* bcr, const double* bcb, const double* bct, const double* bcf,
               const double* bce, double lambda, double* f, double* ws, cudaStream_t s, bool stencil19 = false) {
    int rc;
    DeviceLineTables tx, ty, tz;
    if ((rc = tables_for(X.n, 1, &tx)) || (rc = tables_for(Y.n, 1, &ty)) || (rc = tables_for(Z.n, 1, &tz)))
        return rc;
    const double *ex, *ey, *ez;
    if ((rc = eig_table(X, &ex)) || (rc = eig_table(Y, &ey)) || (rc = eig_table(Z, &ez))) return rc;
    return run_solve_passes(X, Y, Z, tx, ty, tz, ex, ey, ez, bcl, bcr, bcb, bct, bcf, bce, lambda, f, ws, s,
                            stencil19);
}

// Library-owned workspaces, one grow-only buffer per (device, stream).
struct WsCache {
    std::mutex mu;
    std::map<std::pair<int, void*>, std::pair<void*, size_t>> map;
};
WsCache& ws_cache() {
    static WsCache* c = new WsCache();
    return *c;
}

}  // namespace

int cached_workspace(void* stream, size_t bytes, void** out) {
    WsCache& c = ws_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    auto key = std::make_pair(current_device(), stream);
    auto& slot = c.map[key];
    if (slot.second < bytes) {
        if (slot.first) {
            cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
            cudaFree(slot.first);
            slot.first = nullptr;
            slot.second = 0;
        }
        void* p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess)
            return fail(CHZ_ERROR_ALLOC, "workspace allocation of %zu bytes failed", bytes);
        slot.first = p;
        slot.second = bytes;
    }
    *out = slot.first;
    return CHZ_SUCCESS;
}

namespace {

int solve_common(double left, double right, int nx, int xbc, const double* bcl, const double* bcr,
                 double bottom, double top, int ny, int ybc, const double* bcb, const double* bct,
                 double front, double back, int nz, int zbc, const double* bcf, const double* bce,
                 double lambda, double* f, void* ws, size_t ws_bytes, bool own_ws, void* stream,
                 bool stencil19 = false) {
    g_last_error[0] = 0;
    int rc;
    AxisSolve X, Y, Z;
    if ((rc = setup_axis(nx, xbc, left, right, &X)) || (rc = setup_axis(ny, ybc, bottom, top, &Y)) ||
        (rc = setup_axis(nz, zbc, front, back, &Z)))
        return rc;
    if (stencil19) {
        // the reference's 19-point division takes one grid spacing (dx2) and
        // no half-sample shift: cubic cells, codes 1 and 3
        auto ok = [](int bc) { return bc == 1 || bc == 3; };
        if (!ok(X.bc) || !ok(Y.bc) || !ok(Z.bc))
            return fail(CHZ_ERROR_INVALID_VALUE, "the 19-point solve takes boundary codes 1 and 3 only");
        const double tol = 1e-12 * X.d2;
        if (std::fabs(X.d2 - Y.d2) > tol || std::fabs(X.d2 - Z.d2) > tol)
            return fail(CHZ_ERROR_INVALID_VALUE, "the 19-point solve needs equal grid spacing on all axes");
    }
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    if (!f) return fail(CHZ_ERROR_INVALID_VALUE, "f is NULL");
    if ((rc = check_faces(X, bcl, bcr, "x")) || (rc = check_faces(Y, bcb, bct, "y")) ||
        (rc = check_faces(Z, bcf, bce, "z")))
        return rc;
    const size_t need = chz_helmholtz_workspace_size(nx, ny, nz, 0);
    if (own_ws) {
        if ((rc = cached_workspace(stream, need, &ws))) return rc;
    } else {
        if (!ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 255))
            return fail(CHZ_ERROR_WORKSPACE, "workspace needs %zu bytes, 256-byte aligned", need);
    }
    return solve_fp64(X, Y, Z, bcl, bcr, bcb, bct, bcf, bce, lambda, f, static_cast<double*>(ws),
                      static_cast<cudaStream_t>(stream), stencil19);
}

}  // namespace
}  // namespace chz

using namespace chz;

extern "C" {

int chz_version(void) { return 100; }

const char* chz_status_string(int status) {
    switch (status) {
        case CHZ_SUCCESS: return "CHZ_SUCCESS";
        case CHZ_ERROR_INVALID_VALUE: return "CHZ_ERROR_INVALID_VALUE";
        case CHZ_ERROR_UNSUPPORTED_SIZE: return "CHZ_ERROR_UNSUPPORTED_SIZE";
        case CHZ_ERROR_NOT_CUBIC: return "CHZ_ERROR_NOT_CUBIC";
        case CHZ_ERROR_CUDA: return "CHZ_ERROR_CUDA";
        case CHZ_ERROR_ALLOC: return "CHZ_ERROR_ALLOC";
        case CHZ_ERROR_WORKSPACE: return "CHZ_ERROR_WORKSPACE";
        case CHZ_ERROR_TIMEOUT: return "CHZ_ERROR_TIMEOUT";
        default: return "CHZ_ERROR_UNKNOWN";
    }
}

const char* chz_last_error(void) { return g_last_error; }

int chz_do_transform(double* d_data, double* d_out, int nx, int ny, int nz, int x_kind, int y_kind,
                     int z_kind, void* stream) {
    return do_transform_common(d_data, d_out, nx, ny, nz, x_kind, y_kind, z_kind, stream, true);
}

int chz_do_transform_any(double* d_data, double* d_out, int nx, int ny, int nz, int x_kind, int y_kind,
                         int z_kind, void* stream) {
    return do_transform_common(d_data, d_out, nx, ny, nz, x_kind, y_kind, z_kind, stream, false);
}

size_t chz_helmholtz_workspace_size(int nx, int ny, int nz, int precision) {
    if (nx < 1 || ny < 1 || nz < 1) return 0;
    const size_t pe = padded_elems(nx, ny, nz);
    size_t bytes = pe * sizeof(double);
    if (precision == 1) {
        // FP32 work array + FP64 solution array + two FP64 norm accumulators,
        // each piece 256-byte aligned
        auto r256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
        // (FP32 rows padded to a multiple of 4 values: 16-byte row pitch)
        const size_t pe32 = (size_t)((nx + 2 + 3) & ~3) * (ny + 2) * (nz + 2);
        bytes = r256(pe32 * sizeof(float)) + r256((size_t)(nx + 1) * (ny + 1) * (nz + 1) * sizeof(double)) + 256;
    }
    return (bytes + 255) & ~(size_t)255;
}

int chz_helmholtz_solve_19pt(double left, double right, int nx, int xbc, const double* bcl, const double* bcr,
                             double bottom, double top, int ny, int ybc, const double* bcb, const double* bct,
                             double front, double back, int nz, int zbc, const double* bcf, const double* bce,
                             double lambda, double* f, void* stream) {
    return solve_common(left, right, nx, xbc, bcl, bcr, bottom, top, ny, ybc, bcb, bct, front, back, nz, zbc, bcf,
                        bce, lambda, f, nullptr, 0, true, stream, true);
}

int chz_helmholtz_solve(double left, double right, int nx, int xbc, const double* bcl, const double* bcr,
                        double bottom, double top, int ny, int ybc, const double* bcb, const double* bct,
                        double front, double back, int nz, int zbc, const double* bcf, const double* bce,
                        double lambda, double* f, void* stream) {
    return solve_common(left, right, nx, xbc, bcl, bcr, bottom, top, ny, ybc, bcb, bct, front, back, nz,
                        zbc, bcf, bce, lambda, f, nullptr, 0, true, stream);
}

int chz_helmholtz_solve_ws(double left, double right, int nx, int xbc, const double* bcl, const double* bcr,
                           double bottom, double top, int ny, int ybc, const double* bcb, const double* bct,
                           double front, double back, int nz, int zbc, const double* bcf, const double* bce,
                           double lambda, double* f, void* workspace, size_t workspace_bytes, void* stream) {
    return solve_common(left, right, nx, xbc, bcl, bcr, bottom, top, ny, ybc, bcb, bct, front, back, nz,
                        zbc, bcf, bce, lambda, f, workspace, workspace_bytes, false, stream);
}

int chz_release_cached(void) {
    cudaDeviceSynchronize();
    const int dev = current_device();
    {
        WsCache& c = ws_cache();
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto it = c.map.begin(); it != c.map.end();) {
            if (it->first.first == dev) {
                if (it->second.first) cudaFree(it->second.first);
                it = c.map.erase(it);
            } else {
                ++it;
            }
        }
    }
    {
        EigCache& c = eig_cache();
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto it = c.map.begin(); it != c.map.end();) {
            if (std::get<3>(it->first) == dev) {
                cudaFree(it->second);
                it = c.map.erase(it);
            } else {
                ++it;
            }
        }
    }
    return CHZ_SUCCESS;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The reference's C++-linkage signatures (drop-in).  Synchronous, and on error
// they print and exit the process as the reference does.
// ---------------------------------------------------------------------------

static void exit_on(int rc, int code) {
    if (rc == CHZ_SUCCESS) return;
    printf("%s\n", chz_last_error());
    exit(code);
}

// After the synchronous entry points' device synchronisation: a CUDA error,
// or a kernel wait that ran out (its results are not valid), ends the process
// as the reference's CUDA error checks do (funcinterface.cu:104-107,
// cuda_helmholtz_solver.cu:22-29).
static void exit_on_device_error(int code) {
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        printf("CUDA ERROR: %s !\n", cudaGetErrorString(e));
        exit(code);
    }
    const int flags = chz_debug_flags(1);
    if (flags != 0) {
        printf("cuhelmholtz_b200: a kernel wait ran out (flags %d)\n", flags);
        exit(code);
    }
}

// funcinterface.cu:25-40
void do_transform(double* d_data, double* d_out, int NX, int NY, int NZ, transform_kind X_TRANS,
                  transform_kind Y_TRANS, transform_kind Z_TRANS) {
    const int rc = chz_do_transform(d_data, d_out, NX, NY, NZ, X_TRANS, Y_TRANS, Z_TRANS, nullptr);
    if (rc == CHZ_ERROR_NOT_CUBIC) {
        printf("the matrix for inplace transform must be cubic!\n");
        exit(0);
    }
    exit_on(rc, 0);
    exit_on_device_error(0);
}

// funcinterface.cu:200-334
void do_transform_nocubic(double* d_data, double* d_out, int NX, int NY, int NZ, transform_kind X_TRANS,
                          transform_kind Y_TRANS, transform_kind Z_TRANS) {
    exit_on(chz_do_transform_any(d_data, d_out, NX, NY, NZ, X_TRANS, Y_TRANS, Z_TRANS, nullptr), 0);
    exit_on_device_error(0);
}

// funcinterface.cu:42-198
void do_transform_cubic(double* d_data, int NX, int NY, int NZ, transform_kind X_TRANS,
                        transform_kind Y_TRANS, transform_kind Z_TRANS) {
    exit_on(chz_do_transform_any(d_data, d_data, NX, NY, NZ, X_TRANS, Y_TRANS, Z_TRANS, nullptr), 0);
    exit_on_device_error(0);
}

// funcinterface.cu:337-342
void freeMemory_cubic() {}

// cuda_helmholtz_solver.cu:33-380
int cuda_helmholtz_solver(double left, double right, int NX, int xbc, double* bcl, double* bcr, double bottom,
                          double top, int NY, int ybc, double* bcb, double* bct, double front, double back,
                          int NZ, int zbc, double* bcf, double* bce, double lambda, double* f) {
    if (xbc < 0 || xbc > 4 || ybc < 0 || ybc > 4 || zbc < 0 || zbc > 4) {
        printf("bad boundary condition\n");
        exit(1);
    }
    const int rc = chz_helmholtz_solve(left, right, NX, xbc, bcl, bcr, bottom, top, NY, ybc, bcb, bct, front,
                                       back, NZ, zbc, bcf, bce, lambda, f, nullptr);
    if (rc != CHZ_SUCCESS) {
        std::printf("%s\n", chz_last_error());
        exit(-1);
    }
    exit_on_device_error(-1);
    return 0;
}
