// FP32 transforms with FP64 iterative refinement: chz_helmholtz_solve_refined;
// and the solve with FISHPACK's PERTRB, chz_helmholtz_solve_pertrb (end of file).
//
// The system is the reference's (cuda_helmholtz_solver.cu:33-380): A u = b on
// the unknown windows, b = f with the boundary terms of _3d_bc*_ini_*
// (_cuda_helmholtz_.inl:70-227), A the 7-point operator with homogeneous
// closures (Dirichlet neighbours 0, Neumann ghost = mirror, periodic wrap).
//
//   u0 = S32(b);  repeat: r = b - A u (FP64), c = S32(r), u += c
//
// Singular case (lambda = 0, every code 0 or 3): the solve removes the
// constant mode, whose coefficient is the weighted sum 1^T W x over the window
// (W = 1/2 at Neumann boundary nodes, per axis; 1^T W A = 0).  The residual
// keeps b's incompatible part c_b = 1^T W b / 1^T W 1 forever, so it is
// subtracted in FP64 before r is rounded to FP32, and the constant mode that
// FP32 round-off leaves in u (invisible to the residual) is removed at the end.
//
// S32 is the five-pass diagonal solve with FP32 transforms (FP64 tables
// rounded to FP32, eigenvalue division in FP64); r is formed in FP64 and stored
// as FP32 straight into the work array, which the next correction's first pass
// transforms in place; the last pass of each correction adds c into the FP64
// solution u (and the final one writes u + c into f).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace {

struct ResidualArgs {
    BcArgs bc;                 // b = f + boundary terms
    const double* u;           // (NZ+1)(NY+1)(NX+1), same layout as f
    float* r;                  // padded (NZ+2)(NY+2)(pitch32(NX)) work array
    long long ry, rz;          // its row and plane pitch
    double lambda;
    double* sums;              // [0] += r^2, [1] += b^2
    const double* shift;       // singular case: *shift * inv_w is subtracted from r
    double inv_w;
};

// Row pitch (values) of the FP32 work array: NX + 2 rounded up to a multiple
// of 4, so that rows start on 16-byte boundaries (bulk tensor copies).
__host__ __device__ __forceinline__ long long pitch32(int nx) { return (nx + 2 + 3) & ~3; }

// Weight of node (i, j, k) in the constant mode's coefficient.
__device__ __forceinline__ double mode_weight(const BcArgs& b, int i, int j, int k) {
    double w = 1.0;
    if (b.xbc == 3 && (i == 0 || i == b.nx)) w *= 0.5;
    if (b.ybc == 3 && (j == 0 || j == b.ny)) w *= 0.5;
    if (b.zbc == 3 && (k == 0 || k == b.nz)) w *= 0.5;
    return w;
}

__device__ __forceinline__ void block_add(double v, double* out) {
    __shared__ double part[32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) part[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? part[lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) atomicAdd(out, v);
    }
}

// out += 1^T W x over the window, x = b (f with boundary terms) when u is
// NULL, else u.
__global__ void mode_sum(BcArgs b, const double* u, double* out) {
    const int i = b.xs + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = b.ys + blockIdx.y;
    const int k = b.zs + blockIdx.z;
    double v = 0.0;
    if (i <= b.xe) {
        const long long o = (long long)k * (b.nx + 1) * (b.ny + 1) + (long long)j * (b.nx + 1) + i;
        v = mode_weight(b, i, j, k) * (u ? u[o] : bc_terms(b.f[o], b, i, j, k));
    }
    block_add(v, out);
}

// u -= (*sum) * inv_w on the window.
__global__ void remove_mode(double* u, BcArgs b, const double* sum, double inv_w) {
    const int i = b.xs + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = b.ys + blockIdx.y;
    const int k = b.zs + blockIdx.z;
    if (i > b.xe) return;
    const long long o = (long long)k * (b.nx + 1) * (b.ny + 1) + (long long)j * (b.nx + 1) + i;
    u[o] -= *sum * inv_w;
}

// r = b - A u at the unknown nodes, with A's homogeneous closures: Dirichlet
// neighbours are 0 (their values are in b), a Neumann ghost mirrors the
// interior neighbour (the flux is in b), periodic neighbours wrap.
//
// A block of 32 x 8 threads marches up kResZ planes of a 32 x 8 column.  The u
// values of each plane, with a one-point halo, and the f values of the
// column are staged in shared memory by cp.async, kAhead planes ahead of the
// plane being computed (rings of kRing plane tiles); the closures are folded
// into the halo values as they are loaded, so the stencil itself reads only
// shared memory.
constexpr int kResX = 32, kResY = 8, kResZ = 32;
constexpr int kHX = kResX + 2, kHY = kResY + 2, kHalo = kHX * kHY;
constexpr int kAhead = 5;  // planes requested ahead of the computed one
constexpr int kRing = 8;   // >= kAhead + 3: a load reuses the slot of plane k - 3

// Source index along one axis for window-relative neighbour g (one step
// outside the window at most): -1 when the value is 0 (Dirichlet neighbour).
__device__ __forceinline__ int closure_index(int g, int s, int e, int n, int bc) {
    if (g >= s && g <= e) return g;
    if (g == s - 1) {
        if (bc == 0) return n - 1;             // periodic: s = 0
        if (bc == 3 || bc == 4) return s + 1;  // Neumann mirror
        return -1;                             // Dirichlet
    }
    if (g == e + 1) {
        if (bc == 0) return 0;
        if (bc == 2 || bc == 3) return e - 1;
        return -1;
    }
    return -1;  // beyond the halo: never read
}

// Per-thread copy plan of one plane tile: the (x, y) offsets of the (at most
// two) halo entries this thread copies, or -1 when the entry is 0
// (Dirichlet neighbour, or outside the halo); the z closure is applied per
// plane.
struct HaloPlan {
    long long off[2];
    long long foff;  // the thread's own point in f, or -1
};

__device__ __forceinline__ HaloPlan halo_plan(const BcArgs& b, int i0, int j0, long long sy, int tid) {
    HaloPlan h;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int e = tid + r * kResX * kResY;
        h.off[r] = -1;
        if (e < kHalo) {
            const int hy = e / kHX, hx = e - hy * kHX;
            const int ii = closure_index(i0 - 1 + hx, b.xs, b.xe, b.nx, b.xbc);
            const int jj = closure_index(j0 - 1 + hy, b.ys, b.ye, b.ny, b.ybc);
            if (ii >= 0 && jj >= 0) h.off[r] = (long long)jj * sy + ii;
        }
    }
    const int ty = tid / kResX, tx = tid - ty * kResX;
    const int i = i0 + tx, j = j0 + ty;
    h.foff = (i <= b.xe && j <= b.ye) ? (long long)j * sy + i : -1;
    return h;
}

// Issues the copies of plane p (u with halo, f of the column) and commits
// them as one group.
__device__ __forceinline__ void load_plane(double* tile, double* ftile, const double* u, const BcArgs& b,
                                           const HaloPlan& h, int p, long long sz, int tid) {
    const int kk = closure_index(p, b.zs, b.ze, b.nz, b.zbc);
    const long long base = (long long)kk * sz;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int e = tid + r * kResX * kResY;
        if (e < kHalo) {
            const bool valid = kk >= 0 && h.off[r] >= 0;
            cp_async_elem<8>(tile + e, valid ? u + base + h.off[r] : u, valid);
        }
    }
    const bool fv = p >= b.zs && p <= b.ze && h.foff >= 0;
    cp_async_elem<8>(ftile + tid, fv ? b.f + (long long)p * sz + h.foff : b.f, fv);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__global__ void __launch_bounds__(kResX * kResY) residual_kernel(ResidualArgs a) {
    __shared__ __align__(16) double ring[kRing][kHalo];
    __shared__ __align__(16) double fring[kRing][kResX * kResY];
    const BcArgs& b = a.bc;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kResX + tx;
    const int i0 = b.xs + blockIdx.x * kResX, j0 = b.ys + blockIdx.y * kResY;
    const int i = i0 + tx, j = j0 + ty;
    const int k0 = b.zs + blockIdx.z * kResZ;
    const int k1 = min(k0 + kResZ - 1, b.ze);
    const long long sy = b.nx + 1, sz = (long long)(b.nx + 1) * (b.ny + 1);
    const bool act = i <= b.xe && j <= b.ye;
    const bool side = (i == b.xs || i == b.xe || j == b.ys || j == b.ye);
    const double shift = a.shift ? *a.shift * a.inv_w : 0.0;
    double r2 = 0.0, b2 = 0.0;
    const HaloPlan hp = halo_plan(b, i0, j0, sy, tid);
    // plane p lives in slot (p - k0 + 1) & (kRing - 1); planes k0 - 1 .. k0 + kAhead - 1 first
    for (int q = 0; q < kAhead + 1; ++q) {
        const int p = k0 - 1 + q;
        if (p <= k1 + 1) load_plane(ring[q], fring[q], a.u, b, hp, p, sz, tid);
        else asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    const int c = (ty + 1) * kHX + tx + 1;
    for (int k = k0; k <= k1; ++k) {
        const int q = k - k0;  // slot of plane k - 1 is q & (kRing - 1)
        // planes up to k + 1 have landed (planes k + 2 .. k + kAhead - 1 may be in flight)
        asm volatile("cp.async.wait_group %0;\n" ::"n"(kAhead - 2) : "memory");
        __syncthreads();  // also: every thread is done with plane k - 3's slot
        {
            const int p = k + kAhead;
            const int sl = (q + kAhead + 1) & (kRing - 1);
            if (p <= k1 + 1) load_plane(ring[sl], fring[sl], a.u, b, hp, p, sz, tid);
            else asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
        if (act) {
            const double* lo = ring[q & (kRing - 1)];
            const double* mid = ring[(q + 1) & (kRing - 1)];
            const double* hi = ring[(q + 2) & (kRing - 1)];
            const double uc = mid[c];
            const double au = (((mid[c - 1] - 2.0 * uc + mid[c + 1]) * b.dx2 +
                                (mid[c - kHX] - 2.0 * uc + mid[c + kHX]) * b.dy2) +
                               (lo[c] - 2.0 * uc + hi[c]) * b.dz2) + a.lambda * uc;
            const double fv = fring[(q + 1) & (kRing - 1)][tid];
            const double bv = (side || k == b.zs || k == b.ze) ? bc_terms(fv, b, i, j, k) : fv;
            const double rv = (bv - au) - shift;
            a.r[k * a.rz + j * a.ry + i] = (float)rv;
            r2 += rv * rv;
            b2 += bv * bv;
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (a.sums) {
        // block reduction, then one atomic per block
        __shared__ double s0[32], s1[32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            r2 += __shfl_down_sync(0xffffffffu, r2, off);
            b2 += __shfl_down_sync(0xffffffffu, b2, off);
        }
        const int t = threadIdx.y * kResX + threadIdx.x;
        const int lane = t & 31, wid = t >> 5;
        if (lane == 0) {
            s0[wid] = r2;
            s1[wid] = b2;
        }
        __syncthreads();
        if (wid == 0) {
            constexpr int nw = kResX * kResY / 32;
            r2 = lane < nw ? s0[lane] : 0.0;
            b2 = lane < nw ? s1[lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                r2 += __shfl_down_sync(0xffffffffu, r2, off);
                b2 += __shfl_down_sync(0xffffffffu, b2, off);
            }
            if (lane == 0) {
                atomicAdd(a.sums, r2);
                atomicAdd(a.sums + 1, b2);
            }
        }
    }
}

// Copies the solution window of u into f (when refinement stops early).
__global__ void copy_window(double* f, const double* u, int nx, int ny, int xs, int xe, int ys, int zs) {
    const int i = xs + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = ys + blockIdx.y;
    const int k = zs + blockIdx.z;
    if (i > xe) return;
    const long long o = (long long)k * (nx + 1) * (ny + 1) + (long long)j * (nx + 1) + i;
    f[o] = u[o];
}

// One FP32 diagonal solve: x forward (from `in`: f with boundary terms, or
// the FP32 residual in the work array), y forward, z forward + divide + z
// inverse, y inverse, x inverse into `out` (FP64; out = acc + c when acc).
int solve32_passes(const AxisSolve& X, const AxisSolve& Y, const AxisSolve& Z, const DeviceLineTables& tx,
                   const DeviceLineTables& ty, const DeviceLineTables& tz, const double* ex, const double* ey,
                   const double* ez, double lambda, const BcArgs* bc, const double* f_in, float* w,
                   double* out, const double* acc, cudaStream_t s) {
    int rc;
    const int nx = X.n, ny = Y.n, nz = Z.n;
    const long long fy = nx + 1, fz = (long long)(nx + 1) * (ny + 1);
    const long long wy = pitch32(nx), wz = wy * (ny + 2);
    {
        const LineGeom g = line_geometry(nx, 0, true);
        PassArgs a{};
        a.kind = X.kf; a.kind2 = -1;
        a.u0 = Y.s; a.nu = Y.e - Y.s + 1; a.v0 = Z.s;
        if (f_in) {
            a.in_su = fy; a.in_sv = fz;
        } else {
            a.in_su = wy; a.in_sv = wz;
        }
        a.in_sl = 1;
        a.ld_lo = X.s; a.ld_hi = X.e;
        a.out_su = wy; a.out_sv = wz; a.out_sl = 1;
        a.st_lo = X.sp0; a.st_hi = X.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        if (bc) { a.has_bc = 1; a.bc = *bc; }
        rc = f_in ? launch_line_pass(0, kIoF64, kIoF32, true, f_in, w, a, tx, g, Z.e - Z.s + 1, s, "refine_x_fwd")
                  : launch_line_pass(0, kIoF32, kIoF32, true, w, w, a, tx, g, Z.e - Z.s + 1, s, "refine_x_fwd");
        if (rc) return cuda_fail(rc, "refine pass 1");
    }
    {
        const LineGeom g = line_geometry(ny, 0, false);
        PassArgs a{};
        a.kind = Y.kf; a.kind2 = -1;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = Z.s;
        a.in_su = 1; a.in_sv = wz; a.in_sl = wy;
        a.ld_lo = Y.s; a.ld_hi = Y.e;
        a.out_su = 1; a.out_sv = wz; a.out_sl = wy;
        a.st_lo = Y.sp0; a.st_hi = Y.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(0, kIoF32, kIoF32, false, w, w, a, ty, g, Z.e - Z.s + 1, s, "refine_y_fwd");
        if (rc) return cuda_fail(rc, "refine pass 2");
    }
    {
        const LineGeom g = line_geometry(nz, 0, false);
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
        rc = launch_line_pass(0, kIoF32, kIoF32, false, w, w, a, tz, g, Y.sp1 - Y.sp0 + 1, s, "refine_z_fwd_div_inv");
        if (rc) return cuda_fail(rc, "refine pass 3");
    }
    {
        const LineGeom g = line_geometry(ny, 0, false);
        PassArgs a{};
        a.kind = Y.ki; a.kind2 = -1;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = Z.s;
        a.in_su = 1; a.in_sv = wz; a.in_sl = wy;
        a.ld_lo = Y.sp0; a.ld_hi = Y.sp1;
        a.out_su = 1; a.out_sv = wz; a.out_sl = wy;
        a.st_lo = Y.s; a.st_hi = Y.e;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(0, kIoF32, kIoF32, false, w, w, a, ty, g, Z.e - Z.s + 1, s, "refine_y_inv");
        if (rc) return cuda_fail(rc, "refine pass 4");
    }
    {
        const LineGeom g = line_geometry(nx, 0, true);
        PassArgs a{};
        a.kind = X.ki; a.kind2 = -1;
        a.u0 = Y.s; a.nu = Y.e - Y.s + 1; a.v0 = Z.s;
        a.in_su = wy; a.in_sv = wz; a.in_sl = 1;
        a.ld_lo = X.sp0; a.ld_hi = X.sp1;
        a.out_su = fy; a.out_sv = fz; a.out_sl = 1;
        a.st_lo = X.s; a.st_hi = X.e;
        a.scale = solver_scale(X, Y, Z); a.use_scale = 1;
        a.acc = acc;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(0, kIoF32, kIoF64, true, w, out, a, tx, g, Z.e - Z.s + 1, s, "refine_x_inv");
        if (rc) return cuda_fail(rc, "refine pass 5");
    }
    return CHZ_SUCCESS;
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace
}  // namespace chz

using namespace chz;

extern "C" int chz_helmholtz_solve_refined(double left, double right, int nx, int xbc, const double* bcl,
                                           const double* bcr, double bottom, double top, int ny, int ybc,
                                           const double* bcb, const double* bct, double front, double back,
                                           int nz, int zbc, const double* bcf, const double* bce, double lambda,
                                           double* f, int max_corrections, double tol, int* corrections_done,
                                           double* rel_residual, void* workspace, size_t workspace_bytes,
                                           void* stream) {
    g_last_error[0] = 0;
    int rc;
    AxisSolve X, Y, Z;
    if ((rc = setup_axis(nx, xbc, left, right, &X)) || (rc = setup_axis(ny, ybc, bottom, top, &Y)) ||
        (rc = setup_axis(nz, zbc, front, back, &Z)))
        return rc;
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    if (!f) return fail(CHZ_ERROR_INVALID_VALUE, "f is NULL");
    if (max_corrections < 0 || max_corrections > 64)
        return fail(CHZ_ERROR_INVALID_VALUE, "max_corrections must be in 0..64");
    if ((rc = check_faces(X, bcl, bcr, "x")) || (rc = check_faces(Y, bcb, bct, "y")) ||
        (rc = check_faces(Z, bcf, bce, "z")))
        return rc;
    const size_t need = chz_helmholtz_workspace_size(nx, ny, nz, 1);
    if (workspace) {
        if (workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255))
            return fail(CHZ_ERROR_WORKSPACE, "workspace needs %zu bytes, 256-byte aligned", need);
    } else {
        if ((rc = cached_workspace(stream, need, &workspace))) return rc;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(workspace);
    float* w = reinterpret_cast<float*>(base);
    const size_t wbytes = round256((size_t)pitch32(nx) * (ny + 2) * (nz + 2) * sizeof(float));
    double* u = reinterpret_cast<double*>(base + wbytes);
    const size_t ubytes = round256((size_t)(nx + 1) * (ny + 1) * (nz + 1) * sizeof(double));
    double* sums = reinterpret_cast<double*>(base + wbytes + ubytes);  // [0..1] norms, [2] b's mode, [3] u's

    DeviceLineTables tx, ty, tz;
    if ((rc = tables_for(nx, 0, &tx)) || (rc = tables_for(ny, 0, &ty)) || (rc = tables_for(nz, 0, &tz))) return rc;
    const double *ex, *ey, *ez;
    if ((rc = eig_table(X, &ex)) || (rc = eig_table(Y, &ey)) || (rc = eig_table(Z, &ez))) return rc;

    BcArgs bc{};
    bc.xbc = X.bc; bc.ybc = Y.bc; bc.zbc = Z.bc;
    bc.xs = X.s; bc.xe = X.e; bc.ys = Y.s; bc.ye = Y.e; bc.zs = Z.s; bc.ze = Z.e;
    bc.nx = nx; bc.ny = ny; bc.nz = nz;
    bc.dx = X.d; bc.dy = Y.d; bc.dz = Z.d;
    bc.dx2 = X.d2; bc.dy2 = Y.d2; bc.dz2 = Z.d2;
    bc.f = f;
    bc.bcl = bcl; bc.bcr = bcr; bc.bcb = bcb; bc.bct = bct; bc.bcf = bcf; bc.bce = bce;

    const bool track = tol > 0.0 || rel_residual != nullptr;
    const bool singular = lambda == 0.0 && (X.bc == 0 || X.bc == 3) && (Y.bc == 0 || Y.bc == 3) &&
                          (Z.bc == 0 || Z.bc == 3);
    const double inv_w = 1.0 / ((double)nx * (double)ny * (double)nz);  // 1^T W 1 over the window
    int done = 0;
    double last_rel = -1.0;
    // initial FP32 solve: into f directly when there is nothing to refine
    if (max_corrections == 0) {
        if ((rc = solve32_passes(X, Y, Z, tx, ty, tz, ex, ey, ez, lambda, &bc, f, w, f, nullptr, s))) return rc;
    } else {
        if ((rc = solve32_passes(X, Y, Z, tx, ty, tz, ex, ey, ez, lambda, &bc, f, w, u, nullptr, s))) return rc;
        const dim3 rblock(128, 1, 1);
        const dim3 rgrid((X.e - X.s + 1 + 127) / 128, Y.e - Y.s + 1, Z.e - Z.s + 1);
        const dim3 resblock(kResX, kResY, 1);  // planes per block: kResZ
        const dim3 resgrid((X.e - X.s + kResX) / kResX, (Y.e - Y.s + kResY) / kResY, (Z.e - Z.s + kResZ) / kResZ);
        if (singular) {
            cudaError_t e = cudaMemsetAsync(sums + 2, 0, 2 * sizeof(double), s);
            if (e != cudaSuccess) return cuda_fail((int)e, "memset");
            mode_sum<<<rgrid, rblock, 0, s>>>(bc, nullptr, sums + 2);
            count_launch();
        }
        double prev = -1.0;
        bool copied = false;
        for (int it = 0; it < max_corrections; ++it) {
            ResidualArgs ra;
            ra.bc = bc;
            ra.u = u;
            ra.r = w;
            ra.ry = pitch32(nx);
            ra.rz = pitch32(nx) * (ny + 2);
            ra.lambda = lambda;
            ra.sums = track ? sums : nullptr;
            ra.shift = singular ? sums + 2 : nullptr;
            ra.inv_w = inv_w;
            if (track) {
                cudaError_t e = cudaMemsetAsync(sums, 0, 2 * sizeof(double), s);
                if (e != cudaSuccess) return cuda_fail((int)e, "memset");
            }
            trace_begin(s, "refine_residual");
            residual_kernel<<<resgrid, resblock, 0, s>>>(ra);
            count_launch();
            trace_end(s);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail((int)e, "residual");
            if (track) {
                double h[2];
                e = cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) return cuda_fail((int)e, "residual norm");
                const double rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
                last_rel = rel;
                // stop: residual small enough, or no longer decreasing
                if ((tol > 0.0 && rel <= tol) || (prev >= 0.0 && rel > 0.5 * prev)) {
                    const dim3 cgrid = rgrid;
                    copy_window<<<cgrid, rblock, 0, s>>>(f, u, nx, ny, X.s, X.e, Y.s, Z.s);
                    count_launch();
                    copied = true;
                    break;
                }
                prev = rel;
            }
            const bool last = (it == max_corrections - 1);
            if ((rc = solve32_passes(X, Y, Z, tx, ty, tz, ex, ey, ez, lambda, nullptr, nullptr, w, last ? f : u, u, s)))
                return rc;
            ++done;
        }
        (void)copied;
        if (singular) {
            mode_sum<<<rgrid, rblock, 0, s>>>(bc, f, sums + 3);
            remove_mode<<<rgrid, rblock, 0, s>>>(f, bc, sums + 3, inv_w);
            count_launch();
            count_launch();
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail((int)e, "constant mode");
        }
    }
    rc = launch_periodic_fixup(f, nx, ny, nz, X.bc, Y.bc, Z.bc, s);
    if (rc) return cuda_fail(rc, "periodic planes");
    if (corrections_done) *corrections_done = done;
    if (rel_residual) *rel_residual = last_rel;
    return CHZ_SUCCESS;
}

// Solve with FISHPACK's PERTRB (the constant hw3crt subtracts from the
// right-hand side of a singular problem so that a solution exists).  The
// diagonal solve already removes the constant mode, which solves the system
// with b - PERTRB, so the solution is the plain solve's; PERTRB itself is the
// weighted mean 1^T W b / 1^T W 1 over the unknown window (mode_sum), read
// back before the solve overwrites f.
extern "C" int chz_helmholtz_solve_pertrb(double left, double right, int nx, int xbc, const double* bcl,
                                          const double* bcr, double bottom, double top, int ny, int ybc,
                                          const double* bcb, const double* bct, double front, double back, int nz,
                                          int zbc, const double* bcf, const double* bce, double lambda, double* f,
                                          double* pertrb, void* stream) {
    g_last_error[0] = 0;
    if (!pertrb) return fail(CHZ_ERROR_INVALID_VALUE, "pertrb is NULL");
    *pertrb = 0.0;
    int rc;
    AxisSolve X, Y, Z;
    if ((rc = setup_axis(nx, xbc, left, right, &X)) || (rc = setup_axis(ny, ybc, bottom, top, &Y)) ||
        (rc = setup_axis(nz, zbc, front, back, &Z)))
        return rc;
    const bool singular = lambda == 0.0 && (X.bc == 0 || X.bc == 3) && (Y.bc == 0 || Y.bc == 3) &&
                          (Z.bc == 0 || Z.bc == 3);
    if (!singular)
        return chz_helmholtz_solve(left, right, nx, xbc, bcl, bcr, bottom, top, ny, ybc, bcb, bct, front, back, nz,
                                   zbc, bcf, bce, lambda, f, stream);
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    if (!f) return fail(CHZ_ERROR_INVALID_VALUE, "f is NULL");
    if ((rc = check_faces(X, bcl, bcr, "x")) || (rc = check_faces(Y, bcb, bct, "y")) ||
        (rc = check_faces(Z, bcf, bce, "z")))
        return rc;
    const size_t need = chz_helmholtz_workspace_size(nx, ny, nz, 0);
    void* ws = nullptr;
    if ((rc = cached_workspace(stream, need + 256, &ws))) return rc;
    double* acc = reinterpret_cast<double*>(static_cast<char*>(ws) + need);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    BcArgs bc{};
    bc.xbc = X.bc; bc.ybc = Y.bc; bc.zbc = Z.bc;
    bc.xs = X.s; bc.xe = X.e; bc.ys = Y.s; bc.ye = Y.e; bc.zs = Z.s; bc.ze = Z.e;
    bc.nx = nx; bc.ny = ny; bc.nz = nz;
    bc.dx = X.d; bc.dy = Y.d; bc.dz = Z.d;
    bc.dx2 = X.d2; bc.dy2 = Y.d2; bc.dz2 = Z.d2;
    bc.f = f;
    bc.bcl = bcl; bc.bcr = bcr; bc.bcb = bcb; bc.bct = bct; bc.bcf = bcf; bc.bce = bce;
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(double), s);
    if (e != cudaSuccess) return cuda_fail((int)e, "memset");
    const dim3 block(128, 1, 1);
    const dim3 grid((X.e - X.s + 1 + 127) / 128, Y.e - Y.s + 1, Z.e - Z.s + 1);
    mode_sum<<<grid, block, 0, s>>>(bc, nullptr, acc);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail((int)e, "weighted mean");
    double h = 0.0;
    e = cudaMemcpyAsync(&h, acc, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail((int)e, "weighted mean read-back");
    *pertrb = h / ((double)nx * (double)ny * (double)nz);  // 1^T W 1 over the window
    return chz_helmholtz_solve_ws(left, right, nx, xbc, bcl, bcr, bottom, top, ny, ybc, bcb, bct, front, back, nz,
                                  zbc, bcf, bce, lambda, f, ws, need, stream);
}
