// FP32 transforms with FP64 iterative refinement: chz_helmholtz_solve_refined.
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
__global__ void residual_kernel(ResidualArgs a) {
    const BcArgs& b = a.bc;
    const int i = b.xs + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = b.ys + blockIdx.y;
    const int k = b.zs + blockIdx.z;
    double r2 = 0.0, b2 = 0.0;
    if (i <= b.xe) {
        const long long sy = b.nx + 1, sz = (long long)(b.nx + 1) * (b.ny + 1);
        const long long o = k * sz + j * sy + i;
        const double* u = a.u;
        const double uc = u[o];
        // x neighbours
        double ul, ur;
        if (i == b.xs) {
            ul = (b.xbc == 0) ? u[o - i + (b.nx - 1)] : (b.xbc >= 3 ? u[o + 1] : 0.0);
        } else {
            ul = u[o - 1];
        }
        if (i == b.xe) {
            ur = (b.xbc == 0) ? u[o - i] : ((b.xbc == 2 || b.xbc == 3) ? u[o - 1] : 0.0);
        } else {
            ur = u[o + 1];
        }
        double dl, dr;
        if (j == b.ys) {
            dl = (b.ybc == 0) ? u[o + (b.ny - 1 - j) * sy] : (b.ybc >= 3 ? u[o + sy] : 0.0);
        } else {
            dl = u[o - sy];
        }
        if (j == b.ye) {
            dr = (b.ybc == 0) ? u[o - j * sy] : ((b.ybc == 2 || b.ybc == 3) ? u[o - sy] : 0.0);
        } else {
            dr = u[o + sy];
        }
        double fl, fr;
        if (k == b.zs) {
            fl = (b.zbc == 0) ? u[o + (long long)(b.nz - 1 - k) * sz] : (b.zbc >= 3 ? u[o + sz] : 0.0);
        } else {
            fl = u[o - sz];
        }
        if (k == b.ze) {
            fr = (b.zbc == 0) ? u[o - (long long)k * sz] : ((b.zbc == 2 || b.zbc == 3) ? u[o - sz] : 0.0);
        } else {
            fr = u[o + sz];
        }
        const double au = (((ul - 2.0 * uc + ur) * b.dx2 + (dl - 2.0 * uc + dr) * b.dy2) +
                           (fl - 2.0 * uc + fr) * b.dz2) + a.lambda * uc;
        const double bv = bc_terms(__ldg(b.f + o), b, i, j, k);
        const double rv = a.shift ? (bv - au) - *a.shift * a.inv_w : bv - au;
        a.r[k * a.rz + j * a.ry + i] = (float)rv;
        r2 = rv * rv;
        b2 = bv * bv;
    }
    if (a.sums) {
        // block reduction, then one atomic per block
        __shared__ double s0[32], s1[32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            r2 += __shfl_down_sync(0xffffffffu, r2, off);
            b2 += __shfl_down_sync(0xffffffffu, b2, off);
        }
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) {
            s0[wid] = r2;
            s1[wid] = b2;
        }
        __syncthreads();
        if (wid == 0) {
            const int nw = blockDim.x >> 5;
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
            residual_kernel<<<rgrid, rblock, 0, s>>>(ra);
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
