// Adjoint of the Helmholtz solve map (chz_helmholtz_adjoint).
//
// The forward map is the whole in-place API map of cuda_helmholtz_solver
// (cuda_helmholtz_solver.cu:33-380):
//   u_W = A^-1 b,  b = f_W + boundary terms (linear in f's Dirichlet faces and
//   the Neumann arrays, _cuda_helmholtz_.inl:70-227); u = f elsewhere, except
//   periodic planes N, which copy plane 0 (x, then y, then z).
// A is not symmetric (the Neumann ghost closure 2u[1]-2u[0]), but W A is, with
// W = diag(1/2 at Neumann boundary nodes, 1 elsewhere) per axis, so
// A^-T = W A^-1 W^-1: the adjoint solve is the forward solve (same transform
// kinds) between two diagonal scalings.  Given g = dL/du:
//   G   = g with the periodic copies reversed (g[N plane] added to plane 0)
//   w   = W A^-1 (W^-1 G_W)                        (one homogeneous solve)
//   dL/df      = w on the window; G on other nodes (0 on periodic N planes),
//                plus -h^-2 w at the Dirichlet faces the boundary terms read
//   dL/dbc*    = +-2 h^-1 w at the window's boundary nodes (Neumann arrays)
//   dL/dlambda = -<w, u_W>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace {

struct Grid {
    int nx, ny, nz;
    long long sy, sz;  // (nx+1), (nx+1)(ny+1)
};

__device__ __forceinline__ double neu_w(int i, int n, int bc) {
    // 1/2 at Neumann boundary nodes of the unknown window
    if ((bc == 3 || bc == 4) && i == 0) return 0.5;
    if ((bc == 2 || bc == 3) && i == n) return 0.5;
    return 1.0;
}

// G: reverse the periodic copies, in the reverse of their order (z, y, x).
// One pass per axis; the source plane never lies on that axis' N plane.
__global__ void reverse_periodic(double* G, Grid g, int axis) {
    const long long n1 = axis == 0 ? (long long)(g.ny + 1) * (g.nz + 1)
                       : axis == 1 ? (long long)(g.nx + 1) * (g.nz + 1)
                                   : (long long)(g.nx + 1) * (g.ny + 1);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n1;
         e += (long long)gridDim.x * blockDim.x) {
        long long src, dst;
        if (axis == 0) {
            const int k = (int)(e / (g.ny + 1)), j = (int)(e % (g.ny + 1));
            dst = k * g.sz + j * g.sy + g.nx;
            src = k * g.sz + j * g.sy;
        } else if (axis == 1) {
            const int k = (int)(e / (g.nx + 1)), i = (int)(e % (g.nx + 1));
            dst = k * g.sz + (long long)g.ny * g.sy + i;
            src = k * g.sz + i;
        } else {
            const int j = (int)(e / (g.nx + 1)), i = (int)(e % (g.nx + 1));
            dst = (long long)g.nz * g.sz + j * g.sy + i;
            src = j * g.sy + i;
        }
        G[src] += G[dst];
        G[dst] = 0.0;
    }
}

struct AdjArgs {
    Grid g;
    int xbc, ybc, zbc;
    int xs, xe, ys, ye, zs, ze;
    double dx, dy, dz, dx2, dy2, dz2;
};

// R = W^-1 G on the window, 0 elsewhere (the right-hand side of the
// homogeneous solve).
__global__ void scale_in(double* R, const double* G, AdjArgs a) {
    const long long total = a.g.sz * (a.g.nz + 1);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / a.g.sz);
        const long long r = e - k * a.g.sz;
        const int j = (int)(r / a.g.sy);
        const int i = (int)(r - j * a.g.sy);
        const bool in = i >= a.xs && i <= a.xe && j >= a.ys && j <= a.ye && k >= a.zs && k <= a.ze;
        double v = 0.0;
        if (in) {
            const double w = neu_w(i, a.g.nx, a.xbc) * neu_w(j, a.g.ny, a.ybc) * neu_w(k, a.g.nz, a.zbc);
            v = G[e] / w;
        }
        R[e] = v;
    }
}

// df, the Neumann-array gradients and -<w, u> from R = A^-1 W^-1 G.
__global__ void finish(double* df, const double* R, const double* u, AdjArgs a, double* bcl, double* bcr,
                       double* bcb, double* bct, double* bcf, double* bce, double* dlam) {
    const int i = a.xs + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = a.ys + blockIdx.y;
    const int k = a.zs + blockIdx.z;
    double acc = 0.0;
    if (i <= a.xe) {
        const long long o = k * a.g.sz + j * a.g.sy + i;
        const double w = R[o] * (neu_w(i, a.g.nx, a.xbc) * neu_w(j, a.g.ny, a.ybc) * neu_w(k, a.g.nz, a.zbc));
        df[o] = w;
        acc = -w * u[o];
        const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
        // x boundary terms
        if (i == a.xs) {
            if (a.xbc == 1 || a.xbc == 2) df[o - i] += -a.dx2 * w;
            if ((a.xbc == 3 || a.xbc == 4) && bcl) bcl[(long long)k * (ny + 1) + j] = 2.0 * a.dx * w;
        }
        if (i == a.xe) {
            if (a.xbc == 1 || a.xbc == 4) df[o - i + nx] += -a.dx2 * w;
            if ((a.xbc == 2 || a.xbc == 3) && bcr) bcr[(long long)k * (ny + 1) + j] = -2.0 * a.dx * w;
        }
        if (j == a.ys) {
            if (a.ybc == 1 || a.ybc == 2) df[o - j * a.g.sy] += -a.dy2 * w;
            if ((a.ybc == 3 || a.ybc == 4) && bcb) bcb[(long long)k * (nx + 1) + i] = 2.0 * a.dy * w;
        }
        if (j == a.ye) {
            if (a.ybc == 1 || a.ybc == 4) df[o + (long long)(ny - j) * a.g.sy] += -a.dy2 * w;
            if ((a.ybc == 2 || a.ybc == 3) && bct) bct[(long long)k * (nx + 1) + i] = -2.0 * a.dy * w;
        }
        if (k == a.zs) {
            if (a.zbc == 1 || a.zbc == 2) df[o - (long long)k * a.g.sz] += -a.dz2 * w;
            if ((a.zbc == 3 || a.zbc == 4) && bcf) bcf[(long long)j * (nx + 1) + i] = 2.0 * a.dz * w;
        }
        if (k == a.ze) {
            if (a.zbc == 1 || a.zbc == 4) df[o + (long long)(nz - k) * a.g.sz] += -a.dz2 * w;
            if ((a.zbc == 2 || a.zbc == 3) && bce) bce[(long long)j * (nx + 1) + i] = -2.0 * a.dz * w;
        }
    }
    if (dlam) {
        __shared__ double red[32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        if (lane == 0) red[wid] = acc;
        __syncthreads();
        if (wid == 0) {
            acc = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
            if (lane == 0) atomicAdd(dlam, acc);
        }
    }
}

}  // namespace
}  // namespace chz

using namespace chz;

extern "C" int chz_helmholtz_adjoint(double left, double right, int nx, int xbc, double bottom, double top, int ny,
                                     int ybc, double front, double back, int nz, int zbc, double lambda,
                                     const double* g, const double* u, double* df, double* dbcl, double* dbcr,
                                     double* dbcb, double* dbct, double* dbcf, double* dbce, double* dlambda,
                                     int precision, int corrections, void* workspace, size_t workspace_bytes,
                                     void* stream) {
    g_last_error[0] = 0;
    int rc;
    AxisSolve X, Y, Z;
    if ((rc = setup_axis(nx, xbc, left, right, &X)) || (rc = setup_axis(ny, ybc, bottom, top, &Y)) ||
        (rc = setup_axis(nz, zbc, front, back, &Z)))
        return rc;
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    if (!g || !u || !df) return fail(CHZ_ERROR_INVALID_VALUE, "g, u and df must be device arrays");
    if (precision != 0 && precision != 1) return fail(CHZ_ERROR_INVALID_VALUE, "precision must be 0 or 1");
    const size_t npts = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    const size_t fmax = std::max((size_t)(nx + 1) * (ny + 1), std::max((size_t)(nx + 1) * (nz + 1),
                                                                        (size_t)(ny + 1) * (nz + 1)));
    const size_t need = chz_helmholtz_adjoint_workspace_size(nx, ny, nz, precision);
    if (!workspace || workspace_bytes < need || (reinterpret_cast<uintptr_t>(workspace) & 255))
        return fail(CHZ_ERROR_WORKSPACE, "adjoint workspace needs %zu bytes, 256-byte aligned", need);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(workspace);
    auto r256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
    double* R = reinterpret_cast<double*>(base);
    double* zeros = reinterpret_cast<double*>(base + r256(npts * 8));
    double* dl = reinterpret_cast<double*>(base + r256(npts * 8) + r256(fmax * 8));
    void* solve_ws = base + r256(npts * 8) + r256(fmax * 8) + 256;
    const size_t solve_ws_bytes = workspace_bytes - (r256(npts * 8) + r256(fmax * 8) + 256);

    Grid gr{nx, ny, nz, nx + 1, (long long)(nx + 1) * (ny + 1)};
    AdjArgs a;
    a.g = gr;
    a.xbc = X.bc; a.ybc = Y.bc; a.zbc = Z.bc;
    a.xs = X.s; a.xe = X.e; a.ys = Y.s; a.ye = Y.e; a.zs = Z.s; a.ze = Z.e;
    a.dx = X.d; a.dy = Y.d; a.dz = Z.d; a.dx2 = X.d2; a.dy2 = Y.d2; a.dz2 = Z.d2;

    cudaError_t e = cudaMemcpyAsync(df, g, npts * 8, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(zeros, 0, fmax * 8, s);
    if (e == cudaSuccess && dlambda) e = cudaMemsetAsync(dl, 0, 8, s);
    if (e != cudaSuccess) return cuda_fail((int)e, "adjoint setup");
    const int ax_bc[3] = {Z.bc, Y.bc, X.bc};
    for (int q = 0; q < 3; ++q) {  // z, then y, then x
        if (ax_bc[q] != 0) continue;
        reverse_periodic<<<148 * 4, 256, 0, s>>>(df, gr, 2 - q);
        count_launch();
    }
    scale_in<<<148 * 8, 256, 0, s>>>(R, df, a);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail((int)e, "adjoint scaling");
    // homogeneous solve on R: zero Dirichlet faces (R is 0 off the window) and zero Neumann data
    const double* zf = zeros;
    if (precision == 0) {
        if (solve_ws_bytes < chz_helmholtz_workspace_size(nx, ny, nz, 0))
            return fail(CHZ_ERROR_WORKSPACE, "adjoint workspace too small for the solve");
        rc = chz_helmholtz_solve_ws(left, right, nx, xbc, zf, zf, bottom, top, ny, ybc, zf, zf, front, back, nz,
                                    zbc, zf, zf, lambda, R, solve_ws, solve_ws_bytes, stream);
    } else {
        rc = chz_helmholtz_solve_refined(left, right, nx, xbc, zf, zf, bottom, top, ny, ybc, zf, zf, front, back,
                                         nz, zbc, zf, zf, lambda, R, corrections, 0.0, nullptr, nullptr, solve_ws,
                                         solve_ws_bytes, stream);
    }
    if (rc != CHZ_SUCCESS) return rc;
    // Neumann-array gradients are 0 outside the window's boundary nodes
    const size_t fx = (size_t)(ny + 1) * (nz + 1), fy = (size_t)(nx + 1) * (nz + 1), fz = (size_t)(nx + 1) * (ny + 1);
    double* outs[6] = {dbcl, dbcr, dbcb, dbct, dbcf, dbce};
    const size_t lens[6] = {fx, fx, fy, fy, fz, fz};
    for (int q = 0; q < 6; ++q) {
        if (outs[q] && (e = cudaMemsetAsync(outs[q], 0, lens[q] * 8, s)) != cudaSuccess)
            return cuda_fail((int)e, "adjoint face gradients");
    }
    const dim3 blk(128, 1, 1);
    const dim3 grd((X.e - X.s + 1 + 127) / 128, Y.e - Y.s + 1, Z.e - Z.s + 1);
    finish<<<grd, blk, 0, s>>>(df, R, u, a, dbcl, dbcr, dbcb, dbct, dbcf, dbce, dlambda ? dl : nullptr);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail((int)e, "adjoint finish");
    if (dlambda) {
        e = cudaMemcpyAsync(dlambda, dl, 8, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_fail((int)e, "adjoint dlambda");
    }
    return CHZ_SUCCESS;
}

extern "C" size_t chz_helmholtz_adjoint_workspace_size(int nx, int ny, int nz, int precision) {
    if (nx < 1 || ny < 1 || nz < 1) return 0;
    auto r256 = [](size_t b) { return (b + 255) & ~(size_t)255; };
    const size_t npts = (size_t)(nx + 1) * (ny + 1) * (nz + 1);
    const size_t fmax = std::max((size_t)(nx + 1) * (ny + 1), std::max((size_t)(nx + 1) * (nz + 1),
                                                                        (size_t)(ny + 1) * (nz + 1)));
    return r256(npts * 8) + r256(fmax * 8) + 256 + chz_helmholtz_workspace_size(nx, ny, nz, precision);
}
