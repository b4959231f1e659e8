// Slab-decomposed Helmholtz solve: the per-rank steps of one solve split over
// several GPUs by z planes (no counterpart in the reference, whose solver runs
// on one GPU).  The reference's non-cubic path already transforms x, then y,
// then z with a transpose between the axes (cudasymmfft/funcinterface.cu:
// 200-334); split over z, the x and y passes stay local to a rank's planes and
// the transpose before and after the z pass becomes an all-to-all between
// ranks.  These entry points are the local steps; the exchange is the
// caller's (cuhelmholtz_b200.slab over torch.distributed / NCCL).
//
//   chz_slab_forward : x and y forward passes (boundary terms applied) of the
//                      slab's planes inside the z unknown window, f -> work slab
//   chz_slab_z       : the fused z pass (forward, eigenvalue division, inverse)
//                      on a pencil holding a block of y rows for every plane of
//                      the z unknown window
//   chz_slab_inverse : y and x inverse passes, work slab -> f, scaled, and the
//                      x and y periodic copies of the slab's planes
//
// Index arithmetic stays global: the kernels receive base pointers moved back
// by the slab's (or pencil's) first plane, so plane k of the slab is plane k
// of the whole problem; only planes inside the slab are ever addressed.
#include <cuda_runtime.h>

#include <cstdint>

#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace {

struct SlabProblem {
    AxisSolve X, Y, Z;
    DeviceLineTables tx, ty, tz;
    const double *ex = nullptr, *ey = nullptr, *ez = nullptr;
};

int slab_setup(double left, double right, int nx, int xbc, const double* bcl, const double* bcr, double bottom,
               double top, int ny, int ybc, const double* bcb, const double* bct, double front, double back,
               int nz, int zbc, const double* bcf, const double* bce, bool need_faces, bool need_eig,
               SlabProblem* P) {
    g_last_error[0] = 0;
    int rc;
    if ((rc = setup_axis(nx, xbc, left, right, &P->X)) || (rc = setup_axis(ny, ybc, bottom, top, &P->Y)) ||
        (rc = setup_axis(nz, zbc, front, back, &P->Z)))
        return rc;
    if ((rc = check_len(nx, "x")) || (rc = check_len(ny, "y")) || (rc = check_len(nz, "z"))) return rc;
    if (need_faces && ((rc = check_faces(P->X, bcl, bcr, "x")) || (rc = check_faces(P->Y, bcb, bct, "y")) ||
                       (rc = check_faces(P->Z, bcf, bce, "z"))))
        return rc;
    if ((rc = tables_for(nx, 1, &P->tx)) || (rc = tables_for(ny, 1, &P->ty)) || (rc = tables_for(nz, 1, &P->tz)))
        return rc;
    if (need_eig && ((rc = eig_table(P->X, &P->ex)) || (rc = eig_table(P->Y, &P->ey)) ||
                     (rc = eig_table(P->Z, &P->ez))))
        return rc;
    return CHZ_SUCCESS;
}

// Planes [k0, k1] of the z unknown window inside slab [z0, z0 + nzl); k1 < k0
// when there are none.  The boundary terms of a Dirichlet z face read f on
// plane 0 (or nz): the slab holding the first (last) unknown plane must hold
// that plane as well.
int slab_planes(const SlabProblem& P, int z0, int nzl, int* k0, int* k1) {
    const int nz = P.Z.n;
    if (z0 < 0 || nzl < 1 || z0 + nzl > nz + 1)
        return fail(CHZ_ERROR_INVALID_VALUE, "slab planes [%d, %d) outside 0..%d", z0, z0 + nzl, nz);
    *k0 = z0 > P.Z.s ? z0 : P.Z.s;
    *k1 = z0 + nzl - 1 < P.Z.e ? z0 + nzl - 1 : P.Z.e;
    const bool dir_lo = P.Z.bc == 1 || P.Z.bc == 2, dir_hi = P.Z.bc == 1 || P.Z.bc == 4;
    if (dir_lo && *k0 <= P.Z.s && P.Z.s <= *k1 && z0 > 0)
        return fail(CHZ_ERROR_INVALID_VALUE, "the slab holding plane %d must hold plane 0 (Dirichlet z face)",
                    P.Z.s);
    if (dir_hi && *k0 <= P.Z.e && P.Z.e <= *k1 && z0 + nzl - 1 < nz)
        return fail(CHZ_ERROR_INVALID_VALUE, "the slab holding plane %d must hold plane %d (Dirichlet z face)",
                    P.Z.e, nz);
    return CHZ_SUCCESS;
}

}  // namespace
}  // namespace chz

using namespace chz;

extern "C" int chz_slab_forward(double left, double right, int nx, int xbc, const double* bcl, const double* bcr,
                                double bottom, double top, int ny, int ybc, const double* bcb, const double* bct,
                                double front, double back, int nz, int zbc, const double* bcf, const double* bce,
                                const double* f_slab, int z0, int nzl, double* ws_slab, void* stream) {
    SlabProblem P;
    int rc = slab_setup(left, right, nx, xbc, bcl, bcr, bottom, top, ny, ybc, bcb, bct, front, back, nz, zbc, bcf,
                        bce, true, false, &P);
    if (rc) return rc;
    if (!f_slab || !ws_slab) return fail(CHZ_ERROR_INVALID_VALUE, "f_slab / ws_slab is NULL");
    if (reinterpret_cast<uintptr_t>(ws_slab) & 255) return fail(CHZ_ERROR_WORKSPACE, "ws_slab must be 256-byte aligned");
    int k0, k1;
    if ((rc = slab_planes(P, z0, nzl, &k0, &k1))) return rc;
    if (k1 < k0) return CHZ_SUCCESS;
    const AxisSolve &X = P.X, &Y = P.Y, &Z = P.Z;
    const long long fy = nx + 1, fz = (long long)(nx + 1) * (ny + 1);
    const long long wy = nx + 2, wz = (long long)(nx + 2) * (ny + 2);
    const double* fv = f_slab - (long long)z0 * fz;   // plane k of the problem at fv + k * fz
    double* wv = ws_slab - (long long)z0 * wz;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    BcArgs bc{};
    bc.xbc = X.bc; bc.ybc = Y.bc; bc.zbc = Z.bc;
    bc.xs = X.s; bc.xe = X.e; bc.ys = Y.s; bc.ye = Y.e; bc.zs = Z.s; bc.ze = Z.e;
    bc.nx = nx; bc.ny = ny; bc.nz = nz;
    bc.dx = X.d; bc.dy = Y.d; bc.dz = Z.d;
    bc.dx2 = X.d2; bc.dy2 = Y.d2; bc.dz2 = Z.d2;
    bc.f = fv;
    bc.bcl = bcl; bc.bcr = bcr; bc.bcb = bcb; bc.bct = bct; bc.bcf = bcf; bc.bce = bce;
    {
        const LineGeom g = line_geometry(nx, 1, true);
        PassArgs a{};
        a.kind = X.kf; a.kind2 = -1;
        a.u0 = Y.s; a.nu = Y.e - Y.s + 1; a.v0 = k0;
        a.in_su = fy; a.in_sv = fz; a.in_sl = 1;
        a.ld_lo = X.s; a.ld_hi = X.e;
        a.out_su = wy; a.out_sv = wz; a.out_sl = 1;
        a.st_lo = X.sp0; a.st_hi = X.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        a.has_bc = 1; a.bc = bc;
        rc = launch_line_pass(1, kIoF64, kIoF64, true, fv, wv, a, P.tx, g, k1 - k0 + 1, s, "slab_x_fwd");
        if (rc) return cuda_fail(rc, "slab x forward");
    }
    {
        const LineGeom g = line_geometry(ny, 1, false);
        PassArgs a{};
        a.kind = Y.kf; a.kind2 = -1;
        a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = k0;
        a.in_su = 1; a.in_sv = wz; a.in_sl = wy;
        a.ld_lo = Y.s; a.ld_hi = Y.e;
        a.out_su = 1; a.out_sv = wz; a.out_sl = wy;
        a.st_lo = Y.sp0; a.st_hi = Y.sp1;
        a.scale = 1.0; a.use_scale = 0;
        a.PR = g.PR; a.log2W = g.log2W;
        rc = launch_line_pass(1, kIoF64, kIoF64, false, wv, wv, a, P.ty, g, k1 - k0 + 1, s, "slab_y_fwd");
        if (rc) return cuda_fail(rc, "slab y forward");
    }
    return CHZ_SUCCESS;
}

extern "C" int chz_slab_z(double left, double right, int nx, int xbc, double bottom, double top, int ny, int ybc,
                          double front, double back, int nz, int zbc, double lambda, double* pencil, int j0, int nj,
                          void* stream) {
    SlabProblem P;
    int rc = slab_setup(left, right, nx, xbc, nullptr, nullptr, bottom, top, ny, ybc, nullptr, nullptr, front, back,
                        nz, zbc, nullptr, nullptr, false, true, &P);
    if (rc) return rc;
    const AxisSolve &X = P.X, &Y = P.Y, &Z = P.Z;
    if (!pencil) return fail(CHZ_ERROR_INVALID_VALUE, "pencil is NULL");
    if (reinterpret_cast<uintptr_t>(pencil) & 255) return fail(CHZ_ERROR_WORKSPACE, "pencil must be 256-byte aligned");
    if (nj < 1 || j0 < Y.sp0 || j0 + nj - 1 > Y.sp1)
        return fail(CHZ_ERROR_INVALID_VALUE, "pencil rows [%d, %d) outside the spectral y window %d..%d", j0,
                    j0 + nj, Y.sp0, Y.sp1);
    const long long wy = nx + 2, wp = (long long)(nx + 2) * nj;   // row and plane strides of the pencil
    double* pv = pencil - (long long)Z.s * wp - 0;                   // plane k at pv + k * wp
    const LineGeom g = line_geometry(nz, 1, false);
    PassArgs a{};
    a.kind = Z.kf; a.kind2 = Z.ki;
    a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = 0;
    a.in_su = 1; a.in_sv = wy; a.in_sl = wp;
    a.ld_lo = Z.s; a.ld_hi = Z.e;
    a.out_su = 1; a.out_sv = wy; a.out_sl = wp;
    a.st_lo = Z.s; a.st_hi = Z.e;
    a.scale = 1.0; a.use_scale = 0;
    a.PR = g.PR; a.log2W = g.log2W;
    a.has_div = 1;
    a.dv.ex = P.ex; a.dv.ey = P.ey + j0; a.dv.ez = P.ez;   // pencil row v is problem row j0 + v
    a.dv.lambda = lambda;
    a.dv.perturb = (lambda == 0.0 && (X.bc == 0 || X.bc == 3) && (Y.bc == 0 || Y.bc == 3) &&
                    (Z.bc == 0 || Z.bc == 3));
    a.dv.xz_hi = X.bc == 0 ? 1 : 0;
    a.dv.yz_hi = (Y.bc == 0 ? 1 : 0) - j0;
    a.dv.zz_hi = Z.bc == 0 ? 1 : 0;
    a.dv.lo = Z.sp0; a.dv.hi = Z.sp1;
    rc = launch_line_pass(1, kIoF64, kIoF64, false, pv, pv, a, P.tz, g, nj, static_cast<cudaStream_t>(stream),
                          "slab_z_fwd_div_inv");
    if (rc) return cuda_fail(rc, "slab z pass");
    return CHZ_SUCCESS;
}

extern "C" int chz_slab_inverse(double left, double right, int nx, int xbc, double bottom, double top, int ny,
                                int ybc, double front, double back, int nz, int zbc, double* ws_slab,
                                double* f_slab, int z0, int nzl, void* stream) {
    SlabProblem P;
    int rc = slab_setup(left, right, nx, xbc, nullptr, nullptr, bottom, top, ny, ybc, nullptr, nullptr, front, back,
                        nz, zbc, nullptr, nullptr, false, false, &P);
    if (rc) return rc;
    if (!f_slab || !ws_slab) return fail(CHZ_ERROR_INVALID_VALUE, "f_slab / ws_slab is NULL");
    if (reinterpret_cast<uintptr_t>(ws_slab) & 255) return fail(CHZ_ERROR_WORKSPACE, "ws_slab must be 256-byte aligned");
    const AxisSolve &X = P.X, &Y = P.Y, &Z = P.Z;
    if (z0 < 0 || nzl < 1 || z0 + nzl > nz + 1)
        return fail(CHZ_ERROR_INVALID_VALUE, "slab planes [%d, %d) outside 0..%d", z0, z0 + nzl, nz);
    const int k0 = z0 > Z.s ? z0 : Z.s;
    const int k1 = z0 + nzl - 1 < Z.e ? z0 + nzl - 1 : Z.e;
    const long long fy = nx + 1, fz = (long long)(nx + 1) * (ny + 1);
    const long long wy = nx + 2, wz = (long long)(nx + 2) * (ny + 2);
    double* fv = f_slab - (long long)z0 * fz;
    double* wv = ws_slab - (long long)z0 * wz;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k0 <= k1) {
        {
            const LineGeom g = line_geometry(ny, 1, false);
            PassArgs a{};
            a.kind = Y.ki; a.kind2 = -1;
            a.u0 = X.sp0; a.nu = X.sp1 - X.sp0 + 1; a.v0 = k0;
            a.in_su = 1; a.in_sv = wz; a.in_sl = wy;
            a.ld_lo = Y.sp0; a.ld_hi = Y.sp1;
            a.out_su = 1; a.out_sv = wz; a.out_sl = wy;
            a.st_lo = Y.s; a.st_hi = Y.e;
            a.scale = 1.0; a.use_scale = 0;
            a.PR = g.PR; a.log2W = g.log2W;
            rc = launch_line_pass(1, kIoF64, kIoF64, false, wv, wv, a, P.ty, g, k1 - k0 + 1, s, "slab_y_inv");
            if (rc) return cuda_fail(rc, "slab y inverse");
        }
        {
            const LineGeom g = line_geometry(nx, 1, true);
            PassArgs a{};
            a.kind = X.ki; a.kind2 = -1;
            a.u0 = Y.s; a.nu = Y.e - Y.s + 1; a.v0 = k0;
            a.in_su = wy; a.in_sv = wz; a.in_sl = 1;
            a.ld_lo = X.sp0; a.ld_hi = X.sp1;
            a.out_su = fy; a.out_sv = fz; a.out_sl = 1;
            a.st_lo = X.s; a.st_hi = X.e;
            a.scale = solver_scale(X, Y, Z); a.use_scale = 1;
            a.PR = g.PR; a.log2W = g.log2W;
            rc = launch_line_pass(1, kIoF64, kIoF64, true, wv, fv, a, P.tx, g, k1 - k0 + 1, s, "slab_x_inv");
            if (rc) return cuda_fail(rc, "slab x inverse");
        }
    }
    // x and y periodic copies of every plane of the slab (the z copy crosses slabs)
    rc = launch_periodic_fixup(f_slab, nx, ny, nzl - 1, X.bc, Y.bc, 1, s);
    if (rc) return cuda_fail(rc, "slab periodic planes");
    return CHZ_SUCCESS;
}

extern "C" size_t chz_slab_work_elems(int nx, int ny, int nzl) {
    if (nx < 1 || ny < 1 || nzl < 1) return 0;
    return (size_t)(nx + 2) * (ny + 2) * nzl;
}
