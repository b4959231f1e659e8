/* Drop-in replacement for the reference's cudahelmholtz/cuda_helmholtz_solver.h
 * (cuda_helmholtz_solver.h:5-11): identical C++-linkage signature.
 *
 *   laplace u + lambda * u = f
 *
 * f is a device array of (NX+1)(NY+1)(NZ+1) doubles, [z][y][x], overwritten
 * with u.  Boundary codes per axis: 0 periodic, 1 Dirichlet-Dirichlet,
 * 2 Dirichlet-Neumann, 3 Neumann-Neumann, 4 Neumann-Dirichlet.  Like the
 * reference it returns 0, is synchronous, and exits the process on a bad
 * boundary code ("bad boundary condition", exit(1)) or a CUDA error.  The
 * status-returning, stream-ordered form is chz_helmholtz_solve in
 * cuhelmholtz_b200.h. */
#pragma once
int cuda_helmholtz_solver(double left, double right, int NX, int xbc,
        double *bcl, double *bcr,
        double bottom, double top, int NY, int ybc,
        double *bcb, double *bct,
        double front, double back, int NZ, int zbc,
        double *bcf, double *bce, // bce = bc back
        double lambda, double * f);
