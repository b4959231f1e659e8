/*
 * cuhelmholtz_b200 -- C ABI of the B200-native (sm_100a) 3-D mixed
 * DFT/DST/DCT transform and FFT-diagonalised Helmholtz solver.
 *
 * Every entry point takes plain device pointers, sizes and an optional CUDA
 * stream handle (`void*` holding a cudaStream_t; NULL = legacy default stream),
 * returns a chz_status code instead of exiting the process, and is
 * stream-ordered: it enqueues work and returns without synchronising.
 *
 * Layouts (identical to the reference's):
 *   transform array : (NZ+2)(NY+2)(NX+2) doubles, [z][y][x], rows of NX+2
 *                     (cudasymmfft/funcinterface.cu:48-83 plan strides)
 *   solver f        : (NZ+1)(NY+1)(NX+1) doubles, [z][y][x], in place
 *                     (cudahelmholtz/cuda_helmholtz_solver.cu:178-179)
 *   Neumann faces   : x faces (NZ+1)(NY+1) [z][y], y faces (NZ+1)(NX+1) [z][x],
 *                     z faces (NY+1)(NX+1) [y][x]; NULL where the boundary
 *                     code does not read them (testgpurectangle.cu:46-57)
 *
 * The C++-linkage drop-in signatures of the reference live in funcinterface.h
 * and cuda_helmholtz_solver.h next to this header.
 */
#ifndef CUHELMHOLTZ_B200_H_
#define CUHELMHOLTZ_B200_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum chz_status {
    CHZ_SUCCESS = 0,
    CHZ_ERROR_INVALID_VALUE = 1,    /* bad size, boundary code, kind or NULL pointer */
    CHZ_ERROR_UNSUPPORTED_SIZE = 2, /* N odd, < 4, > 2048, or N/2 has a prime factor > 13 */
    CHZ_ERROR_NOT_CUBIC = 3,        /* in-place do_transform on a non-cubic grid */
    CHZ_ERROR_CUDA = 4,             /* a CUDA runtime call failed */
    CHZ_ERROR_ALLOC = 5,            /* device allocation failed */
    CHZ_ERROR_WORKSPACE = 6,        /* caller workspace too small or misaligned */
    CHZ_ERROR_TIMEOUT = 7           /* a kernel's bounded wait ran out (see chz_stream_status) */
} chz_status;

/* transform kinds: same values as the reference's enum transform_kind
 * (cudasymmfft/global.h:6-15). */
enum {
    CHZ_DCT_1 = 0, CHZ_DCT_2 = 1, CHZ_DCT_3 = 2, CHZ_DST_1 = 3,
    CHZ_DST_2 = 4, CHZ_DST_3 = 5, CHZ_DFT_R2C = 6, CHZ_DFT_C2R = 7
};

/* Library version, major * 10000 + minor * 100 + patch. */
int chz_version(void);

/* Human-readable name of a status code. */
const char* chz_status_string(int status);

/* Detail of the last error raised on the calling host thread ("" if none). */
const char* chz_last_error(void);

/* 3-D mixed transform (replaces do_transform, cudasymmfft/funcinterface.cu:25-40).
 * d_out == NULL or d_out == d_data: in place, the grid must be a cube
 * (CHZ_ERROR_NOT_CUBIC otherwise, where the reference exits).  Otherwise the
 * result is written to d_out and d_data is left unchanged (the reference uses
 * d_data as scratch).  Entries outside each kind's output window are not
 * written. */
int chz_do_transform(double* d_data, double* d_out, int nx, int ny, int nz,
                     int x_kind, int y_kind, int z_kind, void* stream);

/* Same transform without the cubic restriction on in-place calls. */
int chz_do_transform_any(double* d_data, double* d_out, int nx, int ny, int nz,
                         int x_kind, int y_kind, int z_kind, void* stream);

/* Device workspace the solver needs for these sizes (bytes).
 * precision: 0 = FP64 solve, 1 = FP32 + FP64-refinement solve. */
size_t chz_helmholtz_workspace_size(int nx, int ny, int nz, int precision);

/* Helmholtz solve  lap_h u + lambda u = f  (replaces cuda_helmholtz_solver,
 * cudahelmholtz/cuda_helmholtz_solver.cu:33-380), FP64, in place on f.
 * Uses a library-owned workspace cached per (device, stream). */
int chz_helmholtz_solve(double left, double right, int nx, int xbc,
                        const double* bcl, const double* bcr,
                        double bottom, double top, int ny, int ybc,
                        const double* bcb, const double* bct,
                        double front, double back, int nz, int zbc,
                        const double* bcf, const double* bce,
                        double lambda, double* f, void* stream);

/* The solve with the reference's 19-point variant (_nonpoisson_devide_19points_,
 * _cuda_helmholtz_.inl:255-274, commented out at cuda_helmholtz_solver.cu:325
 * and :338): the spectral division by the eigenvalues of the compact 19-point
 * Laplacian, (2/3 (ci cj + ci ck + cj ck + ci + cj + ck) - 4) / h^2 + lambda,
 * with the right-hand side filtered by 1/2 + (ci + cj + ck) / 6,
 * ca = cos(m pi / N); the boundary terms are the 7-point solve's.  As the
 * reference kernel: one grid spacing on all axes and codes 1 and 3 only
 * (CHZ_ERROR_INVALID_VALUE otherwise).  Mode (0,0,0) of an all-Neumann
 * lambda = 0 problem is set to 0 (the reference divides by 0 there). */
int chz_helmholtz_solve_19pt(double left, double right, int nx, int xbc,
                             const double* bcl, const double* bcr,
                             double bottom, double top, int ny, int ybc,
                             const double* bcb, const double* bct,
                             double front, double back, int nz, int zbc,
                             const double* bcf, const double* bce,
                             double lambda, double* f, void* stream);

/* Helmholtz solve as chz_helmholtz_solve that also returns PERTRB, as
 * FISHPACK's hw3crt does (hw3crt_wrapper.cpp:20-28 passes &pertrb to hw3crt_
 * but does not return it): when lambda = 0 and every code is 0 or 3 the
 * problem is singular and PERTRB is the constant removed from the right-hand
 * side so that a solution exists -- the weighted mean of b (f with the
 * boundary terms) over the unknown window, weight 1/2 per Neumann boundary
 * index; otherwise 0.  The solution is chz_helmholtz_solve's (its constant
 * mode is 0; hw3crt returns the same solution plus an arbitrary constant).
 * *pertrb is a host value; in the singular case the call waits for `stream`
 * to read it back. */
int chz_helmholtz_solve_pertrb(double left, double right, int nx, int xbc,
                               const double* bcl, const double* bcr,
                               double bottom, double top, int ny, int ybc,
                               const double* bcb, const double* bct,
                               double front, double back, int nz, int zbc,
                               const double* bcf, const double* bce,
                               double lambda, double* f, double* pertrb, void* stream);

/* As chz_helmholtz_solve with a caller-owned device workspace of at least
 * chz_helmholtz_workspace_size(nx, ny, nz, 0) bytes, 256-byte aligned. */
int chz_helmholtz_solve_ws(double left, double right, int nx, int xbc,
                           const double* bcl, const double* bcr,
                           double bottom, double top, int ny, int ybc,
                           const double* bcb, const double* bct,
                           double front, double back, int nz, int zbc,
                           const double* bcf, const double* bce,
                           double lambda, double* f,
                           void* workspace, size_t workspace_bytes, void* stream);

/* Adjoint of the solve map (no counterpart in the reference).  The forward
 * map is the whole in-place API map of chz_helmholtz_solve: f (with its
 * Dirichlet faces), the six Neumann arrays and lambda -> u.  Given
 * g = dL/du (full (NZ+1)(NY+1)(NX+1) grid) and the forward solution u, writes
 * dL/df into df (full grid), dL/d(Neumann array) into dbcl..dbce (each may be
 * NULL; entries the solve does not read get 0) and, if dlambda is not NULL,
 * dL/dlambda into the device scalar *dlambda.  A^-T = W A^-1 W^-1 with W =
 * 1/2 at Neumann boundary nodes, so the work is one homogeneous solve
 * (precision 0: FP64; 1: FP32 + `corrections` FP64 refinements) between two
 * scalings.  workspace: at least chz_helmholtz_adjoint_workspace_size bytes,
 * 256-byte aligned.  All pointers are device pointers. */
size_t chz_helmholtz_adjoint_workspace_size(int nx, int ny, int nz, int precision);
int chz_helmholtz_adjoint(double left, double right, int nx, int xbc,
                          double bottom, double top, int ny, int ybc,
                          double front, double back, int nz, int zbc, double lambda,
                          const double* g, const double* u, double* df,
                          double* dbcl, double* dbcr, double* dbcb, double* dbct,
                          double* dbcf, double* dbce, double* dlambda,
                          int precision, int corrections,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Batched FP64 solves: `count` independent problems of any supported sizes,
 * boundary codes, domains and lambdas (no counterpart in the reference, which
 * solves one problem per call).  The plan precomputes every problem's pass
 * descriptors and a work array for all of them; each chz_batch_solve replays
 * on `stream` a CUDA graph captured once, of one of two launch forms:
 *   0: ONE persistent launch over a device work queue (every tile of the five
 *      passes of every problem, pass by pass, then each problem's periodic
 *      planes; an item waits -- bounded -- for its problem's previous pass),
 *      with the reset of its counters;
 *   1: per pass, one launch of the register-resident line kernel for each
 *      group of problems with the same line length and kinds (the lengths
 *      with a register radix plan: powers of two 32..1024 and the mixed
 *      N = 24..384 listed under chz_set_kernel_family), then one launch of
 *      the shared-memory mixed-radix kernel over the other problems; then one
 *      launch for the periodic planes.
 * The plan times both at creation and keeps the faster
 * (chz_batch_plan_launch).  A wait that runs out is reported by
 * chz_stream_status.
 *   dims    : 3*count cell counts (nx, ny, nz per problem)
 *   bcs     : 3*count boundary codes 0..4
 *   domains : 6*count extents (left, right, bottom, top, front, back), or
 *             NULL for the unit cube
 *   lambdas : count values
 * chz_batch_solve takes count device pointers f[i] (solved in place, layout
 * as chz_helmholtz_solve) and 6*count face pointers (bcl, bcr, bcb, bct, bcf,
 * bce per problem; NULL entries where unused; faces == NULL if none are
 * used).  It synchronises `stream` once to upload the pointers, then returns
 * with the graph enqueued. */
typedef struct chz_batch_plan chz_batch_plan;
int chz_batch_plan_create(int count, const int* dims, const int* bcs, const double* domains,
                          const double* lambdas, chz_batch_plan** plan);
int chz_batch_solve(chz_batch_plan* plan, double* const* f, const double* const* faces, void* stream);
size_t chz_batch_workspace_bytes(const chz_batch_plan* plan);
int chz_batch_plan_destroy(chz_batch_plan* plan);

/* Autotuner of the batch plans (on by default): chz_batch_plan_create times
 * every pass over all problems (one launch per pass) at tile sizes of
 * 1024..16384 values per tile, then at the three radix schedules, on scratch
 * stand-ins for the problems' arrays, and keeps the fastest per pass.
 * Returns the previous setting. */
int chz_batch_set_autotune(int on);

/* Tile size chosen for each of the five passes (values per tile; targets[5])
 * and its measured time per launch in ms (ms[5]; 0 when not tuned). */
int chz_batch_plan_tiles(const chz_batch_plan* plan, int* targets, float* ms);

/* Radix schedule chosen for each of the five passes (variants[5]): 0 radix
 * 8s first, then 4 or 2, then the odd primes; 1 the same in reverse order; 2
 * radix 4s (and a 2) in place of the 8s.  The autotuner times the three at
 * the chosen tile size, per pass, over all problems. */
int chz_batch_plan_radix(const chz_batch_plan* plan, int* variants);

/* Fixes the radix schedule of plans created afterwards (0..2 as above; -1,
 * the default, lets the autotuner choose).  Returns the previous setting, or
 * -2 for an unknown schedule. */
int chz_batch_set_radix_schedule(int variant);

/* Launch form of a plan (*mode: 0 persistent, 1 per pass) and the measured
 * time of one batched solve in each (ms[2]; 0 when not timed: the autotuner
 * off or the form fixed by chz_batch_set_launch_mode). */
int chz_batch_plan_launch(const chz_batch_plan* plan, int* mode, float* ms);

/* Fixes the launch form of plans created afterwards (0 or 1 as above; -1, the
 * default, times both).  Returns the previous setting, or -2 for an unknown
 * form. */
int chz_batch_set_launch_mode(int mode);

/* Kernel launches one chz_batch_solve of this plan replays (1 in the
 * persistent form; the groups, leftover launches and periodic-plane launch in
 * the per-pass form); CHZ_ERROR_INVALID_VALUE (negative) for a NULL plan. */
int chz_batch_plan_kernels(const chz_batch_plan* plan);

/* Helmholtz solve with FP32 transforms and FP64 iterative refinement.
 * u0 = S32(b); then up to max_corrections times: r = b - A u in FP64 (the
 * 7-point operator with the boundary terms, as the FP64 solve's system),
 * u += S32(r).  S32 is the diagonal solve with FP32 transforms.  With
 * tol > 0 (or rel_residual != NULL) the relative residual ||r|| / ||b|| is
 * read back before each correction (a stream synchronisation) and refinement
 * stops when it is <= tol or no longer halves; with tol <= 0 and
 * rel_residual == NULL exactly max_corrections corrections run with no
 * synchronisation.  corrections_done / rel_residual (may be NULL) report the
 * corrections applied and the last residual measured (-1 if none).
 * workspace: NULL for the library-owned one, else at least
 * chz_helmholtz_workspace_size(nx, ny, nz, 1) bytes, 256-byte aligned.
 * No counterpart in the reference (its solver is FP64 only). */
int chz_helmholtz_solve_refined(double left, double right, int nx, int xbc,
                                const double* bcl, const double* bcr,
                                double bottom, double top, int ny, int ybc,
                                const double* bcb, const double* bct,
                                double front, double back, int nz, int zbc,
                                const double* bcf, const double* bce,
                                double lambda, double* f, int max_corrections, double tol,
                                int* corrections_done, double* rel_residual,
                                void* workspace, size_t workspace_bytes, void* stream);

/* FP64 Helmholtz solve that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- device memory owned
 * by another allocator or arena, a hard memory budget, or code that must not
 * wait on the allocator.  The work array and the per-axis tables are
 * file-scope __device__ arrays of fixed size (64 MiB + about 108 KiB), held by every
 * GPU that loads the library until exit.  Limits: (NX+2)(NY+2)(NZ+2) <= 2^23
 * and at most 1024 cells per axis; larger problems return
 * CHZ_ERROR_UNSUPPORTED_SIZE.  All calls share the arrays (calls that overlap
 * on the GPU race); each call rewrites everything it reads.  The first call on
 * a device looks up the arrays' addresses; make it before any stream capture.
 * Same arguments and results as chz_helmholtz_solve. */
int chz_helmholtz_solve_noalloc(double left, double right, int nx, int xbc,
                                const double* bcl, const double* bcr,
                                double bottom, double top, int ny, int ybc,
                                const double* bcb, const double* bct,
                                double front, double back, int nz, int zbc,
                                const double* bcf, const double* bce,
                                double lambda, double* f, void* stream);

/* Slab-decomposed solve over several GPUs (no counterpart in the reference,
 * whose solver runs on one GPU): f is split into slabs of whole z planes, the
 * rank of slab r holding planes [z0, z0 + nzl) as a contiguous array
 * (nzl (NY+1)(NX+1) doubles), and one solve is
 *   1. chz_slab_forward on every rank: x and y forward passes (boundary terms
 *      applied) of the slab's planes inside the z unknown window, f_slab ->
 *      ws_slab (nzl (NY+2)(NX+2) doubles, 256-byte aligned;
 *      chz_slab_work_elems), plane k of the slab at ws_slab + (k - z0)(NY+2)(NX+2);
 *   2. an all-to-all: the rank of y-row block [j0, j0 + nj) of the spectral y
 *      window receives those rows of every unknown z plane, as the pencil
 *      (Ze - Zs + 1) x nj x (NX+2) doubles, [k - Zs][j - j0][x];
 *   3. chz_slab_z on every rank: the fused z pass (forward, eigenvalue
 *      division, inverse) on its pencil (256-byte aligned);
 *   4. the reverse all-to-all into ws_slab;
 *   5. chz_slab_inverse on every rank: y and x inverse passes, ws_slab ->
 *      f_slab, scaled as the solve, plus the x and y periodic copies;
 *   6. with a periodic z axis, plane NZ <- plane 0 (across slabs: the caller's).
 * The exchanges are the caller's (cuhelmholtz_b200.slab does them over
 * torch.distributed).  The slab holding the first (last) unknown z plane of a
 * Dirichlet z face must hold plane 0 (NZ), whose values the boundary terms
 * read.  Face arrays are the whole problem's.  The result equals
 * chz_helmholtz_solve's on the whole grid.  Stream-ordered. */
int chz_slab_forward(double left, double right, int nx, int xbc, const double* bcl, const double* bcr,
                     double bottom, double top, int ny, int ybc, const double* bcb, const double* bct,
                     double front, double back, int nz, int zbc, const double* bcf, const double* bce,
                     const double* f_slab, int z0, int nzl, double* ws_slab, void* stream);
int chz_slab_z(double left, double right, int nx, int xbc, double bottom, double top, int ny, int ybc,
               double front, double back, int nz, int zbc, double lambda, double* pencil, int j0, int nj,
               void* stream);
int chz_slab_inverse(double left, double right, int nx, int xbc, double bottom, double top, int ny, int ybc,
                     double front, double back, int nz, int zbc, double* ws_slab, double* f_slab, int z0,
                     int nzl, void* stream);
size_t chz_slab_work_elems(int nx, int ny, int nzl);

/* Releases the library-owned workspaces and cached tables of the current
 * device (after synchronising it). */
int chz_release_cached(void);

/* Launch tracing (the reference's per-stage host timers, TIME_TEST blocks in
 * cudasymmfft/dst1funcinplace.cu:21-47, replaced by CUDA events).  With
 * tracing on, every kernel launch of this library is bracketed by CUDA events
 * recorded on its own stream.  chz_trace_collect waits for them, writes one
 * line "label launches total_ms" per kernel label into buf (NUL-terminated,
 * truncated to len), clears the records and returns the number of launches
 * collected (-1 on a CUDA error). */
int chz_trace_enable(int on);
int chz_trace_collect(char* buf, size_t len);

/* Kernel family: 0 (default) uses the TMA-pipelined kernel for the strided
 * (y, z) passes of N = 128, 192, 256, 320, 512, the register-resident line
 * kernels for the other passes of lengths N = 32..1024 that are powers of two
 * and of the mixed lengths N = 24, 40, 48, 56, 80, 96, 112, 144, 160, 192,
 * 320, 384 (radix plans with factors 3, 5, 7; in FP32 only 192, 320, 384),
 * and the shared-memory mixed-radix kernel elsewhere; 1
 * uses the mixed-radix kernel for every pass; 2 is family 0 without the TMA
 * kernel (all are checked against the same oracle).  Returns the previous
 * setting, or -1 for an unknown family. */
int chz_set_kernel_family(int family);

/* Flags raised by the kernels' bounded waits since the last reset (0 when no
 * wait ran out); reset != 0 clears them.  Synchronous.  -1 on a CUDA error. */
int chz_debug_flags(int reset);

/* Status of the work queued on `stream`: waits for it, then returns
 * CHZ_ERROR_TIMEOUT (and clears the flags) when a kernel of this library on
 * the current device gave up one of its bounded waits since the last check --
 * its results are then not valid -- CHZ_ERROR_CUDA on a CUDA error, else
 * CHZ_SUCCESS.  The stream-ordered entry points return before their kernels
 * run, so a wait that runs out surfaces here (the reference's synchronous
 * C++ entry points in funcinterface.h / cuda_helmholtz_solver.h check it
 * themselves and exit, as they do on a CUDA error).  No counterpart in the
 * reference, whose kernels have no waits. */
int chz_stream_status(void* stream);

/* Limit of the pipelined kernels' bounded waits on a tile copy or a finished
 * tile, in SM clock cycles (default 2e9, about a second; values below 1e6 are
 * raised to 1e6, <= 0 restores the default).  A wait that runs out raises a
 * flag, its CTA stops waiting and ends after its own copies have landed, and
 * chz_stream_status reports CHZ_ERROR_TIMEOUT.  Applies to launches made
 * after the call.  Returns the previous limit. */
long long chz_set_wait_limit(long long cycles);

/* Self-test of the bounded-wait path: one CTA waits `cycles` SM clock cycles
 * (clamped to 1e3 .. 2e9) on an mbarrier that nothing arrives at, the wait
 * runs out and raises a flag, and the kernel ends; chz_stream_status(stream)
 * then returns CHZ_ERROR_TIMEOUT.  No copy is issued and the context stays
 * usable.  Stream-ordered. */
int chz_wait_selftest(long long cycles, void* stream);

/* Number of kernel launches this library has issued in this process. */
unsigned long long chz_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* CUHELMHOLTZ_B200_H_ */
