// Internal host-side interfaces shared by the kernel and API translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "chz_device.cuh"

namespace chz {

// Bit of the device flag word (chz_tma_host.cu) each kind of bounded wait
// raises when it runs out.
enum WaitFlag {
    kFlagProducer = 1,    // the producer gave up waiting for a finished tile
    kFlagConsumer = 2,    // a compute thread gave up waiting for a tile load
    kFlagAlign = 4,       // misaligned shared memory (nothing was started)
    kFlagDrain = 8,       // a load was still in flight when the CTA ended
    kFlagSelfTest = 16,   // the wait of chz_wait_selftest ran out (as it should)
    kFlagBatchWait = 32   // a batch item gave up waiting for its problem's previous pass
};

// Boundary terms of the reference's _3d_bc{1..4}_ini_{x,y,z}_ kernels
// (_cuda_helmholtz_.inl:70-227), applied while the first solver pass loads f.
struct BcArgs {
    int xbc, ybc, zbc;
    int xs, xe, ys, ye, zs, ze;
    int nx, ny, nz;
    double dx, dy, dz, dx2, dy2, dz2;
    const double* f;  // face values are read from the unmodified input f
    const double *bcl, *bcr, *bcb, *bct, *bcf, *bce;
};

// Eigenvalue division of _divide_/_periodic_divide_ (_cuda_helmholtz_.inl:276-421)
// applied between the forward and inverse transforms of the fused z pass.
// ex/ey/ez are per-entry tables (2 cos(mode * pidiv + shift) - 2) * d^2.
struct DivArgs {
    const double* ex;
    const double* ey;
    const double* ez;
    double lambda;
    int perturb;               // zero the (0,0,0) mode
    int xz_hi, yz_hi, zz_hi;   // entry indices <= these belong to mode 0
    int lo, hi;                // spectral window along the line
};

struct PassArgs {
    int kind;    // transform of the pass
    int kind2;   // >= 0: divide, then this inverse transform, in the same pass
    int u0, nu;  // lines: u in [u0, u0+nu), tiled by W per CTA
    int v0;      // v = v0 + blockIdx.y
    long long in_su, in_sv, in_sl;
    int ld_lo, ld_hi;  // loaded part of the input window (rest is zero)
    long long out_su, out_sv, out_sl;
    int st_lo, st_hi;  // stored part of the output window
    double scale;
    int use_scale;
    const double* acc;  // when set: out = acc + scale * value (same indexing as out)
    int PR;       // real-view pitch (>= W)
    int log2W;
    int has_bc;
    int has_div;
    BcArgs bc;
    DivArgs dv;
};

// Boundary-term sum for element (i, j, k) of f, applied in the reference's
// order: x left, x right, y left, y right, z left, z right.
__device__ __forceinline__ double bc_terms(double v, const BcArgs& b, int i, int j, int k) {
    const long long sfy = b.nx + 1;
    const long long sfz = (long long)(b.nx + 1) * (b.ny + 1);
    const double* f = b.f;
    if (i == b.xs) {
        if (b.xbc == 1 || b.xbc == 2) v -= __ldg(f + k * sfz + j * sfy) * b.dx2;
        else if (b.xbc == 3 || b.xbc == 4) v += 2 * __ldg(b.bcl + (long long)k * (b.ny + 1) + j) * b.dx;
    }
    if (i == b.xe) {
        if (b.xbc == 1 || b.xbc == 4) v -= __ldg(f + k * sfz + j * sfy + b.nx) * b.dx2;
        else if (b.xbc == 2 || b.xbc == 3) v -= 2 * __ldg(b.bcr + (long long)k * (b.ny + 1) + j) * b.dx;
    }
    if (j == b.ys) {
        if (b.ybc == 1 || b.ybc == 2) v -= __ldg(f + k * sfz + i) * b.dy2;
        else if (b.ybc == 3 || b.ybc == 4) v += 2 * __ldg(b.bcb + (long long)k * (b.nx + 1) + i) * b.dy;
    }
    if (j == b.ye) {
        if (b.ybc == 1 || b.ybc == 4) v -= __ldg(f + k * sfz + b.ny * sfy + i) * b.dy2;
        else if (b.ybc == 2 || b.ybc == 3) v -= 2 * __ldg(b.bct + (long long)k * (b.nx + 1) + i) * b.dy;
    }
    if (k == b.zs) {
        if (b.zbc == 1 || b.zbc == 2) v -= __ldg(f + j * sfy + i) * b.dz2;
        else if (b.zbc == 3 || b.zbc == 4) v += 2 * __ldg(b.bcf + (long long)j * (b.nx + 1) + i) * b.dz;
    }
    if (k == b.ze) {
        if (b.zbc == 1 || b.zbc == 4) v -= __ldg(f + b.nz * sfz + j * sfy + i) * b.dz2;
        else if (b.zbc == 2 || b.zbc == 3) v -= 2 * __ldg(b.bce + (long long)j * (b.nx + 1) + i) * b.dz;
    }
    return v;
}

// Register budget: 3 CTAs of 256 threads per SM except with radices 7..13
// (2 CTAs), whose butterflies hold more values.
// One axis of a Helmholtz solve (cuda_helmholtz_solver.cu:44-172).
struct AxisSolve {
    int n, bc;
    int s, e;        // unknown window (cuda_helmholtz_solver.cu:78-103)
    int sp0, sp1;    // spectral window: unknown window, or 0..N+1 when periodic
    int kf, ki;      // forward / inverse kinds
    double d, d2;    // 1/h and 1/h^2 (solver.cu:44-49)
    double pidiv, shift;
};

struct LineGeom {
    int N, M, W, log2W, PR;
    size_t buf_elems;   // elements of T per buffer
    size_t smem_bytes;
    int threads;
};

// Device tables for one line length and precision (cached for the process).
struct DeviceLineTables {
    int N = 0, M = 0;
    RadixPlan rp{};
    void* twM = nullptr;
    void* twN = nullptr;
    void* tw4N = nullptr;
    void* inv4sin = nullptr;
};

// Returns 0 on success; fills `out` with device pointers (cached).
int get_line_tables(int N, int is_double, int device, DeviceLineTables* out);
int factor_radices(int M, RadixPlan* rp);
bool radix_plan_is_pow2(const RadixPlan& rp);
LineGeom line_geometry(int N, int is_double, bool contig);
// The same with an explicit tile size: W = the largest power of two with
// W * N <= target (2 <= W <= 64), halved while the shared memory would exceed
// `max_smem` bytes.
LineGeom line_geometry_target(int N, int is_double, bool contig, int target, size_t max_smem);

// Array pointers of one problem of a batched solve, set at every call.
struct BatchPtrs {
    double* f;
    const double* face[6];  // bcl, bcr, bcb, bct, bcf, bce
};

// One problem of a group of a batched pass that a register-resident kernel
// runs (every member of a group has the same line length and kinds).
struct BatchMember {
    PassArgs a;        // the problem's pass; f and the Neumann faces come from ptrs[prob]
    int prob;          // problem index (into the pointer table)
    int ntx;           // tiles along u (the kernel's W lines each)
    int in_user;       // input: the problem's f (else its work array at ws_off)
    int out_user;      // output: the problem's f
    long long ws_off;  // offset of the problem's work array in ws (doubles)
};

// A group launch: tiles 0 .. ntiles - 1 over the members, member m owning
// tiles start[m] .. start[m + 1] - 1.
struct FastBatchArgs {
    const BatchMember* members;
    const int* start;
    int count;
    int ntiles;
    const BatchPtrs* ptrs;
    double* ws;
};

// Register-resident kernels: lengths they take (FP64 every power of two 16 ..
// 512 and the mixed lengths with a radix plan; FP32 the powers of two), lines
// per tile of the persistent kernel at a half length M (0: none), and the
// launch of one batched group (FP64).
bool fast_path_supported(int M, bool is_double);
int fast_lines_per_tile(int M);
int launch_fast_batch(bool contig, int kind, int kind2, const FastBatchArgs& g, const LineTables<double>& tb,
                      cudaStream_t stream);

// Launchers (return cudaError_t as int).
enum IoType { kIoF64 = 0, kIoF32 = 1 };
int launch_line_pass(int is_double, int in_type, int out_type, bool contig, const void* in,
                     void* out, const PassArgs& a, const DeviceLineTables& tb,
                     const LineGeom& g, int nv, cudaStream_t stream, const char* label);

// Launch tracing: with tracing on, every kernel launch is bracketed by CUDA
// events recorded on its own stream; trace_collect() waits for them and
// reports per-label totals.  launch_count() counts every launch of this library.
void trace_begin(cudaStream_t stream, const char* label);
void trace_end(cudaStream_t stream);
unsigned long long launch_count();
void count_launch();
int launch_periodic_fixup(double* f, int nx, int ny, int nz, int xbc, int ybc, int zbc,
                          cudaStream_t stream);

// Host helpers shared by the API translation units (chz_api.cu).
int fail(int status, const char* fmt, ...);
int cuda_fail(int err, const char* where);
int check_len(int n, const char* axis);
int setup_axis(int n, int bc, double lo, double hi, AxisSolve* a);
int check_faces(const AxisSolve& a, const double* lo, const double* hi, const char* name);
double solver_scale(const AxisSolve& x, const AxisSolve& y, const AxisSolve& z);
int run_solve_passes(const AxisSolve& X, const AxisSolve& Y, const AxisSolve& Z, const DeviceLineTables& tx,
                     const DeviceLineTables& ty, const DeviceLineTables& tz, const double* ex, const double* ey,
                     const double* ez, const double* bcl, const double* bcr, const double* bcb,
                     const double* bct, const double* bcf, const double* bce, double lambda, double* f,
                     double* ws, cudaStream_t s, bool stencil19 = false);
extern thread_local char g_last_error[512];
int current_device();
int tables_for(int n, int is_double, DeviceLineTables* t);
int eig_table(const AxisSolve& a, const double** out);
int cached_workspace(void* stream, size_t bytes, void** out);
size_t padded_elems(int nx, int ny, int nz);

}  // namespace chz
