// Batched FP64 Helmholtz solves: many independent problems of different
// sizes, boundary codes and lambdas solved together.
//
// A plan holds, for each of the five line passes, one descriptor per problem
// (windows, strides, kinds, tables) and the prefix sums of the problems' tile
// counts.  Each pass is ONE launch over the tiles of all problems: a CTA finds
// its problem by binary search over the prefix sums and runs the generic
// line-pass tile body on it.  The periodic planes of all problems are one more
// launch.  The six launches are captured once into a CUDA graph; every call
// uploads the problems' array pointers (a small pinned copy) and replays the
// graph.  Pass p of a problem finishes before pass p+1 starts because the
// launches are stream-ordered, so no device-side waiting is involved.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "chz_generic.cuh"
#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace {

constexpr int kPasses = 5;

struct ProbPtrs {
    double* f;
    const double* face[6];  // bcl, bcr, bcb, bct, bcf, bce
};

struct BatchItem {
    PassArgs a;
    LineTables<double> tb;
    int buf_elems;
    int ntx;
    int in_user;   // input is the problem's f (else its work array)
    int out_user;  // output is the problem's f
    long long ws_off;
};

struct FixItem {
    int nx, ny, nz, px, py, pz;
};

__device__ __forceinline__ int find_problem(const int* start, int count, int b) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <bool CONTIG>
__global__ void __launch_bounds__(kThreads, 2)
batch_pass(const BatchItem* __restrict__ items, const int* __restrict__ start, int count,
           const ProbPtrs* __restrict__ ptrs, double* ws) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int s = find_problem(start, count, blockIdx.x);
    const BatchItem& it = items[s];
    PassArgs a = it.a;
    const ProbPtrs& p = ptrs[s];
    if (a.has_bc) {
        a.bc.f = p.f;
        a.bc.bcl = p.face[0];
        a.bc.bcr = p.face[1];
        a.bc.bcb = p.face[2];
        a.bc.bct = p.face[3];
        a.bc.bcf = p.face[4];
        a.bc.bce = p.face[5];
    }
    const double* in = it.in_user ? p.f : ws + it.ws_off;
    double* out = it.out_user ? p.f : ws + it.ws_off;
    const int local = blockIdx.x - start[s];
    line_pass_tile<double, double, double, CONTIG, kRadixAll>(in, out, a, it.tb, it.buf_elems, local % it.ntx,
                                                              local / it.ntx, smem_raw);
}

// Periodic planes of every problem (one CTA per problem).
__global__ void batch_fixup(const FixItem* __restrict__ fx, const ProbPtrs* __restrict__ ptrs) {
    const FixItem q = fx[blockIdx.x];
    if (!q.px && !q.py && !q.pz) return;
    double* f = ptrs[blockIdx.x].f;
    const long long sfy = q.nx + 1, sfz = (long long)(q.nx + 1) * (q.ny + 1);
    const long long nX = q.px ? (long long)(q.ny + 1) * (q.nz + 1) : 0;
    const long long nY = q.py ? (long long)(q.nx + 1) * (q.nz + 1) : 0;
    const long long nZ = q.pz ? (long long)(q.nx + 1) * (q.ny + 1) : 0;
    for (long long e = threadIdx.x; e < nX + nY + nZ; e += blockDim.x) {
        int i, j, k;
        if (e < nX) {
            k = (int)(e / (q.ny + 1));
            j = (int)(e - (long long)k * (q.ny + 1));
            i = q.nx;
        } else if (e < nX + nY) {
            const long long r = e - nX;
            k = (int)(r / (q.nx + 1));
            i = (int)(r - (long long)k * (q.nx + 1));
            j = q.ny;
        } else {
            const long long r = e - nX - nY;
            j = (int)(r / (q.nx + 1));
            i = (int)(r - (long long)j * (q.nx + 1));
            k = q.nz;
        }
        const int si = (q.px && i == q.nx) ? 0 : i;
        const int sj = (q.py && j == q.ny) ? 0 : j;
        const int sk = (q.pz && k == q.nz) ? 0 : k;
        f[k * sfz + j * sfy + i] = f[sk * sfz + sj * sfy + si];
    }
}

}  // namespace
}  // namespace chz

using namespace chz;

struct chz_batch_plan {
    int count = 0;
    int device = 0;
    std::vector<AxisSolve> ax;          // 3 per problem
    std::vector<FixItem> fix_h;
    BatchItem* items_d[kPasses] = {};
    int* start_d[kPasses] = {};
    int tiles[kPasses] = {};
    size_t smem[kPasses] = {};
    bool contig[kPasses] = {};
    FixItem* fix_d = nullptr;
    ProbPtrs* ptrs_d = nullptr;
    ProbPtrs* ptrs_h = nullptr;  // pinned
    double* ws = nullptr;
    size_t ws_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
};

namespace {

void free_plan(chz_batch_plan* p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (int q = 0; q < kPasses; ++q) {
        if (p->items_d[q]) cudaFree(p->items_d[q]);
        if (p->start_d[q]) cudaFree(p->start_d[q]);
    }
    if (p->fix_d) cudaFree(p->fix_d);
    if (p->ptrs_d) cudaFree(p->ptrs_d);
    if (p->ptrs_h) cudaFreeHost(p->ptrs_h);
    if (p->ws) cudaFree(p->ws);
    if (p->graph_stream) cudaStreamDestroy(p->graph_stream);
    delete p;
}

// Records the six launches of one batched solve on `s`.
int enqueue(chz_batch_plan* p, cudaStream_t s) {
    for (int q = 0; q < kPasses; ++q) {
        if (p->tiles[q] == 0) continue;
        if (p->contig[q])
            batch_pass<true><<<p->tiles[q], kThreads, p->smem[q], s>>>(p->items_d[q], p->start_d[q], p->count,
                                                                       p->ptrs_d, p->ws);
        else
            batch_pass<false><<<p->tiles[q], kThreads, p->smem[q], s>>>(p->items_d[q], p->start_d[q], p->count,
                                                                        p->ptrs_d, p->ws);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail((int)e, "batched pass");
    }
    batch_fixup<<<p->count, 256, 0, s>>>(p->fix_d, p->ptrs_d);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail((int)e, "batched periodic planes");
    return CHZ_SUCCESS;
}

}  // namespace

extern "C" {

int chz_batch_plan_create(int count, const int* dims, const int* bcs, const double* domains,
                          const double* lambdas, chz_batch_plan** out) {
    g_last_error[0] = 0;
    if (!out || !dims || !bcs || !lambdas) return fail(CHZ_ERROR_INVALID_VALUE, "NULL argument");
    if (count < 1) return fail(CHZ_ERROR_INVALID_VALUE, "count must be >= 1");
    *out = nullptr;
    chz_batch_plan* p = new (std::nothrow) chz_batch_plan();
    if (!p) return fail(CHZ_ERROR_ALLOC, "host allocation failed");
    p->count = count;
    cudaGetDevice(&p->device);
    p->ax.resize(3 * (size_t)count);
    p->fix_h.resize(count);
    std::vector<long long> ws_off(count);
    long long ws_total = 0;
    int rc;
    for (int i = 0; i < count; ++i) {
        const double* d = domains ? domains + 6 * i : nullptr;
        const double unit[6] = {0, 1, 0, 1, 0, 1};
        if (!d) d = unit;
        for (int a = 0; a < 3; ++a) {
            if ((rc = setup_axis(dims[3 * i + a], bcs[3 * i + a], d[2 * a], d[2 * a + 1], &p->ax[3 * i + a])) ||
                (rc = check_len(dims[3 * i + a], "batch"))) {
                free_plan(p);
                return rc;
            }
        }
        ws_off[i] = ws_total;
        ws_total += (long long)((padded_elems(dims[3 * i], dims[3 * i + 1], dims[3 * i + 2]) + 31) & ~(size_t)31);
        p->fix_h[i] = {dims[3 * i], dims[3 * i + 1], dims[3 * i + 2], bcs[3 * i] == 0, bcs[3 * i + 1] == 0,
                       bcs[3 * i + 2] == 0};
    }
    // descriptors of every pass
    std::vector<BatchItem> items[kPasses];
    std::vector<int> start[kPasses];
    for (int q = 0; q < kPasses; ++q) {
        items[q].resize(count);
        start[q].resize(count + 1);
        p->contig[q] = (q == 0 || q == 4);
    }
    for (int i = 0; i < count; ++i) {
        const AxisSolve& X = p->ax[3 * i];
        const AxisSolve& Y = p->ax[3 * i + 1];
        const AxisSolve& Z = p->ax[3 * i + 2];
        DeviceLineTables tx, ty, tz;
        const double *ex, *ey, *ez;
        if ((rc = tables_for(X.n, 1, &tx)) || (rc = tables_for(Y.n, 1, &ty)) || (rc = tables_for(Z.n, 1, &tz)) ||
            (rc = eig_table(X, &ex)) || (rc = eig_table(Y, &ey)) || (rc = eig_table(Z, &ez))) {
            free_plan(p);
            return rc;
        }
        const int nx = X.n, ny = Y.n, nz = Z.n;
        const long long fy = nx + 1, fz = (long long)(nx + 1) * (ny + 1);
        const long long wy = nx + 2, wz = (long long)(nx + 2) * (ny + 2);
        const double lam = lambdas[i];
        auto fill = [&](int q, int kind, int kind2, const DeviceLineTables& t, int n, bool contig, int u0, int u1,
                        int v0, int v1, long long isu, long long isv, long long isl, int ld0, int ld1, long long osu,
                        long long osv, long long osl, int st0, int st1, int in_user, int out_user) {
            const LineGeom g = line_geometry(n, 1, contig);
            BatchItem& it = items[q][i];
            std::memset(&it, 0, sizeof(it));
            PassArgs& a = it.a;
            a.kind = kind; a.kind2 = kind2;
            a.u0 = u0; a.nu = u1 - u0 + 1; a.v0 = v0;
            a.in_su = isu; a.in_sv = isv; a.in_sl = isl; a.ld_lo = ld0; a.ld_hi = ld1;
            a.out_su = osu; a.out_sv = osv; a.out_sl = osl; a.st_lo = st0; a.st_hi = st1;
            a.scale = 1.0; a.use_scale = 0;
            a.PR = g.PR; a.log2W = g.log2W;
            it.tb.twM = static_cast<const double2*>(t.twM);
            it.tb.twN = static_cast<const double2*>(t.twN);
            it.tb.tw4N = static_cast<const double2*>(t.tw4N);
            it.tb.inv4sin = static_cast<const double*>(t.inv4sin);
            it.tb.N = t.N; it.tb.M = t.M; it.tb.rp = t.rp;
            it.buf_elems = (int)g.buf_elems;
            it.ntx = (a.nu + g.W - 1) / g.W;
            it.in_user = in_user; it.out_user = out_user;
            it.ws_off = ws_off[i];
            start[q][i + 1] = it.ntx * (v1 - v0 + 1);
            p->smem[q] = std::max(p->smem[q], g.smem_bytes);
        };
        fill(0, X.kf, -1, tx, nx, true, Y.s, Y.e, Z.s, Z.e, fy, fz, 1, X.s, X.e, wy, wz, 1, X.sp0, X.sp1, 1, 0);
        {
            BcArgs& bc = items[0][i].a.bc;
            items[0][i].a.has_bc = 1;
            bc.xbc = X.bc; bc.ybc = Y.bc; bc.zbc = Z.bc;
            bc.xs = X.s; bc.xe = X.e; bc.ys = Y.s; bc.ye = Y.e; bc.zs = Z.s; bc.ze = Z.e;
            bc.nx = nx; bc.ny = ny; bc.nz = nz;
            bc.dx = X.d; bc.dy = Y.d; bc.dz = Z.d;
            bc.dx2 = X.d2; bc.dy2 = Y.d2; bc.dz2 = Z.d2;
        }
        fill(1, Y.kf, -1, ty, ny, false, X.sp0, X.sp1, Z.s, Z.e, 1, wz, wy, Y.s, Y.e, 1, wz, wy, Y.sp0, Y.sp1, 0, 0);
        fill(2, Z.kf, Z.ki, tz, nz, false, X.sp0, X.sp1, Y.sp0, Y.sp1, 1, wy, wz, Z.s, Z.e, 1, wy, wz, Z.s, Z.e, 0, 0);
        {
            PassArgs& a = items[2][i].a;
            a.has_div = 1;
            a.dv.ex = ex; a.dv.ey = ey; a.dv.ez = ez;
            a.dv.lambda = lam;
            a.dv.perturb = (lam == 0.0 && (X.bc == 0 || X.bc == 3) && (Y.bc == 0 || Y.bc == 3) &&
                            (Z.bc == 0 || Z.bc == 3));
            a.dv.xz_hi = X.bc == 0 ? 1 : 0;
            a.dv.yz_hi = Y.bc == 0 ? 1 : 0;
            a.dv.zz_hi = Z.bc == 0 ? 1 : 0;
            a.dv.lo = Z.sp0; a.dv.hi = Z.sp1;
        }
        fill(3, Y.ki, -1, ty, ny, false, X.sp0, X.sp1, Z.s, Z.e, 1, wz, wy, Y.sp0, Y.sp1, 1, wz, wy, Y.s, Y.e, 0, 0);
        fill(4, X.ki, -1, tx, nx, true, Y.s, Y.e, Z.s, Z.e, wy, wz, 1, X.sp0, X.sp1, fy, fz, 1, X.s, X.e, 0, 1);
        items[4][i].a.scale = solver_scale(X, Y, Z);
        items[4][i].a.use_scale = 1;
    }
    for (int q = 0; q < kPasses; ++q) {
        start[q][0] = 0;
        for (int i = 0; i < count; ++i) start[q][i + 1] += start[q][i];
        p->tiles[q] = start[q][count];
    }
    // device copies, workspace, pinned pointer table
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < kPasses && e == cudaSuccess; ++q) {
        e = cudaMalloc(&p->items_d[q], sizeof(BatchItem) * count);
        if (e == cudaSuccess) e = cudaMalloc(&p->start_d[q], sizeof(int) * (count + 1));
        if (e == cudaSuccess)
            e = cudaMemcpy(p->items_d[q], items[q].data(), sizeof(BatchItem) * count, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(p->start_d[q], start[q].data(), sizeof(int) * (count + 1), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMalloc(&p->fix_d, sizeof(FixItem) * count);
    if (e == cudaSuccess) e = cudaMemcpy(p->fix_d, p->fix_h.data(), sizeof(FixItem) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&p->ptrs_d, sizeof(ProbPtrs) * count);
    if (e == cudaSuccess) e = cudaMallocHost(&p->ptrs_h, sizeof(ProbPtrs) * count);
    p->ws_bytes = (size_t)ws_total * sizeof(double);
    if (e == cudaSuccess) e = cudaMalloc(&p->ws, p->ws_bytes);
    if (e == cudaSuccess) {
        // one attribute per kernel instantiation: the largest need of its passes
        size_t sc = 0, ss = 0;
        for (int q = 0; q < kPasses; ++q) (p->contig[q] ? sc : ss) = std::max(p->contig[q] ? sc : ss, p->smem[q]);
        e = cudaFuncSetAttribute(batch_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sc);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(batch_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss);
    }
    if (e != cudaSuccess) {
        const int st = (e == cudaErrorMemoryAllocation) ? fail(CHZ_ERROR_ALLOC, "batch plan allocation failed")
                                                        : cuda_fail((int)e, "batch plan");
        free_plan(p);
        return st;
    }
    *out = p;
    return CHZ_SUCCESS;
}

size_t chz_batch_workspace_bytes(const chz_batch_plan* plan) { return plan ? plan->ws_bytes : 0; }

int chz_batch_solve(chz_batch_plan* p, double* const* f, const double* const* faces, void* stream) {
    g_last_error[0] = 0;
    if (!p || !f) return fail(CHZ_ERROR_INVALID_VALUE, "NULL argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    for (int i = 0; i < p->count; ++i) {
        if (!f[i]) return fail(CHZ_ERROR_INVALID_VALUE, "f[%d] is NULL", i);
        p->ptrs_h[i].f = f[i];
        for (int k = 0; k < 6; ++k) p->ptrs_h[i].face[k] = faces ? faces[6 * i + k] : nullptr;
        int rc;
        if ((rc = check_faces(p->ax[3 * i], p->ptrs_h[i].face[0], p->ptrs_h[i].face[1], "x")) ||
            (rc = check_faces(p->ax[3 * i + 1], p->ptrs_h[i].face[2], p->ptrs_h[i].face[3], "y")) ||
            (rc = check_faces(p->ax[3 * i + 2], p->ptrs_h[i].face[4], p->ptrs_h[i].face[5], "z")))
            return rc;
    }
    // the pinned table is reused: wait for the previous call's upload first
    cudaError_t e = cudaMemcpyAsync(p->ptrs_d, p->ptrs_h, sizeof(ProbPtrs) * p->count, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail((int)e, "pointer upload");
    if (!p->exec) {
        // capture the six launches once, on a private stream (the legacy
        // default stream cannot be captured); the graph replays on any stream
        if (!p->graph_stream) {
            e = cudaStreamCreateWithFlags(&p->graph_stream, cudaStreamNonBlocking);
            if (e != cudaSuccess) return cuda_fail((int)e, "capture stream");
        }
        cudaStream_t cs = p->graph_stream;
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail((int)e, "begin capture");
        const int rc = enqueue(p, cs);
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
        if (rc != CHZ_SUCCESS) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e2 != cudaSuccess) return cuda_fail((int)e2, "end capture");
        e = cudaGraphInstantiate(&p->exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            return cuda_fail((int)e, "graph instantiate");
        }
        p->graph = g;
    }
    trace_begin(s, "batch_graph");
    e = cudaGraphLaunch(p->exec, s);
    for (int q = 0; q < kPasses + 1; ++q) count_launch();
    trace_end(s);
    if (e != cudaSuccess) return cuda_fail((int)e, "graph launch");
    return CHZ_SUCCESS;
}

int chz_batch_plan_destroy(chz_batch_plan* plan) {
    if (plan) {
        cudaDeviceSynchronize();
        free_plan(plan);
    }
    return CHZ_SUCCESS;
}

}  // extern "C"
