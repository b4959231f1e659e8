// Batched FP64 Helmholtz solves: many independent problems of different
// sizes, boundary codes and lambdas solved together.
//
// A plan holds, for each of the five line passes, one descriptor per problem
// (windows, strides, kinds, tables, radix schedule) and the prefix sums of the
// problems' tile counts.  A solve takes one of two launch forms.  Persistent:
// ONE launch over a device work queue whose items are every tile of pass 0 of
// every problem, then pass 1, ..., then one periodic-plane item per problem; a
// CTA takes the next item with an atomic counter, finds its pass and problem,
// waits (bounded) until the problem's previous pass has all its tiles done (a
// per-problem, per-pass completion counter released by the tiles), runs the
// generic line-pass tile body and releases its own counter.  Items are handed
// out in pass order and only to running CTAs, so every item waited for is
// already held by a running CTA: no deadlock, whatever the residency.  Per
// pass: one launch per pass over all problems' tiles, then one for the
// periodic planes.  The solve is captured once into a CUDA graph that every
// call replays after uploading the problems' array pointers.
//
// Tile sizes, radix schedules and the launch form come from a project-written
// autotuner: at plan creation each pass is timed over all problems (one launch
// per pass) at several tile sizes, then at several radix schedules of every
// length, then a whole solve in each launch form, and the fastest is kept.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <cstring>
#include <map>
#include <tuple>
#include <new>
#include <vector>

#include "chz_generic.cuh"
#include "chz_internal.h"
#include "cuhelmholtz_b200.h"

namespace chz {
namespace tma {
int* device_flags();
long long wait_limit();
}  // namespace tma
namespace {

constexpr int kPasses = 5;

using ProbPtrs = BatchPtrs;

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

// items[s] is the pass of problem prob[s] (prob == nullptr: of problem s).
template <bool CONTIG>
__global__ void __launch_bounds__(kThreads, 2)
batch_pass(const BatchItem* __restrict__ items, const int* __restrict__ start, int count,
           const ProbPtrs* __restrict__ ptrs, double* ws, const int* __restrict__ prob) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int s = find_problem(start, count, blockIdx.x);
    const BatchItem& it = items[s];
    PassArgs a = it.a;
    const ProbPtrs& p = ptrs[prob ? prob[s] : s];
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

// Periodic planes of one problem, by the threads of one CTA.
__device__ __forceinline__ void fixup_problem(const FixItem& q, double* f) {
    if (!q.px && !q.py && !q.pz) return;
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
        f[k * sfz + j * sfy + i] = __ldcg(f + sk * sfz + sj * sfy + si);
    }
}

// The periodic planes of every problem, one CTA per problem (the per-pass
// launch form's last launch).
__global__ void __launch_bounds__(kThreads) batch_fixup(const FixItem* __restrict__ fix,
                                                        const ProbPtrs* __restrict__ ptrs) {
    fixup_problem(fix[blockIdx.x], ptrs[blockIdx.x].f);
}

// The persistent batched solve.  items[q] / start[q]: pass q's descriptors and
// tile prefix sums; pass_off[q]: index of pass q's first item in the queue
// (pass_off[kPasses]: the periodic-plane items, one per problem;
// pass_off[kPasses + 1]: the end); done[s * kPasses + q]: tiles of problem s's
// pass q finished; next: the queue head.  done and next start at 0.
constexpr int kChunk = 4;   // queue items a CTA takes at once

struct PersistArgs {
    const BatchItem* items[kPasses];
    const int* start[kPasses];
    const int* owner;            // problem of every pass tile, by queue index
    int pass_off[kPasses + 2];
    const FixItem* fix;
    const ProbPtrs* ptrs;
    double* ws;
    int count;
    int* done;
    int* next;
    int* flags;
    long long wait_limit;
};

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__global__ void __launch_bounds__(kThreads, 2) batch_persistent(PersistArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ PassArgs s_args;
    __shared__ LineTables<double> s_tb;
    // The queue state is the same for every thread of the CTA: it lives in
    // shared memory, so no register stays live across the tile body (whose
    // FFT stages need all 128 of them).
    __shared__ int s_g, s_g1;          // current item, end of the taken chunk
    __shared__ int s_q, s_s;           // its pass (kPasses: periodic planes) and problem
    __shared__ int s_cur_q, s_cur_s;   // (pass, problem) of the descriptor in s_args
    const int total = A.pass_off[kPasses + 1];
    if (threadIdx.x == 0) {
        s_g = s_g1 = 0;
        s_cur_q = s_cur_s = -1;
    }
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_g >= s_g1) {            // chunk used up: take the next one
                s_g = atomicAdd(A.next, kChunk);
                s_g1 = min(s_g + kChunk, total);
            }
            const int g = s_g;
            if (g < total) {
                int q = 0;
                while (q < kPasses && g >= A.pass_off[q + 1]) ++q;
                s_q = q;
                s_s = (q < kPasses) ? __ldg(A.owner + g) : g - A.pass_off[kPasses];
            }
        }
        __syncthreads();
        if (s_g >= total) break;
        if (s_q != s_cur_q || s_s != s_cur_s) {
            const int q = s_q, s = s_s;
            // the problem's previous pass must be complete (every one of its
            // tiles released its counter); bounded wait, then a flag
            if (q > 0 && threadIdx.x == 0) {
                const int need = A.start[q - 1][s + 1] - A.start[q - 1][s];
                const int* cnt = A.done + (long long)s * kPasses + (q - 1);
                const long long t0 = clock64();
                while (ld_acquire(cnt) < need) {
                    if (clock64() - t0 > A.wait_limit) {
                        atomicOr(A.flags, kFlagBatchWait);
                        break;
                    }
                }
            }
            // the item's pass descriptor, with the problem's pointers, staged
            // in shared memory once per (pass, problem)
            if (q < kPasses && threadIdx.x == 0) {
                const ProbPtrs& p = A.ptrs[s];
                s_args = A.items[q][s].a;
                s_tb = A.items[q][s].tb;
                if (s_args.has_bc) {
                    s_args.bc.f = p.f;
                    s_args.bc.bcl = p.face[0];
                    s_args.bc.bcr = p.face[1];
                    s_args.bc.bcb = p.face[2];
                    s_args.bc.bct = p.face[3];
                    s_args.bc.bcf = p.face[4];
                    s_args.bc.bce = p.face[5];
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                s_cur_q = q;
                s_cur_s = s;
            }
            __threadfence();   // every thread reads after the acquire
        }
        if (s_q < kPasses) {
            const BatchItem& it = A.items[s_q][s_s];
            const int local = s_g - A.pass_off[s_q] - A.start[s_q][s_s];
            const double* in = it.in_user ? A.ptrs[s_s].f : A.ws + it.ws_off;
            double* out = it.out_user ? A.ptrs[s_s].f : A.ws + it.ws_off;
            // one tile body for the contiguous (x) and strided (y, z) passes
            // a per-thread copy of the descriptor: read from shared memory by
            // reference, the tile body's loads of it spill registers
            const PassArgs a = s_args;
            const LineTables<double> tbl = s_tb;
            line_pass_tile<double, double, double, kContigRuntime, kRadixAll>(
                in, out, a, tbl, it.buf_elems, local % it.ntx, local / it.ntx, smem_raw,
                s_q == 0 || s_q == kPasses - 1);
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();   // release the tile's writes with the counter
                atomicAdd(A.done + (long long)s_s * kPasses + s_q, 1);
            }
        } else {
            fixup_problem(A.fix[s_s], A.ptrs[s_s].f);
        }
        __syncthreads();
        if (threadIdx.x == 0) ++s_g;
    }
}

}  // namespace
}  // namespace chz

using namespace chz;

// The problems of one pass that a register-resident kernel takes, grouped
// by (length, kinds): one launch each.
struct FastGroup {
    std::vector<int> probs;   // member problems
    int kind = 0, kind2 = -1;
    chz::LineTables<double> tb{};
    chz::BatchMember* members_d = nullptr;
    int* start_d = nullptr;
    int count = 0;
    int ntiles = 0;
};

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
    int target[kPasses] = {};            // tile size (values per tile) of each pass
    float tuned_ms[kPasses] = {};        // its measured time (0: not tuned)
    int plan_variant[kPasses] = {};      // radix schedule chosen for each pass
    int* counters = nullptr;             // count * kPasses pass counters + the queue head
    int* owner = nullptr;                // problem of every pass tile, by queue index
    int grid = 0;                        // CTAs of the persistent launch
    size_t smem_all = 0;                 // its dynamic shared memory
    bool periodic = false;               // some problem has a periodic axis
    int mode = 0;                        // 0: one persistent launch; 1: launches per pass
    float mode_ms[2] = {};               // measured solve time of each form (0: not timed)
    // launches per pass: the register-resident groups, then one launch of the
    // generic kernel over the problems no group takes (the leftovers)
    std::vector<FastGroup> groups[kPasses];
    BatchItem* left_items_d[kPasses] = {};
    int* left_start_d[kPasses] = {};
    int* left_prob_d[kPasses] = {};
    int left_count[kPasses] = {};
    int left_tiles[kPasses] = {};
    size_t left_smem[kPasses] = {};
    // The launches of the per-pass form ("units": the groups of pass q, then
    // its leftover launch) run as a graph of branches: a unit waits only for
    // the units of pass q - 1 that hold one of its problems (deps), so
    // independent launches run at once.
    std::vector<std::vector<int>> deps[kPasses];
    std::vector<cudaEvent_t> done[kPasses];
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> join;      // one per branch stream: its last work, joined into the caller's stream
    cudaEvent_t fork = nullptr;
};

namespace {

void free_plan(chz_batch_plan* p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (int q = 0; q < kPasses; ++q) {
        if (p->items_d[q]) cudaFree(p->items_d[q]);
        if (p->start_d[q]) cudaFree(p->start_d[q]);
        for (FastGroup& g : p->groups[q]) {
            if (g.members_d) cudaFree(g.members_d);
            if (g.start_d) cudaFree(g.start_d);
        }
        if (p->left_items_d[q]) cudaFree(p->left_items_d[q]);
        if (p->left_start_d[q]) cudaFree(p->left_start_d[q]);
        if (p->left_prob_d[q]) cudaFree(p->left_prob_d[q]);
        for (cudaEvent_t ev : p->done[q]) cudaEventDestroy(ev);
    }
    for (cudaStream_t st : p->branch) cudaStreamDestroy(st);
    for (cudaEvent_t ev : p->join) cudaEventDestroy(ev);
    if (p->fork) cudaEventDestroy(p->fork);
    if (p->fix_d) cudaFree(p->fix_d);
    if (p->ptrs_d) cudaFree(p->ptrs_d);
    if (p->ptrs_h) cudaFreeHost(p->ptrs_h);
    if (p->ws) cudaFree(p->ws);
    if (p->counters) cudaFree(p->counters);
    if (p->owner) cudaFree(p->owner);
    if (p->graph_stream) cudaStreamDestroy(p->graph_stream);
    delete p;
}

// One problem's pass before the tile shape is chosen.
struct PassTemplate {
    BatchItem it;     // everything but the tile-dependent fields
    int n;            // line length
    int nv;           // planes of lines
};

constexpr size_t kBatchMaxSmem = 110 * 1024;  // two CTAs per SM
constexpr int kDefaultTarget = 4096;            // values per tile without tuning
constexpr int kTargets[] = {1024, 2048, 4096, 8192, 16384};
std::atomic<int> g_autotune{1};
std::atomic<int> g_force_variant{-1};   // >= 0: every pass uses this radix schedule (untuned)
std::atomic<int> g_force_mode{-1};      // >= 0: every plan uses this launch form (untimed)

// Fills the tile-dependent fields of pass q for every problem at tile size
// `target` (values per tile); returns the launch's tile count and shared memory.
void materialise(const std::vector<PassTemplate>& tp, bool contig, int target, std::vector<BatchItem>& items,
                 std::vector<int>& start, int* tiles, size_t* smem) {
    const int count = (int)tp.size();
    items.resize(count);
    start.assign(count + 1, 0);
    *smem = 0;
    for (int i = 0; i < count; ++i) {
        const LineGeom g = line_geometry_target(tp[i].n, 1, contig, target, kBatchMaxSmem);
        BatchItem& it = items[i];
        it = tp[i].it;
        it.a.PR = g.PR;
        it.a.log2W = g.log2W;
        it.buf_elems = (int)g.buf_elems;
        it.ntx = (it.a.nu + g.W - 1) / g.W;
        start[i + 1] = start[i] + it.ntx * tp[i].nv;
        *smem = std::max(*smem, g.smem_bytes);
    }
    *tiles = start[count];
}

// Radix schedules the autotuner chooses from, for a complex length M:
// 0: radix 8s first, then 4 or 2, then the odd primes (factor_radices);
// 1: the same radices in reverse order (odd primes first);
// 2: radix 4s (and a 2) in place of the 8s, then the odd primes.
constexpr int kPlanVariants = 3;

bool radix_variant(int M, int variant, RadixPlan* rp) {
    RadixPlan base;
    if (factor_radices(M, &base) != 0) return false;
    if (variant == 0) {
        *rp = base;
        return true;
    }
    int r[16];
    int n = 0;
    if (variant == 1) {
        for (int st = base.nst - 1; st >= 0; --st) r[n++] = base.radix(st);
    } else {
        int m = M, e2 = 0;
        while (m % 2 == 0) { m /= 2; ++e2; }
        while (e2 >= 2) { r[n++] = 4; e2 -= 2; }
        if (e2 == 1) r[n++] = 2;
        for (int st = 0; st < base.nst; ++st)
            if (base.radix(st) % 2) r[n++] = base.radix(st);
    }
    if (n > kMaxStages || n > 16) return false;
    unsigned long long code = 0;
    for (int i = 0; i < n; ++i) code |= (unsigned long long)r[i] << (4 * i);
    rp->nst = n;
    rp->code = code;
    return true;
}

// Gives every problem of a pass its length's radix schedule `variant`
// (problems whose length has no such schedule keep theirs).
void apply_variant(std::vector<BatchItem>& items, int variant) {
    for (BatchItem& it : items) {
        RadixPlan rp;
        if (radix_variant(it.tb.M, variant, &rp)) it.tb.rp = rp;
    }
}

cudaError_t raise_smem(bool contig, size_t bytes);

// Pass q of every problem on the generic kernel (one launch).
cudaError_t launch_pass(chz_batch_plan* p, int q, cudaStream_t s) {
    if (p->tiles[q] == 0) return cudaSuccess;
    if (p->contig[q])
        batch_pass<true><<<p->tiles[q], kThreads, p->smem[q], s>>>(p->items_d[q], p->start_d[q], p->count,
                                                                   p->ptrs_d, p->ws, nullptr);
    else
        batch_pass<false><<<p->tiles[q], kThreads, p->smem[q], s>>>(p->items_d[q], p->start_d[q], p->count,
                                                                    p->ptrs_d, p->ws, nullptr);
    return cudaGetLastError();
}

// Unit u of pass q in the per-pass form: register-resident group u, or (u ==
// the number of groups) the generic kernel over the leftovers.
cudaError_t launch_unit(chz_batch_plan* p, int q, int u, cudaStream_t s) {
    if (u < (int)p->groups[q].size()) {
        const FastGroup& g = p->groups[q][u];
        FastBatchArgs A{g.members_d, g.start_d, g.count, g.ntiles, p->ptrs_d, p->ws};
        return (cudaError_t)launch_fast_batch(p->contig[q], g.kind, g.kind2, A, g.tb, s);
    }
    if (p->left_count[q] == 0 || p->left_tiles[q] == 0) return cudaSuccess;
    if (p->contig[q])
        batch_pass<true><<<p->left_tiles[q], kThreads, p->left_smem[q], s>>>(
            p->left_items_d[q], p->left_start_d[q], p->left_count[q], p->ptrs_d, p->ws, p->left_prob_d[q]);
    else
        batch_pass<false><<<p->left_tiles[q], kThreads, p->left_smem[q], s>>>(
            p->left_items_d[q], p->left_start_d[q], p->left_count[q], p->ptrs_d, p->ws, p->left_prob_d[q]);
    return cudaGetLastError();
}

int units_of(const chz_batch_plan* p, int q) {
    return (int)p->groups[q].size() + ((p->left_count[q] > 0 && p->left_tiles[q] > 0) ? 1 : 0);
}

constexpr int kBranches = 16;   // side streams of the per-pass form

// The per-pass form's dependencies: unit u of pass q waits for the units of
// pass q - 1 that hold one of its problems; plus the branch streams and one
// event per unit.
cudaError_t build_branches(chz_batch_plan* p) {
    std::vector<int> unit_of[kPasses];
    for (int q = 0; q < kPasses; ++q) {
        unit_of[q].assign(p->count, -1);
        // members of each group, read back from the host-side grouping
        for (int u = 0; u < (int)p->groups[q].size(); ++u)
            for (int i : p->groups[q][u].probs) unit_of[q][i] = u;
        for (int i = 0; i < p->count; ++i)
            if (unit_of[q][i] < 0) unit_of[q][i] = (int)p->groups[q].size();   // the leftover unit
    }
    for (int q = 0; q < kPasses; ++q) {
        const int nu = units_of(p, q);
        p->deps[q].assign(nu, {});
        if (q > 0) {
            std::vector<std::vector<char>> seen(nu, std::vector<char>(units_of(p, q - 1) + 1, 0));
            for (int i = 0; i < p->count; ++i) {
                const int u = unit_of[q][i], d = unit_of[q - 1][i];
                if (u < nu && d < units_of(p, q - 1) && !seen[u][d]) {
                    seen[u][d] = 1;
                    p->deps[q][u].push_back(d);
                }
            }
        }
        p->done[q].assign(nu, nullptr);
        for (int u = 0; u < nu; ++u) {
            const cudaError_t e = cudaEventCreateWithFlags(&p->done[q][u], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    cudaError_t e = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
    for (int k = 0; k < kBranches && e == cudaSuccess; ++k) {
        cudaStream_t st = nullptr;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e == cudaSuccess) p->branch.push_back(st);
        cudaEvent_t ev = nullptr;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) p->join.push_back(ev);
    }
    return e;
}

// The five passes of the per-pass form on the branch streams, forked from and
// joined back into `s`.
cudaError_t launch_passes_grouped(chz_batch_plan* p, cudaStream_t s) {
    cudaError_t e = cudaEventRecord(p->fork, s);
    int k = 0;
    for (int q = 0; q < kPasses && e == cudaSuccess; ++q) {
        for (int u = 0; u < units_of(p, q) && e == cudaSuccess; ++u) {
            cudaStream_t st = p->branch[(k++) % p->branch.size()];
            if (q == 0) e = cudaStreamWaitEvent(st, p->fork, 0);
            for (int d : p->deps[q][u])
                if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->done[q - 1][d], 0);
            if (e == cudaSuccess) e = launch_unit(p, q, u, st);
            if (e == cudaSuccess) e = cudaEventRecord(p->done[q][u], st);
        }
    }
    // every branch stream that took work joins back into s (a captured
    // graph's forks must all be joined)
    const int used = std::min<int>(k, (int)p->branch.size());
    for (int b = 0; b < used && e == cudaSuccess; ++b) {
        e = cudaEventRecord(p->join[b], p->branch[b]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, p->join[b], 0);
    }
    return e;
}

// Splits pass q into register-resident groups (problems whose line length has
// a register plan, by (length, kinds)) and the leftovers, and uploads both.
cudaError_t build_groups(chz_batch_plan* p, int q, const std::vector<PassTemplate>& tp,
                         const std::vector<BatchItem>& items) {
    std::map<std::tuple<int, int, int>, std::vector<int>> by_key;
    std::vector<int> left;
    for (int i = 0; i < p->count; ++i) {
        const int n = tp[i].n;
        const int M = n / 2;
        const bool fast = (n % 2 == 0) && fast_path_supported(M, true) && fast_lines_per_tile(M) > 0;
        if (fast) by_key[std::make_tuple(M, items[i].a.kind, items[i].a.kind2)].push_back(i);
        else left.push_back(i);
    }
    cudaError_t e = cudaSuccess;
    for (const auto& kv : by_key) {
        const int M = std::get<0>(kv.first);
        const int W = fast_lines_per_tile(M);
        FastGroup g;
        g.probs = kv.second;
        g.kind = std::get<1>(kv.first);
        g.kind2 = std::get<2>(kv.first);
        g.tb = items[kv.second[0]].tb;
        std::vector<BatchMember> mem;
        std::vector<int> start(1, 0);
        for (int i : kv.second) {
            BatchMember m{};
            m.a = items[i].a;
            m.prob = i;
            m.ntx = (m.a.nu + W - 1) / W;
            m.in_user = items[i].in_user;
            m.out_user = items[i].out_user;
            m.ws_off = items[i].ws_off;
            mem.push_back(m);
            start.push_back(start.back() + m.ntx * tp[i].nv);
        }
        g.count = (int)mem.size();
        g.ntiles = start.back();
        if (e == cudaSuccess) e = cudaMalloc(&g.members_d, sizeof(BatchMember) * mem.size());
        if (e == cudaSuccess) e = cudaMalloc(&g.start_d, sizeof(int) * start.size());
        if (e == cudaSuccess)
            e = cudaMemcpy(g.members_d, mem.data(), sizeof(BatchMember) * mem.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(g.start_d, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice);
        p->groups[q].push_back(g);   // freed with the plan even when an upload failed
    }
    p->left_count[q] = (int)left.size();
    if (left.empty() || e != cudaSuccess) return e;
    std::vector<BatchItem> li;
    std::vector<int> ls(1, 0);
    size_t smem = 0;
    for (int i : left) {
        li.push_back(items[i]);
        ls.push_back(ls.back() + items[i].ntx * tp[i].nv);
        const LineGeom geo = line_geometry_target(tp[i].n, 1, p->contig[q], p->target[q], kBatchMaxSmem);
        smem = std::max(smem, geo.smem_bytes);
    }
    p->left_tiles[q] = ls.back();
    p->left_smem[q] = smem;
    e = cudaMalloc(&p->left_items_d[q], sizeof(BatchItem) * li.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->left_start_d[q], sizeof(int) * ls.size());
    if (e == cudaSuccess) e = cudaMalloc(&p->left_prob_d[q], sizeof(int) * left.size());
    if (e == cudaSuccess) e = cudaMemcpy(p->left_items_d[q], li.data(), sizeof(BatchItem) * li.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->left_start_d[q], ls.data(), sizeof(int) * ls.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(p->left_prob_d[q], left.data(), sizeof(int) * left.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = raise_smem(p->contig[q], smem);
    return e;
}

// The dynamic shared-memory limit is an attribute of the kernel, shared by
// every plan in the process: it only ever rises, so a plan created later with
// smaller tiles never invalidates an earlier plan's launches.
cudaError_t raise_smem(bool contig, size_t bytes) {
    static std::mutex mu;
    static size_t set[2] = {0, 0};
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set[contig ? 1 : 0];
    if (bytes <= cur) return cudaSuccess;
    const cudaError_t e = contig
        ? cudaFuncSetAttribute(batch_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes)
        : cudaFuncSetAttribute(batch_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

cudaError_t upload_pass(chz_batch_plan* p, int q, const std::vector<BatchItem>& items, const std::vector<int>& start) {
    cudaError_t e = cudaMemcpy(p->items_d[q], items.data(), sizeof(BatchItem) * p->count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(p->start_d[q], start.data(), sizeof(int) * (p->count + 1), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = raise_smem(p->contig[q], p->smem[q]);
    return e;
}

// Autotuner: for every pass, times one launch over all problems at each tile
// size of kTargets (after a warm-up launch, CUDA events on a private stream)
// and keeps the fastest.  The launches run on scratch stand-ins for the
// problems' arrays (zeros; the Neumann data read as zeros), so the caller's
// data is not needed.  Returns false when the scratch cannot be allocated (the
// default tile size then stays).
bool autotune(chz_batch_plan* p, const std::vector<PassTemplate>* tmpl, const std::vector<long long>& ws_off,
              size_t face_max) {
    double* fake = nullptr;
    double* zface = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool ok = cudaMalloc(&fake, p->ws_bytes) == cudaSuccess &&
              cudaMalloc(&zface, face_max * sizeof(double)) == cudaSuccess &&
              cudaMemset(fake, 0, p->ws_bytes) == cudaSuccess &&
              cudaMemset(zface, 0, face_max * sizeof(double)) == cudaSuccess &&
              cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
    if (ok && !p->graph_stream) ok = cudaStreamCreateWithFlags(&p->graph_stream, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) {
        for (int i = 0; i < p->count; ++i) {
            p->ptrs_h[i].f = fake + ws_off[i];
            for (int k = 0; k < 6; ++k) p->ptrs_h[i].face[k] = zface;
        }
        ok = cudaMemcpy(p->ptrs_d, p->ptrs_h, sizeof(ProbPtrs) * p->count, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    cudaStream_t s = p->graph_stream;
    for (int q = 0; ok && q < kPasses; ++q) {
        float best = 0.0f;
        int best_t = kDefaultTarget;
        for (int target : kTargets) {
            std::vector<BatchItem> items;
            std::vector<int> start;
            materialise(tmpl[q], p->contig[q], target, items, start, &p->tiles[q], &p->smem[q]);
            float ms = 0.0f;
            ok = upload_pass(p, q, items, start) == cudaSuccess && launch_pass(p, q, s) == cudaSuccess &&
                 cudaEventRecord(e0, s) == cudaSuccess && launch_pass(p, q, s) == cudaSuccess &&
                 launch_pass(p, q, s) == cudaSuccess && cudaEventRecord(e1, s) == cudaSuccess &&
                 cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
            if (!ok) break;
            if (best == 0.0f || ms < best) {
                best = ms;
                best_t = target;
            }
        }
        p->target[q] = best_t;
        p->tuned_ms[q] = best / 2.0f;
        // then the radix schedule at that tile size
        int best_v = 0;
        for (int v = 1; ok && v < kPlanVariants; ++v) {
            std::vector<BatchItem> items;
            std::vector<int> start;
            materialise(tmpl[q], p->contig[q], best_t, items, start, &p->tiles[q], &p->smem[q]);
            apply_variant(items, v);
            float ms = 0.0f;
            ok = upload_pass(p, q, items, start) == cudaSuccess && launch_pass(p, q, s) == cudaSuccess &&
                 cudaEventRecord(e0, s) == cudaSuccess && launch_pass(p, q, s) == cudaSuccess &&
                 launch_pass(p, q, s) == cudaSuccess && cudaEventRecord(e1, s) == cudaSuccess &&
                 cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
            if (ok && ms < best) {
                best = ms;
                best_v = v;
            }
        }
        p->plan_variant[q] = best_v;
        p->tuned_ms[q] = best / 2.0f;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (fake) cudaFree(fake);
    if (zface) cudaFree(zface);
    cudaGetLastError();
    return ok;
}

// Dynamic shared memory and grid of the persistent launch (the largest tile
// buffer of the five passes; as many CTAs as fit the device).
cudaError_t prepare_persistent(chz_batch_plan* p) {
    size_t smem = 0;
    for (int q = 0; q < kPasses; ++q) smem = std::max(smem, p->smem[q]);
    static std::mutex mu;
    static size_t set = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (smem > set) {
            const cudaError_t e =
                cudaFuncSetAttribute(batch_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            set = smem;
        }
    }
    int cps = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cps, batch_persistent, kThreads, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
    if (e != cudaSuccess) return e;
    if (cps < 1) return cudaErrorInvalidConfiguration;
    int total = p->count;
    for (int q = 0; q < kPasses; ++q) total += p->tiles[q];
    p->grid = std::min(total, cps * sms);
    p->smem_all = smem;
    return cudaSuccess;
}

// Records one batched solve on `s`.  Persistent form: the reset of the pass
// counters and the queue head, then the persistent launch.  Per-pass form: the
// five pass launches, then the periodic planes.
int enqueue(chz_batch_plan* p, cudaStream_t s) {
    if (p->mode == 1) {
        {
            const cudaError_t e = launch_passes_grouped(p, s);
            if (e != cudaSuccess) return cuda_fail((int)e, "batched pass");
        }
        if (p->periodic) {
            batch_fixup<<<p->count, kThreads, 0, s>>>(p->fix_d, p->ptrs_d);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail((int)e, "batched periodic planes");
        }
        return CHZ_SUCCESS;
    }
    PersistArgs A{};
    int off = 0;
    for (int q = 0; q < kPasses; ++q) {
        A.items[q] = p->items_d[q];
        A.start[q] = p->start_d[q];
        A.pass_off[q] = off;
        off += p->tiles[q];
    }
    A.pass_off[kPasses] = off;
    A.pass_off[kPasses + 1] = off + p->count;
    A.owner = p->owner;
    A.fix = p->fix_d;
    A.ptrs = p->ptrs_d;
    A.ws = p->ws;
    A.count = p->count;
    A.done = p->counters;
    A.next = p->counters + (size_t)p->count * kPasses;
    A.flags = tma::device_flags();
    A.wait_limit = tma::wait_limit();
    if (!A.flags) return cuda_fail((int)cudaGetLastError(), "batch wait flags");
    cudaError_t e = cudaMemsetAsync(p->counters, 0, sizeof(int) * ((size_t)p->count * kPasses + 1), s);
    if (e != cudaSuccess) return cuda_fail((int)e, "batch counters");
    batch_persistent<<<p->grid, kThreads, p->smem_all, s>>>(A);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail((int)e, "batched solve");
    return CHZ_SUCCESS;
}

// Times a whole solve in each launch form (one warm-up, then two solves timed
// with CUDA events on a private stream) on scratch stand-ins for the problems'
// arrays, as the autotuner does, and keeps the faster form.  Which one wins
// depends on the batch: the persistent launch lets one problem's next pass
// start while other problems still run the previous one, at the price of the
// queue's bookkeeping and one tile body for every pass.  Returns false when
// the scratch cannot be allocated or a launch fails (the persistent form then
// stays).
bool choose_launch_mode(chz_batch_plan* p, const std::vector<long long>& ws_off, size_t face_max) {
    double* fake = nullptr;
    double* zface = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool ok = cudaMalloc(&fake, p->ws_bytes) == cudaSuccess &&
              cudaMalloc(&zface, face_max * sizeof(double)) == cudaSuccess &&
              cudaMemset(fake, 0, p->ws_bytes) == cudaSuccess &&
              cudaMemset(zface, 0, face_max * sizeof(double)) == cudaSuccess &&
              cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
    if (ok && !p->graph_stream) ok = cudaStreamCreateWithFlags(&p->graph_stream, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) {
        for (int i = 0; i < p->count; ++i) {
            p->ptrs_h[i].f = fake + ws_off[i];
            for (int k = 0; k < 6; ++k) p->ptrs_h[i].face[k] = zface;
        }
        ok = cudaMemcpy(p->ptrs_d, p->ptrs_h, sizeof(ProbPtrs) * p->count, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    cudaStream_t s = p->graph_stream;
    for (int m = 0; ok && m < 2; ++m) {
        p->mode = m;
        float ms = 0.0f;
        ok = enqueue(p, s) == CHZ_SUCCESS && cudaEventRecord(e0, s) == cudaSuccess && enqueue(p, s) == CHZ_SUCCESS &&
             enqueue(p, s) == CHZ_SUCCESS && cudaEventRecord(e1, s) == cudaSuccess &&
             cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
        p->mode_ms[m] = ok ? ms / 2.0f : 0.0f;
    }
    // a persistent wait that ran out voids the timing (the flag stays for
    // chz_stream_status to report)
    if (ok) ok = (chz_debug_flags(0) & kFlagBatchWait) == 0;
    p->mode = (ok && p->mode_ms[1] < p->mode_ms[0]) ? 1 : 0;
    if (!ok) p->mode_ms[0] = p->mode_ms[1] = 0.0f;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (fake) cudaFree(fake);
    if (zface) cudaFree(zface);
    g_last_error[0] = 0;
    cudaGetLastError();
    return ok;
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
    // descriptors of every pass (tile shape chosen below)
    std::vector<PassTemplate> tmpl[kPasses];
    for (int q = 0; q < kPasses; ++q) {
        tmpl[q].resize(count);
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
        auto fill = [&](int q, int kind, int kind2, const DeviceLineTables& t, int n, int u0, int u1, int v0, int v1,
                        long long isu, long long isv, long long isl, int ld0, int ld1, long long osu, long long osv,
                        long long osl, int st0, int st1, int in_user, int out_user) {
            PassTemplate& tp = tmpl[q][i];
            BatchItem& it = tp.it;
            std::memset(&it, 0, sizeof(it));
            PassArgs& a = it.a;
            a.kind = kind; a.kind2 = kind2;
            a.u0 = u0; a.nu = u1 - u0 + 1; a.v0 = v0;
            a.in_su = isu; a.in_sv = isv; a.in_sl = isl; a.ld_lo = ld0; a.ld_hi = ld1;
            a.out_su = osu; a.out_sv = osv; a.out_sl = osl; a.st_lo = st0; a.st_hi = st1;
            a.scale = 1.0; a.use_scale = 0;
            it.tb.twM = static_cast<const double2*>(t.twM);
            it.tb.twN = static_cast<const double2*>(t.twN);
            it.tb.tw4N = static_cast<const double2*>(t.tw4N);
            it.tb.inv4sin = static_cast<const double*>(t.inv4sin);
            it.tb.N = t.N; it.tb.M = t.M; it.tb.rp = t.rp;
            it.in_user = in_user; it.out_user = out_user;
            it.ws_off = ws_off[i];
            tp.n = n;
            tp.nv = v1 - v0 + 1;
        };
        fill(0, X.kf, -1, tx, nx, Y.s, Y.e, Z.s, Z.e, fy, fz, 1, X.s, X.e, wy, wz, 1, X.sp0, X.sp1, 1, 0);
        {
            BcArgs& bc = tmpl[0][i].it.a.bc;
            tmpl[0][i].it.a.has_bc = 1;
            bc.xbc = X.bc; bc.ybc = Y.bc; bc.zbc = Z.bc;
            bc.xs = X.s; bc.xe = X.e; bc.ys = Y.s; bc.ye = Y.e; bc.zs = Z.s; bc.ze = Z.e;
            bc.nx = nx; bc.ny = ny; bc.nz = nz;
            bc.dx = X.d; bc.dy = Y.d; bc.dz = Z.d;
            bc.dx2 = X.d2; bc.dy2 = Y.d2; bc.dz2 = Z.d2;
        }
        fill(1, Y.kf, -1, ty, ny, X.sp0, X.sp1, Z.s, Z.e, 1, wz, wy, Y.s, Y.e, 1, wz, wy, Y.sp0, Y.sp1, 0, 0);
        fill(2, Z.kf, Z.ki, tz, nz, X.sp0, X.sp1, Y.sp0, Y.sp1, 1, wy, wz, Z.s, Z.e, 1, wy, wz, Z.s, Z.e, 0, 0);
        {
            PassArgs& a = tmpl[2][i].it.a;
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
        fill(3, Y.ki, -1, ty, ny, X.sp0, X.sp1, Z.s, Z.e, 1, wz, wy, Y.sp0, Y.sp1, 1, wz, wy, Y.s, Y.e, 0, 0);
        fill(4, X.ki, -1, tx, nx, Y.s, Y.e, Z.s, Z.e, wy, wz, 1, X.sp0, X.sp1, fy, fz, 1, X.s, X.e, 0, 1);
        tmpl[4][i].it.a.scale = solver_scale(X, Y, Z);
        tmpl[4][i].it.a.use_scale = 1;
    }
    std::vector<BatchItem> items[kPasses];
    std::vector<int> start[kPasses];
    for (int q = 0; q < kPasses; ++q) {
        p->target[q] = kDefaultTarget;
        materialise(tmpl[q], p->contig[q], p->target[q], items[q], start[q], &p->tiles[q], &p->smem[q]);
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
    size_t face_max = 1;
    for (int i = 0; i < count; ++i) {
        const size_t nx = dims[3 * i], ny = dims[3 * i + 1], nz = dims[3 * i + 2];
        face_max = std::max(face_max, std::max((ny + 1) * (nz + 1), std::max((nx + 1) * (nz + 1), (nx + 1) * (ny + 1))));
        p->periodic = p->periodic || p->fix_h[i].px || p->fix_h[i].py || p->fix_h[i].pz;
    }
    const bool tune = g_autotune.load(std::memory_order_relaxed) != 0;
    if (e == cudaSuccess && tune) {
        if (!autotune(p, tmpl, ws_off, face_max)) {
            for (int q = 0; q < kPasses; ++q) {
                p->target[q] = kDefaultTarget;
                p->tuned_ms[q] = 0.0f;
                p->plan_variant[q] = 0;
            }
        }
    }
    const int forced = g_force_variant.load(std::memory_order_relaxed);
    for (int q = 0; q < kPasses && e == cudaSuccess; ++q) {
        if (forced >= 0) p->plan_variant[q] = forced;
        materialise(tmpl[q], p->contig[q], p->target[q], items[q], start[q], &p->tiles[q], &p->smem[q]);
        apply_variant(items[q], p->plan_variant[q]);
        e = upload_pass(p, q, items[q], start[q]);
        if (e == cudaSuccess) e = build_groups(p, q, tmpl[q], items[q]);
    }
    if (e == cudaSuccess) e = build_branches(p);
    if (e == cudaSuccess) e = cudaMalloc(&p->counters, sizeof(int) * ((size_t)count * kPasses + 1));
    if (e == cudaSuccess) {
        // the problem of every pass tile, in queue order
        std::vector<int> owner;
        for (int q = 0; q < kPasses; ++q)
            for (int i = 0; i < count; ++i)
                owner.insert(owner.end(), (size_t)(start[q][i + 1] - start[q][i]), i);
        e = cudaMalloc(&p->owner, sizeof(int) * std::max<size_t>(owner.size(), 1));
        if (e == cudaSuccess && !owner.empty())
            e = cudaMemcpy(p->owner, owner.data(), sizeof(int) * owner.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = prepare_persistent(p);
    if (e == cudaSuccess) {
        const int fm = g_force_mode.load(std::memory_order_relaxed);
        if (fm >= 0) p->mode = fm;
        else if (tune) choose_launch_mode(p, ws_off, face_max);
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

int chz_batch_set_autotune(int on) { return g_autotune.exchange(on ? 1 : 0); }

int chz_batch_set_radix_schedule(int variant) {
    if (variant < -1 || variant >= kPlanVariants) return -2;
    return g_force_variant.exchange(variant);
}

int chz_batch_plan_tiles(const chz_batch_plan* plan, int* targets, float* ms) {
    if (!plan) return fail(CHZ_ERROR_INVALID_VALUE, "NULL plan");
    for (int q = 0; q < kPasses; ++q) {
        if (targets) targets[q] = plan->target[q];
        if (ms) ms[q] = plan->tuned_ms[q];
    }
    return CHZ_SUCCESS;
}

int chz_batch_set_launch_mode(int mode) {
    if (mode < -1 || mode > 1) return -2;
    return g_force_mode.exchange(mode);
}

int chz_batch_plan_launch(const chz_batch_plan* plan, int* mode, float* ms) {
    if (!plan) return fail(CHZ_ERROR_INVALID_VALUE, "NULL plan");
    if (mode) *mode = plan->mode;
    if (ms) {
        ms[0] = plan->mode_ms[0];
        ms[1] = plan->mode_ms[1];
    }
    return CHZ_SUCCESS;
}

int chz_batch_plan_radix(const chz_batch_plan* plan, int* variants) {
    if (!plan || !variants) return fail(CHZ_ERROR_INVALID_VALUE, "NULL argument");
    for (int q = 0; q < kPasses; ++q) variants[q] = plan->plan_variant[q];
    return CHZ_SUCCESS;
}

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
        // capture the solve (the counter reset and the persistent launch, or
        // the per-pass launches) once, on a private stream (the legacy default
        // stream cannot be captured); the graph replays on any stream
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
    count_launch();
    trace_end(s);
    if (e != cudaSuccess) return cuda_fail((int)e, "graph launch");
    return CHZ_SUCCESS;
}

int chz_batch_plan_kernels(const chz_batch_plan* plan) {
    if (!plan) return fail(CHZ_ERROR_INVALID_VALUE, "NULL plan");
    if (plan->mode == 0) return 1;
    int n = plan->periodic ? 1 : 0;
    for (int q = 0; q < kPasses; ++q) n += units_of(plan, q);
    return n;
}

int chz_batch_plan_destroy(chz_batch_plan* plan) {
    if (plan) {
        cudaDeviceSynchronize();
        free_plan(plan);
    }
    return CHZ_SUCCESS;
}

}  // extern "C"
