// Test infrastructure only: a project-written stand-in for libcuTranspose's
// cut_transpose3d, the one piece of the reference's GPU path that is neither
// vendored nor pinned.  It is linked into oracle/_ref/cudaref_run (the
// reference's own cudasymmfft + cuda_helmholtz_solver, built from the
// reference sources where they lie) and never into the product library.
//
// Signature: cudasymmfft/cutranspose.h:34-38.
// Semantics, read from the reference's six call sites
// (cudasymmfft/funcinterface.cu:120-122, 157-159, 192-194, 243-245, 287-289,
// 329-331): `size` lists the input's extents fastest-first, output dimension i
// is input dimension permutation[i] (so the output extents are
// size[permutation[i]]), output and input may alias (in place), and
// elements_per_thread is a tuning hint.  The permutation is exact: every
// element is copied, none is computed.
#include <cuda_runtime.h>
#include <cstdio>

extern "C" int cut_transpose3d(double* output, const double* input, const int* size,
                               const int* permutation, int elements_per_thread);

namespace {

__global__ void permute3d(double* __restrict__ out, const double* __restrict__ in,
                          long long s0, long long s1, long long s2,
                          int p0, int p1, int p2) {
    const long long sz[3] = {s0, s1, s2};
    const long long o0n = sz[p0], o1n = sz[p1];
    const long long total = s0 * s1 * s2;
    for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < total;
         o += (long long)gridDim.x * blockDim.x) {
        long long c[3];
        const long long o0 = o % o0n;
        const long long rest = o / o0n;
        const long long o1 = rest % o1n;
        const long long o2 = rest / o1n;
        c[p0] = o0;
        c[p1] = o1;
        c[p2] = o2;
        out[o] = in[c[0] + s0 * (c[1] + s1 * c[2])];
    }
}

}  // namespace

extern "C" int cut_transpose3d(double* output, const double* input, const int* size,
                               const int* permutation, int /*elements_per_thread*/) {
    const int p0 = permutation[0], p1 = permutation[1], p2 = permutation[2];
    if (p0 < 0 || p0 > 2 || p1 < 0 || p1 > 2 || p2 < 0 || p2 > 2 || p0 == p1 || p0 == p2 ||
        p1 == p2 || size[0] <= 0 || size[1] <= 0 || size[2] <= 0) {
        fprintf(stderr, "cut_transpose3d: bad size or permutation\n");
        return 1;
    }
    const long long total = (long long)size[0] * size[1] * size[2];
    // through a temporary, so that output == input (the in-place calls of the
    // cubic path) is a plain permutation too
    double* tmp = nullptr;
    if (cudaMalloc(&tmp, total * sizeof(double)) != cudaSuccess) {
        fprintf(stderr, "cut_transpose3d: cudaMalloc failed\n");
        return 2;
    }
    long long blocks = (total + 255) / 256;
    if (blocks > 148LL * 64) blocks = 148LL * 64;
    permute3d<<<(unsigned)blocks, 256>>>(tmp, input, size[0], size[1], size[2], p0, p1, p2);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpy(output, tmp, total * sizeof(double), cudaMemcpyDeviceToDevice);
    cudaFree(tmp);
    if (e != cudaSuccess) {
        fprintf(stderr, "cut_transpose3d: %s\n", cudaGetErrorString(e));
        return 3;
    }
    return 0;
}
