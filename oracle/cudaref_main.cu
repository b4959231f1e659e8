// Test infrastructure: command-line driver around the reference's own GPU path.
//
// Links, unchanged and compiled from the reference sources where they lie, the
// reference's cudasymmfft (do_transform and its pre/post kernels over cuFFT,
// cudasymmfft/funcinterface.cu:25-334) and its solver cuda_helmholtz_solver
// (cudahelmholtz/cuda_helmholtz_solver.cu:33-380), with cuFFT from the CUDA
// toolkit (linked and called only) and oracle/cut_transpose.cu standing in for
// the absent libcuTranspose.  It produces the reference's outputs for the
// checker and times the reference GPU path as a reported figure.  Never part
// of the product; the build recipe is oracle/Makefile, the binary lands in
// oracle/_ref/cudaref_run.
//
// Protocol (little-endian):
//   cudaref_run transform <in.bin> <out.bin> [repeats]
//     in : any number of cases, each
//            int32[8]  {0x43485a54, NX, NY, NZ, x_kind, y_kind, z_kind, inplace}
//            float64[(NZ+2)(NY+2)(NX+2)]  d_data, [z][y][x]
//     out: per case the array do_transform leaves as its result: d_data for an
//          in-place call (d_out = NULL), d_out otherwise
//     stdout: per case "cudaref_seconds <best> <median> <repeats>" (wall time of
//          the synchronous call, input re-uploaded before every repeat)
//   cudaref_run solve <in.bin> <out.bin> [repeats]
//     in : the FISHPACK runner's input format (oracle/fishpack_main.cpp)
//     out: u = f after the in-place cuda_helmholtz_solver call
//     stdout: "cudaref_seconds <best> <median> <repeats>"
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "cuda_helmholtz_solver.h"
#include "funcinterface.h"

namespace {

constexpr int32_t kTransformMagic = 0x43485a54;
constexpr int32_t kSolveMagic = 0x43485a31;

bool read_all(FILE* fp, void* dst, size_t bytes) { return fread(dst, 1, bytes, fp) == bytes; }

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        exit(3);
    }
}

void report(std::vector<double> t) {
    std::sort(t.begin(), t.end());
    printf("cudaref_seconds %.9f %.9f %d\n", t.front(), t[t.size() / 2], (int)t.size());
    fflush(stdout);
}

int run_transform(const char* in, const char* out, int repeats) {
    FILE* fi = fopen(in, "rb");
    if (!fi) { perror("open input"); return 2; }
    FILE* fo = fopen(out, "wb");
    if (!fo) { perror("open output"); return 2; }
    int32_t hdr[8];
    while (read_all(fi, hdr, sizeof(hdr))) {
        if (hdr[0] != kTransformMagic) { fprintf(stderr, "bad magic\n"); return 2; }
        const int nx = hdr[1], ny = hdr[2], nz = hdr[3];
        const int kx = hdr[4], ky = hdr[5], kz = hdr[6], inplace = hdr[7];
        if (nx < 4 || ny < 4 || nz < 4 || (nx | ny | nz) & 1 || kx < 0 || kx > 7 || ky < 0 ||
            ky > 7 || kz < 0 || kz > 7 || (inplace && !(nx == ny && ny == nz))) {
            fprintf(stderr, "bad case %d %d %d %d %d %d %d\n", nx, ny, nz, kx, ky, kz, inplace);
            return 2;
        }
        const size_t n = size_t(nx + 2) * (ny + 2) * (nz + 2);
        std::vector<double> h(n);
        if (!read_all(fi, h.data(), n * sizeof(double))) { fprintf(stderr, "short data\n"); return 2; }
        double *d = nullptr, *dout = nullptr;
        check(cudaMalloc(&d, n * sizeof(double)), "cudaMalloc");
        if (!inplace) {
            check(cudaMalloc(&dout, n * sizeof(double)), "cudaMalloc");
            check(cudaMemset(dout, 0, n * sizeof(double)), "cudaMemset");
        }
        std::vector<double> times;
        for (int r = 0; r < repeats; ++r) {
            check(cudaMemcpy(d, h.data(), n * sizeof(double), cudaMemcpyHostToDevice), "upload");
            check(cudaDeviceSynchronize(), "sync");
            auto t0 = std::chrono::steady_clock::now();
            do_transform(d, inplace ? nullptr : dout, nx, ny, nz, (transform_kind)kx,
                         (transform_kind)ky, (transform_kind)kz);
            check(cudaDeviceSynchronize(), "do_transform");
            auto t1 = std::chrono::steady_clock::now();
            times.push_back(std::chrono::duration<double>(t1 - t0).count());
        }
        check(cudaMemcpy(h.data(), inplace ? d : dout, n * sizeof(double), cudaMemcpyDeviceToHost),
              "download");
        cudaFree(d);
        if (dout) cudaFree(dout);
        if (fwrite(h.data(), sizeof(double), n, fo) != n) { fprintf(stderr, "short write\n"); return 2; }
        report(times);
    }
    fclose(fi);
    fclose(fo);
    return 0;
}

int run_solve(const char* in, const char* out, int repeats) {
    FILE* fp = fopen(in, "rb");
    if (!fp) { perror("open input"); return 2; }
    int32_t hdr[8];
    double dom[7];
    if (!read_all(fp, hdr, sizeof(hdr)) || !read_all(fp, dom, sizeof(dom))) {
        fprintf(stderr, "short header\n");
        return 2;
    }
    if (hdr[0] != kSolveMagic) { fprintf(stderr, "bad magic\n"); return 2; }
    const int nx = hdr[1], ny = hdr[2], nz = hdr[3];
    const int xbc = hdr[4], ybc = hdr[5], zbc = hdr[6], present = hdr[7];
    if (nx < 4 || ny < 4 || nz < 4 || (nx | ny | nz) & 1 || xbc < 0 || xbc > 4 || ybc < 0 ||
        ybc > 4 || zbc < 0 || zbc > 4) {
        fprintf(stderr, "bad case\n");
        return 2;
    }
    const size_t npts = size_t(nx + 1) * (ny + 1) * (nz + 1);
    std::vector<double> f(npts);
    if (!read_all(fp, f.data(), npts * sizeof(double))) { fprintf(stderr, "short f\n"); return 2; }
    const size_t face_len[6] = {size_t(ny + 1) * (nz + 1), size_t(ny + 1) * (nz + 1),
                                size_t(nx + 1) * (nz + 1), size_t(nx + 1) * (nz + 1),
                                size_t(nx + 1) * (ny + 1), size_t(nx + 1) * (ny + 1)};
    double* dface[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int b = 0; b < 6; ++b) {
        if (!(present & (1 << b))) continue;
        std::vector<double> face(face_len[b]);
        if (!read_all(fp, face.data(), face_len[b] * sizeof(double))) {
            fprintf(stderr, "short face %d\n", b);
            return 2;
        }
        check(cudaMalloc(&dface[b], face_len[b] * sizeof(double)), "cudaMalloc");
        check(cudaMemcpy(dface[b], face.data(), face_len[b] * sizeof(double), cudaMemcpyHostToDevice),
              "upload face");
    }
    fclose(fp);
    double* df = nullptr;
    check(cudaMalloc(&df, npts * sizeof(double)), "cudaMalloc");
    std::vector<double> times;
    for (int r = 0; r < repeats; ++r) {
        check(cudaMemcpy(df, f.data(), npts * sizeof(double), cudaMemcpyHostToDevice), "upload f");
        check(cudaDeviceSynchronize(), "sync");
        auto t0 = std::chrono::steady_clock::now();
        cuda_helmholtz_solver(dom[0], dom[1], nx, xbc, dface[0], dface[1], dom[2], dom[3], ny, ybc,
                              dface[2], dface[3], dom[4], dom[5], nz, zbc, dface[4], dface[5], dom[6],
                              df);
        check(cudaDeviceSynchronize(), "cuda_helmholtz_solver");
        auto t1 = std::chrono::steady_clock::now();
        times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    check(cudaMemcpy(f.data(), df, npts * sizeof(double), cudaMemcpyDeviceToHost), "download u");
    cudaFree(df);
    for (double* p : dface)
        if (p) cudaFree(p);
    FILE* fo = fopen(out, "wb");
    if (!fo) { perror("open output"); return 2; }
    if (fwrite(f.data(), sizeof(double), npts, fo) != npts) { fprintf(stderr, "short write\n"); return 2; }
    fclose(fo);
    report(times);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s transform|solve in.bin out.bin [repeats]\n", argv[0]);
        return 2;
    }
    int repeats = argc > 4 ? atoi(argv[4]) : 1;
    if (repeats < 1) repeats = 1;
    if (std::strcmp(argv[1], "transform") == 0) return run_transform(argv[2], argv[3], repeats);
    if (std::strcmp(argv[1], "solve") == 0) return run_solve(argv[2], argv[3], repeats);
    fprintf(stderr, "unknown mode %s\n", argv[1]);
    return 2;
}
