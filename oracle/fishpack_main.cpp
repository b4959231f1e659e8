// Test infrastructure: command-line driver around the reference's CPU solver.
//
// This program is the checker's CPU path and the timed CPU baseline, never the
// product. It links the reference's own wrapper `solver_3d`
// (cudahelmholtz/hw3crt_wrapper.cpp:5-33) and the FISHPACK archive it wraps
// (cudahelmholtz/libfishpack.a, linked and run only). The build recipe is
// oracle/Makefile; the binary lands in oracle/_ref/.
//
// Protocol (all little-endian):
//   input file : int32[8]  {magic 0x43485a31, NX, NY, NZ, xbc, ybc, zbc, present}
//                float64[7] {xs, xf, ys, yf, zs, zf, lambda}
//                float64[(NX+1)(NY+1)(NZ+1)]  f, [z][y][x]
//                then, for bit b = 0..5 of `present` (bcl, bcr, bcb, bct, bcf, bce),
//                the face array of that bit when set: x faces hold (NY+1)(NZ+1)
//                values [z][y], y faces (NX+1)(NZ+1) [z][x], z faces (NX+1)(NY+1) [y][x]
//                (the layout of testgpurectangle.cu:46-57).
//   output file: float64[(NX+1)(NY+1)(NZ+1)]  u (f after the in-place solve)
//   stdout     : "hw3crt_seconds <best> <median> <repeats>"
//
// usage: hw3crt_run <in.bin> <out.bin> [repeats]
//        hw3crt_run <in.bin> <out.bin> pertrb
//   The second form calls hw3crt_ (declared by the reference's
//   hw3crt_wrapper.h) directly, once, with the wrapper's arguments and a
//   workspace twice the wrapper's size, and also prints
//   "pertrb <value> ierror <code>": the wrapper computes PERTRB (the constant
//   FISHPACK subtracts from F when lambda = 0 and no boundary pins the
//   solution) but does not return it.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>

#include "hw3crt_wrapper.h"

static bool read_all(FILE* fp, void* dst, size_t bytes) {
    return fread(dst, 1, bytes, fp) == bytes;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s in.bin out.bin [repeats]\n", argv[0]);
        return 2;
    }
    const bool want_pertrb = argc > 3 && std::strcmp(argv[3], "pertrb") == 0;
    int repeats = (argc > 3 && !want_pertrb) ? atoi(argv[3]) : 1;
    if (repeats < 1) repeats = 1;

    FILE* fp = fopen(argv[1], "rb");
    if (!fp) { perror("open input"); return 2; }
    int32_t hdr[8];
    double dom[7];
    if (!read_all(fp, hdr, sizeof(hdr)) || !read_all(fp, dom, sizeof(dom))) {
        fprintf(stderr, "short header\n");
        return 2;
    }
    if (hdr[0] != 0x43485a31) { fprintf(stderr, "bad magic\n"); return 2; }
    const int nx = hdr[1], ny = hdr[2], nz = hdr[3];
    const int xbc = hdr[4], ybc = hdr[5], zbc = hdr[6];
    const int present = hdr[7];
    if (nx < 2 || ny < 2 || nz < 2) { fprintf(stderr, "bad sizes\n"); return 2; }
    const size_t npts = size_t(nx + 1) * (ny + 1) * (nz + 1);
    std::vector<double> f0(npts);
    if (!read_all(fp, f0.data(), npts * sizeof(double))) { fprintf(stderr, "short f\n"); return 2; }

    const size_t face_len[6] = {
        size_t(ny + 1) * (nz + 1), size_t(ny + 1) * (nz + 1),
        size_t(nx + 1) * (nz + 1), size_t(nx + 1) * (nz + 1),
        size_t(nx + 1) * (ny + 1), size_t(nx + 1) * (ny + 1)};
    std::vector<double> faces[6];
    double* fp_face[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int b = 0; b < 6; ++b) {
        if (present & (1 << b)) {
            faces[b].resize(face_len[b]);
            if (!read_all(fp, faces[b].data(), face_len[b] * sizeof(double))) {
                fprintf(stderr, "short face %d\n", b);
                return 2;
            }
            fp_face[b] = faces[b].data();
        }
    }
    fclose(fp);

    std::vector<double> f(npts);
    if (want_pertrb) {
        std::memcpy(f.data(), f0.data(), npts * sizeof(double));
        int l = nx, m = ny, n = nz, lb = xbc, mb = ybc, nb = zbc, ldimf = nx + 1, mdimf = ny + 1;
        double xs = dom[0], xf = dom[1], ys = dom[2], yf = dom[3], zs = dom[4], zf = dom[5], lam = dom[6];
        const int wsize = 2 * (30 + l + m + 5 * n + std::max(std::max(l, m), n) + 7 * ((l + 1) / 2 + (m + 1) / 2));
        std::vector<double> w(wsize);
        double pertrb = 0.0;
        int ierror = -1;
        hw3crt_(&xs, &xf, &l, &lb, fp_face[0], fp_face[1], &ys, &yf, &m, &mb, fp_face[2], fp_face[3],
                &zs, &zf, &n, &nb, fp_face[4], fp_face[5], &lam, &ldimf, &mdimf, f.data(), &pertrb, &ierror,
                w.data());
        printf("pertrb %.17g ierror %d\n", pertrb, ierror);
        FILE* fo = fopen(argv[2], "wb");
        if (!fo) { perror("open output"); return 2; }
        if (fwrite(f.data(), sizeof(double), npts, fo) != npts) { fprintf(stderr, "short write\n"); return 2; }
        fclose(fo);
        return 0;
    }
    std::vector<double> times;
    for (int r = 0; r < repeats; ++r) {
        std::memcpy(f.data(), f0.data(), npts * sizeof(double));
        auto t0 = std::chrono::steady_clock::now();
        solver_3d(dom[0], dom[1], nx, xbc, fp_face[0], fp_face[1],
                  dom[2], dom[3], ny, ybc, fp_face[2], fp_face[3],
                  dom[4], dom[5], nz, zbc, fp_face[4], fp_face[5],
                  dom[6], f.data());
        auto t1 = std::chrono::steady_clock::now();
        times.push_back(std::chrono::duration<double>(t1 - t0).count());
    }
    std::vector<double> sorted = times;
    std::sort(sorted.begin(), sorted.end());
    printf("hw3crt_seconds %.9f %.9f %d\n", sorted.front(), sorted[sorted.size() / 2], repeats);

    FILE* fo = fopen(argv[2], "wb");
    if (!fo) { perror("open output"); return 2; }
    if (fwrite(f.data(), sizeof(double), npts, fo) != npts) { fprintf(stderr, "short write\n"); return 2; }
    fclose(fo);
    return 0;
}
