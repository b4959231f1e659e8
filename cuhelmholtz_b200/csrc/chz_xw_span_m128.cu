// Instantiation of the warp-local contiguous pass for N = 256 (M = 128), FP64,
// with the input moved as one bulk span (rows of an 8-byte-aligned array: the solver's f), the solver's forward kinds.
#include <cstring>

#include "chz_xtma_launch.cuh"

namespace chz {
namespace xtma {
int launch_w_span_m128(int kind, const double* in, double* out, const PassArgs& a, const LineTables<double>& tb,
                       int nv, cudaStream_t stream, const char* label) {
    return launch_w_kinds<128, kLdSpan>(kind, in, out, a, tb, nv, stream, label);
}
}  // namespace xtma
}  // namespace chz
