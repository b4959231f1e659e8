// Instantiation of the warp-local contiguous pass for N = 256 (M = 128), FP64,
// with the input moved by tensor boxes (16-byte-aligned rows: do_transform arrays, the solver's work array), every kind.
#include <cstring>

#include "chz_xtma_launch.cuh"

namespace chz {
namespace xtma {
int launch_w_tensor_m128(int kind, const double* in, double* out, const PassArgs& a, const LineTables<double>& tb,
                       int nv, cudaStream_t stream, const char* label) {
    return launch_w_kinds<128, kLdTensor>(kind, in, out, a, tb, nv, stream, label);
}
}  // namespace xtma
}  // namespace chz
