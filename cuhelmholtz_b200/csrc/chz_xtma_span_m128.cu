// Instantiation of the contiguous pass for N = 256 (M = 128), FP64, with the
// input moved as one bulk span (rows of an 8-byte-aligned array: the solver's
// f) and the output by tensor boxes: the solver's forward kinds.
#include <cstring>

#include "chz_xtma_launch.cuh"

namespace chz {
namespace xtma {
int launch_span_tensor_m128(int kind, const double* in, double* out, const PassArgs& a,
                            const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label) {
    // the forward DST-III measured slower here than on the cp.async register
    // kernel (256x192x320, codes (2,4,3): 0.125 vs 0.106 ms), so it stays there
    if (kind == kDST3) return -1;
    return launch_kinds<128, kLdSpan, kStTensor>(kind, in, out, a, tb, nv, stream, label);
}
}  // namespace xtma
}  // namespace chz
