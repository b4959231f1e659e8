// Instantiation of the CTA-wide contiguous pass for N = 256 (M = 128), FP64,
// storing its outputs from registers: every kind with a tensor input
// (16-byte-aligned rows), the solver's forward kinds with a span input (f).
#include <cstring>

#include "chz_xtma_launch.cuh"

namespace chz {
namespace xtma {
int launch_direct_m128(bool span, int kind, const double* in, double* out, const PassArgs& a,
                       const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label) {
    return span ? launch_kinds<128, kLdSpan, kStDirect>(kind, in, out, a, tb, nv, stream, label)
                : launch_kinds<128, kLdTensor, kStDirect>(kind, in, out, a, tb, nv, stream, label);
}
}  // namespace xtma
}  // namespace chz
