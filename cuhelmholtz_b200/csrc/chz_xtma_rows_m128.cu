// Instantiation of the contiguous pass for N = 256 (M = 128), FP64, with the
// input moved by tensor boxes and the output by bulk row stores (rows of an
// 8-byte-aligned array: the solver's f, scaled): the solver's inverse kinds.
#include <cstring>

#include "chz_xtma_launch.cuh"

namespace chz {
namespace xtma {
int launch_tensor_rows_m128(int kind, const double* in, double* out, const PassArgs& a,
                            const LineTables<double>& tb, int nv, cudaStream_t stream, const char* label) {
    return launch_kinds<128, kLdTensor, kStRows>(kind, in, out, a, tb, nv, stream, label);
}
}  // namespace xtma
}  // namespace chz
