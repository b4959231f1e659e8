// Instantiation of the register-resident line kernels for N = 112 (M = 56), FP64, single and batched.
#include "chz_fast_launch.cuh"

namespace chz {
namespace fast {
template int launch_fast_kind<double, double, double, 56>(bool, int, int, const void*, void*, const PassArgs&,
                                                           const LineTables<double>&, int, cudaStream_t,
                                                           const char*);
template int launch_fast_batch_kind<56>(bool, int, int, const FastBatchArgs&, const LineTables<double>&,
                                         cudaStream_t);
}  // namespace fast
}  // namespace chz
