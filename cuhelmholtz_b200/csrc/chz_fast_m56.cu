// Instantiation of the register-resident line kernels for N = 112 (M = 56), FP64.
#include "chz_fast_launch.cuh"

namespace chz {
namespace fast {
template int launch_fast_kind<double, double, double, 56>(bool, int, int, const void*, void*, const PassArgs&,
                                                           const LineTables<double>&, int, cudaStream_t,
                                                           const char*);
}  // namespace fast
}  // namespace chz
