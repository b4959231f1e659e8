// Instantiation of the register-resident line kernels for N = 40 (M = 20), FP64.
#include "chz_fast_launch.cuh"

namespace chz {
namespace fast {
template int launch_fast_kind<double, double, double, 20>(bool, int, int, const void*, void*, const PassArgs&,
                                                           const LineTables<double>&, int, cudaStream_t,
                                                           const char*);
}  // namespace fast
}  // namespace chz
