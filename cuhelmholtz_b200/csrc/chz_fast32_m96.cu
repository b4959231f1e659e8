// Instantiation of the register-resident line kernels for N = 192 (M = 96), FP32
// transforms of the refinement solve (FP64 input or output on its x passes).
#include "chz_fast_launch.cuh"

namespace chz {
namespace fast {
template int launch_fast_kind<float, float, float, 96>(bool, int, int, const void*, void*, const PassArgs&,
                                                       const LineTables<float>&, int, cudaStream_t, const char*);
template int launch_fast_kind<float, double, float, 96>(bool, int, int, const void*, void*, const PassArgs&,
                                                        const LineTables<float>&, int, cudaStream_t, const char*);
template int launch_fast_kind<float, float, double, 96>(bool, int, int, const void*, void*, const PassArgs&,
                                                        const LineTables<float>&, int, cudaStream_t, const char*);
}  // namespace fast
}  // namespace chz
