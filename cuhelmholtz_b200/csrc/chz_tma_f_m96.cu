// Instantiation of the TMA-pipelined strided pass for N = 192 (M = 96), FP32.
#include "chz_tma_launch.cuh"

namespace chz {
namespace tma {
template int launch_tma_kind<float, 96>(int, int, const void*, void*, const PassArgs&, const LineTables<float>&, int,
                                        cudaStream_t, const char*);
}  // namespace tma
}  // namespace chz
