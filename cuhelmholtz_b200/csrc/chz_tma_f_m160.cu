// Instantiation of the TMA-pipelined strided pass for N = 320 (M = 160), FP32.
#include "chz_tma_launch.cuh"

namespace chz {
namespace tma {
template int launch_tma_kind<float, 160>(int, int, const void*, void*, const PassArgs&, const LineTables<float>&, int,
                                        cudaStream_t, const char*);
}  // namespace tma
}  // namespace chz
