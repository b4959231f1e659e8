// Instantiation of the TMA-pipelined contiguous pass for N = 256 (M = 128), FP64.
#include <cstring>

#include "chz_xtma_launch.cuh"

namespace chz {
namespace xtma {
template int launch_xtma_kind<128>(int, int, const void*, void*, const PassArgs&, const LineTables<double>&, int,
                                   cudaStream_t, const char*);
}  // namespace xtma
}  // namespace chz
