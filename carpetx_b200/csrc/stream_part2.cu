// Streaming-kernel instantiations, part 2 of kStreamParts: the kernels whose
// group (2 x pair index of stream_pairs.h + 1 for a cell-centred z) is 2
// modulo kStreamParts; split only to compile in parallel.
#include "stream_kernel.cuh"
#include "stream_pairs.h"

namespace cxb {
namespace stream {

KernelFn kernel_part2(int group) {
  switch (group) {
#define CXB_PAIR_CASE(I, V, C, KVI, KCI)                                       \
  case 2 * I:                                                                  \
    if constexpr ((2 * I) % kStreamParts == 2)                                \
      return stream_kernel<V, C, 0>;                                           \
    break;                                                                     \
  case 2 * I + 1:                                                              \
    if constexpr ((2 * I + 1) % kStreamParts == 2)                            \
      return stream_kernel<V, C, 1>;                                           \
    break;
    CXB_STREAM_PAIRS(CXB_PAIR_CASE)
#undef CXB_PAIR_CASE
  default:
    break;
  }
  return nullptr;
}

} // namespace stream
} // namespace cxb
