// Streaming-kernel instantiations, part 1 of kStreamParts (the pairs of
// stream_pairs.h whose index is 1 modulo kStreamParts; split only to compile
// in parallel).
#include "stream_kernel.cuh"
#include "stream_pairs.h"

namespace cxb {
namespace stream {

KernelFn kernel_part1(int pair) {
  switch (pair) {
#define CXB_PAIR_CASE(I, V, C, KVI, KCI)                                       \
  case I:                                                                      \
    if constexpr (I % kStreamParts == 1)                                      \
      return stream_kernel<V, C>;                                              \
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
