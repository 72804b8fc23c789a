// Streaming-kernel instantiations, part 6 of kStreamParts: the kernels whose
// centring (cx << 2 | cy << 1 | cz) is 6, one per stencil pair of
// stream_pairs.h and CTA size; split only to compile in parallel.
#include "stream_kernel.cuh"
#include "stream_pairs.h"

namespace cxb {
namespace stream {

KernelFn kernel_part6(int group, bool small_cta) {
  switch (group) {
#define CXB_PAIR_CASE(I, V, C, KVI, KCI)                                       \
  case kStreamParts * I + 6:                                                   \
    return small_cta ? small::stream_kernel<V, C, 6> : big::stream_kernel<V, C, 6>;
    CXB_STREAM_PAIRS(CXB_PAIR_CASE)
#undef CXB_PAIR_CASE
  default:
    break;
  }
  return nullptr;
}

} // namespace stream
} // namespace cxb
