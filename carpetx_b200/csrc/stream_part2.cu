// Streaming-kernel instantiations, part 2 of kStreamParts: the kernels whose
// centring (cx << 2 | cy << 1 | cz) is 2, one per stencil pair of
// stream_pairs.h and CTA size; split only to compile in parallel.  This
// file's copies of the timeout flag and the wait limit are read and set here.
#include "stream_kernel.cuh"
#include "stream_pairs.h"

namespace cxb {
namespace stream {

KernelFn kernel_part2(int group, bool small_cta, int sched) {
  switch (group) {
#define CXB_PAIR_CASE(I, V, C, KVI, KCI)                                       \
  case kStreamParts * I + 2:                                                   \
    return pick_kernel<V, C, 2>(small_cta, sched);
    CXB_STREAM_PAIRS(CXB_PAIR_CASE)
#undef CXB_PAIR_CASE
  default:
    break;
  }
  return nullptr;
}

int str_set_wait_limit_part2(long long cycles) {
  return cudaMemcpyToSymbol(g_str_wait_limit, &cycles, sizeof cycles) == cudaSuccess ? 0 : -1;
}

int str_timeout_part2() {
  int v = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&v, g_str_timeout, sizeof v) != cudaSuccess)
    return -1;
  if (v)
    cudaMemcpyToSymbol(g_str_timeout, &zero, sizeof zero);
  return v;
}

} // namespace stream
} // namespace cxb
