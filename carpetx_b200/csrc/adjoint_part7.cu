// Adjoint-kernel instantiations of centring 7 ((cx << 2) | (cy << 1) | cz),
// one per linear stencil pair of stream_pairs.h; split only to compile in
// parallel.  This file's copies of the timeout flag and the wait limit are
// read and set here.
#include "adjoint_kernel.cuh"

namespace cxb {
namespace adj {

AdjFn adj_kernel_part7(int pair, size_t *smem) {
  switch (pair) {
#define CXB_ADJ_CASE(I, V, C, KVI, KCI)                                        \
  case I:                                                                      \
    return adj_fn<V, C, 7>(smem);
    CXB_STREAM_PAIRS(CXB_ADJ_CASE)
#undef CXB_ADJ_CASE
  default:
    break;
  }
  return nullptr;
}

int adj_set_wait_limit_part7(long long cycles) {
  return cudaMemcpyToSymbol(g_adj_wait_limit, &cycles, sizeof cycles) == cudaSuccess ? 0 : -1;
}

int adj_timeout_part7() {
  int v = 0, zero = 0;
  if (cudaMemcpyFromSymbol(&v, g_adj_timeout, sizeof v) != cudaSuccess)
    return -1;
  if (v)
    cudaMemcpyToSymbol(g_adj_timeout, &zero, sizeof zero);
  return v;
}

} // namespace adj
} // namespace cxb
