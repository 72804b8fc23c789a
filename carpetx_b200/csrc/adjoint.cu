// Host side of the adjoint of the separable linear prolongations: kernel
// lookup per stencil pair and centring, tiling, launches.  The kernel is in
// adjoint_kernel.cuh; its instantiations are spread over adjoint_part*.cu.
#include <atomic>

#include "adjoint_kernel.cuh"

namespace cxb {
using namespace adj;
namespace {

constexpr int kAdjGroups = kStreamParts * kStreamPairs; // pair x centring

// Kernel and shared-memory size of group 8 pair + centring.
AdjFn adj_kernel(int group, size_t *smem) {
  static AdjFn (*const parts[kStreamParts])(int, size_t *) = {
      adj_kernel_part0, adj_kernel_part1, adj_kernel_part2, adj_kernel_part3,
      adj_kernel_part4, adj_kernel_part5, adj_kernel_part6, adj_kernel_part7};
  if (group < 0 || group >= kAdjGroups)
    return nullptr;
  return parts[group % kStreamParts](group / kStreamParts, smem);
}

template <class V, class C> int adj_upt_of() {
  if constexpr (std::is_same_v<C, CcMinmod>)
    return 0;
  else
    return AdjPair<V, C>::UPT;
}

// Coarse columns per thread of a pair's kernel.
int adj_upt(int pair) {
  switch (pair) {
#define CXB_ADJ_UPT(I, V, C, KVI, KCI)                                         \
  case I:                                                                      \
    return adj_upt_of<V, C>();
    CXB_STREAM_PAIRS(CXB_ADJ_UPT)
#undef CXB_ADJ_UPT
  default:
    break;
  }
  return 2;
}

// Per device (cache_device()): dynamic shared memory allowed and persistent
// grid per group (0: not yet set up on that device).
std::atomic<int> g_adj_grid[kMaxDevices][kAdjGroups];

// Kernel of a group, its dynamic shared memory allowed and its persistent
// grid (SMs x resident CTAs) recorded on first use on the current device.
AdjFn adj_ready(int group, size_t *smem, int *grid) {
  AdjFn k = adj_kernel(group, smem);
  if (!k)
    return nullptr;
  const int dev = cache_device();
  if (dev >= 0 && g_adj_grid[dev][group].load()) {
    *grid = g_adj_grid[dev][group].load();
    return k;
  }
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem) !=
      cudaSuccess)
    return nullptr;
  int per_sm = 0, d = 0, sms = 0;
  cudaGetDevice(&d);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, *smem);
  *grid = sms * (per_sm > 0 ? per_sm : 1);
  if (dev >= 0)
    g_adj_grid[dev][group].store(*grid);
  return k;
}

} // namespace

int adjoint_set_wait_limit(long long cycles) {
  static int (*const parts[kStreamParts])(long long) = {
      adj_set_wait_limit_part0, adj_set_wait_limit_part1, adj_set_wait_limit_part2,
      adj_set_wait_limit_part3, adj_set_wait_limit_part4, adj_set_wait_limit_part5,
      adj_set_wait_limit_part6, adj_set_wait_limit_part7};
  const long long v = cycles >= 0 ? cycles : kWaitCycles;
  for (auto f : parts)
    if (f(v) != 0)
      return -1;
  return 0;
}

int adjoint_take_timeout() {
  static int (*const parts[kStreamParts])() = {adj_timeout_part0, adj_timeout_part1,
                                               adj_timeout_part2, adj_timeout_part3,
                                               adj_timeout_part4, adj_timeout_part5,
                                               adj_timeout_part6, adj_timeout_part7};
  int any = 0;
  for (auto f : parts) {
    const int v = f();
    if (v < 0)
      return -1;
    any |= v;
  }
  return any;
}

int adjoint_pair_of(const BoxDesc &b) {
  for (int d = 0; d < 3; ++d)
    if (b.kind[d] == K_CC_MINMOD1 || b.kind[d] == K_CC_ENO2)
      return -1;
  return stream_pair_of(b.kind[0], b.kind[1], b.kind[2]);
}

int adjoint_group_of(const BoxDesc &b) {
  const int pair = adjoint_pair_of(b);
  const int cm = (kind_info(b.kind[0]).cent == CC ? 4 : 0) |
                 (kind_info(b.kind[1]).cent == CC ? 2 : 0) |
                 (kind_info(b.kind[2]).cent == CC ? 1 : 0);
  return pair < 0 ? -1 : kStreamParts * pair + cm;
}

void adjoint_tiling(BoxDesc &b, int min_items) {
  const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
  const int nu = NT * adj_upt(adjoint_pair_of(b)); // the pair kernel's columns per item
  b.ant[0] = (b.cnx + TMAX - 1) / TMAX;
  b.at[0] = (b.cnx + b.ant[0] - 1) / b.ant[0];
  const int tymax = tile_ty(b.at[0], nu);
  b.ant[1] = (b.cny + tymax - 1) / tymax;
  b.at[1] = (b.cny + b.ant[1] - 1) / b.ant[1];
  // coarse z per item: up to 48 (an item streams 2 (RHI - RLO) fine planes
  // more than it owns), shorter (down to 8) until the box fills min_items
  int maxz = 48;
  const int64_t xy = (int64_t)b.ant[0] * b.ant[1] * b.ncomp;
  while (maxz > 8 && xy * ((cnz + maxz - 1) / maxz) < min_items)
    maxz /= 2;
  const int n = (cnz + maxz - 1) / maxz;
  b.at[2] = (cnz + n - 1) / n;
  b.ant[2] = (cnz + b.at[2] - 1) / b.at[2];
}

int adjoint_level_grid(int group) {
  size_t smem = 0;
  int grid = 0;
  return adj_ready(group, &smem, &grid) ? grid : 0;
}

cudaError_t launch_prolong_adjoint_box(const BoxDesc &b0, int per_group, double *crse_bar,
                                       cudaStream_t s) {
  (void)per_group; // linear operators: per-group and per-variable agree
  if (b0.ncomp <= 0 || b0.cnp <= 0)
    return cudaSuccess;
  const int group = adjoint_group_of(b0);
  size_t smem = 0;
  int grid = 0;
  AdjFn k = adj_ready(group, &smem, &grid);
  if (!k)
    return cudaErrorInvalidValue;
  BoxDesc b = b0;
  b.cbar = crse_bar;
  adjoint_tiling(b, grid);
  const int64_t n64 = (int64_t)b.ant[0] * b.ant[1] * b.ant[2] * b.ncomp;
  if (n64 > INT32_MAX)
    return cudaErrorInvalidValue;
  const int n = (int)n64;
  k<<<n < grid ? n : grid, NT, smem, s>>>(b, nullptr, nullptr, n, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_level(int group, const BoxDesc *d_boxes, const TileRef *d_items,
                                 int nitems, int grid, int *d_counter, cudaStream_t s,
                                 bool after_level) {
  if (nitems <= 0)
    return cudaSuccess;
  size_t smem = 0;
  int unused_grid = 0;
  AdjFn k = adj_ready(group, &smem, &unused_grid);
  if (!k)
    return cudaErrorInvalidValue;
  BoxDesc unused{};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid < nitems ? grid : nitems);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = after_level ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, unused, d_boxes, d_items, nitems, d_counter);
}

} // namespace cxb
