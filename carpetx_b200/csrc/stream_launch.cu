// Host side of the streaming kernel: pair lookup, tiling, launches.
#include <atomic>

#include "cx_async.cuh"

#include "stream_kernel.cuh"
#include "stream_pairs.h"
#include "stream_tuned.h"

namespace cxb {
namespace stream {
KernelFn kernel_part0(int group, bool small_cta, int sched);
KernelFn kernel_part1(int group, bool small_cta, int sched);
KernelFn kernel_part2(int group, bool small_cta, int sched);
KernelFn kernel_part3(int group, bool small_cta, int sched);
KernelFn kernel_part4(int group, bool small_cta, int sched);
KernelFn kernel_part5(int group, bool small_cta, int sched);
KernelFn kernel_part6(int group, bool small_cta, int sched);
KernelFn kernel_part7(int group, bool small_cta, int sched);
int str_set_wait_limit_part0(long long);
int str_set_wait_limit_part1(long long);
int str_set_wait_limit_part2(long long);
int str_set_wait_limit_part3(long long);
int str_set_wait_limit_part4(long long);
int str_set_wait_limit_part5(long long);
int str_set_wait_limit_part6(long long);
int str_set_wait_limit_part7(long long);
int str_timeout_part0();
int str_timeout_part1();
int str_timeout_part2();
int str_timeout_part3();
int str_timeout_part4();
int str_timeout_part5();
int str_timeout_part6();
int str_timeout_part7();

namespace {
// Per device (cache_device()) and schedule: dynamic shared memory allowed
// per group (the attribute applies per device), SM count, persistent grid
// per group.
std::atomic<bool> g_attr_set[kMaxDevices][kStrGroups][2];
std::atomic<int> g_sms[kMaxDevices];
std::atomic<int> g_grid[kMaxDevices][kStrGroups][2];
// Settings of cx_debug_set_stream_schedule per instantiation: schedule
// (-1: none) and z-chunk cap (0: none).
std::atomic<int> g_sched_set[kStrKinds];
std::atomic<int> g_maxz_set[kStrKinds];
struct SetInit {
  SetInit() {
    for (int k = 0; k < kStrKinds; ++k) {
      g_sched_set[k].store(-1);
      g_maxz_set[k].store(0);
    }
  }
} g_set_init;

// Per instantiation: whether its 256-thread kernel has schedule 1, and the
// spread (RHI - RLO) of its z kind.
constexpr bool kHasSched1[kStrKinds] = {
#define CXB_HS(I, V, C, KVI, KCI)                                              \
  has_sched1<V, C, 0>(), has_sched1<V, C, 1>(), has_sched1<V, C, 2>(),         \
      has_sched1<V, C, 3>(), has_sched1<V, C, 4>(), has_sched1<V, C, 5>(),     \
      has_sched1<V, C, 6>(), has_sched1<V, C, 7>(),
    CXB_STREAM_PAIRS(CXB_HS)
#undef CXB_HS
};
constexpr int kZSpread[kStrKinds] = {
#define CXB_ZS(I, V, C, KVI, KCI)                                              \
  V::RHI - V::RLO, C::RHI - C::RLO, V::RHI - V::RLO, C::RHI - C::RLO,          \
      V::RHI - V::RLO, C::RHI - C::RLO, V::RHI - V::RLO, C::RHI - C::RLO,
    CXB_STREAM_PAIRS(CXB_ZS)
#undef CXB_ZS
};

// Threads and dynamic shared memory of a level group's CTA size.
int threads_of(int group) { return group >= kStrKinds ? small::NTS : big::NTS; }
size_t smem_of(int group) {
  return group >= kStrKinds ? sizeof(small::Shared) : sizeof(big::Shared);
}

// Kernel of a level group (instantiation + kStrKinds for the 128-thread
// variant) and schedule; the first lookup on a device allows its dynamic
// shared memory, which may exceed the 48 KB default.
KernelFn kernel_for(int group, int sched) {
  if (group < 0 || group >= kStrGroups)
    return nullptr;
  static KernelFn (*const parts[kStreamParts])(int, bool, int) = {
      kernel_part0, kernel_part1, kernel_part2, kernel_part3,
      kernel_part4, kernel_part5, kernel_part6, kernel_part7};
  const int kind = group % kStrKinds;
  const int sc = group >= kStrKinds ? 0 : sched;
  KernelFn k = parts[kind % kStreamParts](kind, group >= kStrKinds, sc);
  const int dev = cache_device();
  if (k && (dev < 0 || !g_attr_set[dev][group][sc].load())) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(group));
    if (dev >= 0)
      g_attr_set[dev][group][sc].store(true);
  }
  return k;
}

int sms() {
  const int dev = cache_device();
  if (dev >= 0 && g_sms[dev].load())
    return g_sms[dev].load();
  int d = 0, n = 0;
  cudaGetDevice(&d);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
  if (dev >= 0)
    g_sms[dev].store(n);
  return n;
}
} // namespace
} // namespace stream

int stream_sched(int group) {
  using namespace stream;
  if (group < 0 || group >= kStrKinds)
    return 0; // the 128-thread variant (or none)
  if (!kHasSched1[group])
    return 0;
  const int set = g_sched_set[group].load();
  if (set >= 0)
    return set;
  if (kStreamTuned[group].sched >= 0)
    return kStreamTuned[group].sched;
  // untuned: three CTAs per SM for z spreads of 4 (the order-3 conservative
  // and order-3/4 polynomial cell-centred z kinds), measured faster on the
  // mixed 512-box level; two elsewhere
  return kZSpread[group] == 4 ? 1 : 0;
}

int stream_maxz(int kind) {
  using namespace stream;
  if (kind < 0 || kind >= kStrKinds)
    return 128;
  const int set = g_maxz_set[kind].load();
  if (set > 0)
    return set;
  return kStreamTuned[kind].maxz > 0 ? kStreamTuned[kind].maxz : 128;
}

int stream_set_schedule(int kind, int sched, int maxz) {
  using namespace stream;
  if (kind < -1 || kind >= kStrKinds || sched < -1 || sched > 1 || maxz < 0 || maxz > 128 ||
      (maxz > 0 && (maxz < 16 || (maxz & 1))))
    return -1;
  for (int k = kind < 0 ? 0 : kind; k < (kind < 0 ? kStrKinds : kind + 1); ++k) {
    g_sched_set[k].store(sched);
    g_maxz_set[k].store(maxz);
  }
  return 0;
}

int stream_set_wait_limit(long long cycles) {
  using namespace stream;
  static int (*const parts[kStreamParts])(long long) = {
      str_set_wait_limit_part0, str_set_wait_limit_part1, str_set_wait_limit_part2,
      str_set_wait_limit_part3, str_set_wait_limit_part4, str_set_wait_limit_part5,
      str_set_wait_limit_part6, str_set_wait_limit_part7};
  const long long v = cycles >= 0 ? cycles : kWaitCycles;
  for (auto f : parts)
    if (f(v) != 0)
      return -1;
  return 0;
}

int stream_take_timeout() {
  using namespace stream;
  static int (*const parts[kStreamParts])() = {str_timeout_part0, str_timeout_part1,
                                               str_timeout_part2, str_timeout_part3,
                                               str_timeout_part4, str_timeout_part5,
                                               str_timeout_part6, str_timeout_part7};
  int any = 0;
  for (auto f : parts) {
    const int v = f();
    if (v < 0)
      return -1;
    any |= v;
  }
  return any;
}

int stream_pair_of(int kx, int ky, int kz) {
  const int k[3] = {kx, ky, kz};
  int v = -1, c = -1;
  for (int d = 0; d < 3; ++d) {
    if (kind_info(k[d]).cent == CC)
      c = k[d];
    else
      v = k[d];
  }
  static const int pv[kStreamPairs] = {
#define CXB_PV(I, V, C, KVI, KCI) KVI,
      CXB_STREAM_PAIRS(CXB_PV)
#undef CXB_PV
  };
  static const int pc[kStreamPairs] = {
#define CXB_PC(I, V, C, KVI, KCI) KCI,
      CXB_STREAM_PAIRS(CXB_PC)
#undef CXB_PC
  };
  for (int i = 0; i < kStreamPairs; ++i)
    if ((v < 0 || pv[i] == v) && (c < 0 || pc[i] == c))
      return i;
  return -1;
}

int stream_group_of(int kx, int ky, int kz) {
  const int pair = stream_pair_of(kx, ky, kz);
  const int cm = (kind_info(kx).cent == CC ? 4 : 0) | (kind_info(ky).cent == CC ? 2 : 0) |
                 (kind_info(kz).cent == CC ? 1 : 0);
  return pair < 0 ? -1 : kStreamParts * pair + cm;
}

void stream_tiling(BoxDesc &b, int min_items) {
  using namespace stream;
  for (int d = 0; d < 3; ++d)
    b.tbase[d] = b.rlo[d] & ~1;
  // x chunks: the whole width up to kStrMaxWidth, else near-equal even chunks
  constexpr int WFMAX = kStrMaxWidth, PRMAX = kStrUnitRows;
  const int Wt = b.rhi[0] - b.tbase[0] + 1;
  if (Wt <= WFMAX) {
    b.xcw = Wt;
    b.ntile[0] = 1;
  } else {
    const int n = (Wt + WFMAX - 3) / (WFMAX - 2);
    int w = (Wt + n - 1) / n;
    w += w & 1;
    b.xcw = w;
    b.ntile[0] = (Wt + w - 1) / w;
  }
  b.npr = (b.rhi[1] - b.tbase[1]) / kStrFineYPerUnit + 1;
  // boxes with at most kStrSmallUnits column units per x chunk run on the
  // 128-thread variant (one item of 256 unit slots instead of 512)
  b.scta = b.npr * b.xcw <= kStrSmallUnits ? 1 : 0;
  const int nu = b.scta ? small::NU : big::NU;
  b.upi = nu < PRMAX * b.xcw ? nu : PRMAX * b.xcw;
  b.ntile[1] = (b.npr * b.xcw + b.upi - 1) / b.upi;
  // fine z per item: whole columns up to the instantiation's cap (tuned, 128
  // by default), else near-equal even chunks of at most the cap (the z halo
  // and the pipeline start cost extra planes per chunk); shorter chunks
  // (down to 16) when the box alone must fill min_items CTAs
  const int E = b.rhi[2] - b.tbase[2] + 1;
  const int64_t xy_items = (int64_t)b.ntile[0] * b.ntile[1] * b.ncomp;
  int maxz = stream_maxz(stream_group_of(b.kind[0], b.kind[1], b.kind[2]));
  while (maxz > 16 && xy_items * ((E + maxz - 1) / maxz) < min_items)
    maxz /= 2;
  const int nch = (E + maxz - 1) / maxz;
  int zc = (E + nch - 1) / nch;
  zc += zc & 1;
  b.zchunk = zc;
  b.ntile[2] = (E + zc - 1) / zc;
}

int stream_level_grid(int group, int sched) {
  using namespace stream;
  const int sc = group >= kStrKinds ? 0 : (sched ? 1 : 0);
  KernelFn k = kernel_for(group, sc);
  if (!k)
    return 0;
  const int dev = cache_device();
  if (dev >= 0 && g_grid[dev][group][sc].load())
    return g_grid[dev][group][sc].load();
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads_of(group), smem_of(group));
  const int grid = sms() * (per_sm > 0 ? per_sm : 1);
  if (dev >= 0)
    g_grid[dev][group][sc].store(grid);
  return grid;
}

cudaError_t launch_stream_box(const BoxDesc &b, cudaStream_t s) {
  using namespace stream;
  const int64_t n64 = (int64_t)b.ntile[0] * b.ntile[1] * b.ntile[2] * b.ncomp;
  if (n64 <= 0)
    return cudaSuccess;
  if (n64 > INT32_MAX)
    return cudaErrorInvalidValue;
  const int kind = stream_group_of(b.kind[0], b.kind[1], b.kind[2]);
  if (kind < 0)
    return cudaErrorInvalidValue;
  const int group = kind + (b.scta ? kStrKinds : 0);
  const int sched = stream_sched(group);
  KernelFn k = kernel_for(group, sched);
  if (!k)
    return cudaErrorInvalidValue;
  const int n = (int)n64;
  const int cap = stream_level_grid(group, sched);
  k<<<n < cap ? n : cap, threads_of(group), smem_of(group), s>>>(b, nullptr, nullptr, n, nullptr);
  return cudaGetLastError();
}

cudaError_t launch_stream_level(int group, int sched, const BoxDesc *d_boxes,
                                const TileRef *d_items, int nitems, int grid, int *d_counter,
                                cudaStream_t s, bool after_level) {
  using namespace stream;
  if (nitems <= 0)
    return cudaSuccess;
  KernelFn k = kernel_for(group, sched);
  if (!k)
    return cudaErrorInvalidValue;
  BoxDesc unused{};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid < nitems ? grid : nitems);
  cfg.blockDim = dim3(threads_of(group));
  cfg.dynamicSmemBytes = smem_of(group);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = after_level ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, unused, d_boxes, d_items, nitems, d_counter);
}

} // namespace cxb
