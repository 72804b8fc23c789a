// Allocation-free level transfer: cx_level_execute_noalloc.
//
// For callers that cannot allocate device memory while they transfer a
// level: a host framework whose own allocator owns all device memory, or
// code that has already handed every byte of the GPU to such an allocator,
// so that a cudaMalloc would fail or would take memory the framework counts
// on.  The level plan (cx_level_plan_create) allocates its device work list
// with cudaMalloc; this entry point instead keeps the work list in one fixed
// device array, declared below, that every GPU loading the library holds
// until the process exits.
//
// The work list is built on the host in a static staging buffer under a
// mutex and copied into the device array on the caller's stream; then the
// same streaming kernels as cx_level_plan_execute run from it.  No
// cudaMalloc, cudaFree or allocating library call is made on the way.
#include <algorithm>
#include <mutex>

#include "../../include/carpetx_b200.h"
#include "cx_internal.h"

namespace cxb {
int validate_box_for_level(const cx_box_t &x, int per_group, BoxDesc *b, bool *empty);
bool box_uses_stream(cx_op_t op, int per_group);
int record_failure(int status, const char *what);
} // namespace cxb

using namespace cxb;

namespace {

constexpr int kMaxBoxes = CX_NOALLOC_MAX_BOXES;
constexpr int kMaxItems = CX_NOALLOC_MAX_ITEMS;

struct WorkList {
  BoxDesc boxes[kMaxBoxes];
  TileRef items[kMaxItems];
  int counters[kStrGroups]; // item counter per group, zeroed by every call
};

// The scratch: one work list per GPU (about 1.7 MB), shared by every call.
static __device__ __align__(256) WorkList g_scratch;

// Host staging of the work list (static, reused by every call under the lock).
WorkList g_stage;
std::mutex g_lock;

constexpr int kMaxDevices = 64;
WorkList *g_dev_scratch[kMaxDevices] = {}; // device address of g_scratch per device

// Device address of g_scratch for the current device, looked up once per
// device (with that device current) and cached; called with g_lock held, so
// two threads making their first call at once do not race on the cache.
int scratch_address(WorkList **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return record_failure(CX_ENODEVICE, "no current CUDA device");
  }
  if (!g_dev_scratch[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return record_failure(CX_ECUDA, "cudaGetSymbolAddress of the level scratch failed");
    }
    g_dev_scratch[dev] = static_cast<WorkList *>(p);
  }
  *out = g_dev_scratch[dev];
  return CX_OK;
}

int planes_of(const BoxDesc &b, int tz) {
  const int L = sep_rhi(b.kind[2]) - sep_rlo(b.kind[2]);
  const int z0 = b.tbase[2] + tz * b.zchunk;
  const int z1 = std::min(z0 + b.zchunk - 1, b.rhi[2]);
  return (z1 >> 1) - (z0 >> 1) + 1 + L;
}

} // namespace

extern "C" int cx_level_execute_noalloc(const cx_box_t *boxes, int nboxes, int per_group,
                                        cx_stream_t stream) {
  if (nboxes < 0 || (nboxes > 0 && !boxes))
    return record_failure(CX_EINVAL, "invalid argument");
  if (nboxes > kMaxBoxes)
    return record_failure(CX_EINVAL, "too many boxes for the allocation-free level transfer "
                                     "(at most CX_NOALLOC_MAX_BOXES)");
  cudaStream_t s = (cudaStream_t)stream;
  std::lock_guard<std::mutex> guard(g_lock);
  WorkList *dev = nullptr;
  if (int e = scratch_address(&dev))
    return e;
  // boxes, validated as cx_prolong_box does
  int nb = 0;
  bool point[kMaxBoxes];
  for (int i = 0; i < nboxes; ++i) {
    bool empty = false;
    BoxDesc &b = g_stage.boxes[nb];
    if (int e = validate_box_for_level(boxes[i], per_group, &b, &empty))
      return e;
    if (empty)
      continue;
    point[nb] = !box_uses_stream(boxes[i].op, per_group);
    if (b.ntile[0] > INT16_MAX || b.ntile[1] > INT16_MAX || b.ntile[2] > INT16_MAX ||
        b.ncomp > INT16_MAX)
      return record_failure(CX_EINVAL, "too many tiles or components in a box");
    ++nb;
  }
  // items of the streaming boxes, grouped by kernel instantiation: pass 0
  // counts per instantiation, pass 1 places them at off[g] + fill[g]
  int cnt[kStrGroups] = {};
  int off[kStrGroups + 1] = {};
  for (int pass = 0; pass < 2; ++pass) {
    int fill[kStrGroups] = {};
    int total = 0;
    for (int id = 0; id < nb; ++id) {
      if (point[id])
        continue;
      const BoxDesc &b = g_stage.boxes[id];
      const int g = stream_group_of(b.kind[0], b.kind[1], b.kind[2]) + (b.scta ? kStrKinds : 0);
      for (int c = 0; c < b.ncomp; ++c)
        for (int tz = 0; tz < b.ntile[2]; ++tz)
          for (int tx = 0; tx < b.ntile[0]; ++tx) {
            const int xb = b.tbase[0] + tx * b.xcw;
            const int W = std::min(b.xcw, b.rhi[0] - xb + 1);
            const int nub = (b.npr * W + b.upi - 1) / b.upi;
            for (int ub = 0; ub < nub; ++ub) {
              if (++total > kMaxItems)
                return record_failure(CX_EINVAL,
                                      "too many work items for the allocation-free level "
                                      "transfer (at most CX_NOALLOC_MAX_ITEMS)");
              if (pass == 0)
                ++cnt[g];
              else
                g_stage.items[off[g] + fill[g]++] =
                    TileRef{id, (int16_t)tx, (int16_t)ub, (int16_t)tz, (int16_t)c};
            }
          }
    }
    if (pass == 0)
      for (int g = 0; g < kStrGroups; ++g)
        off[g + 1] = off[g] + cnt[g];
  }
  // within an instantiation: most streamed planes first (load balance), in
  // place, with a total order so the list is the same every call
  const BoxDesc *bx = g_stage.boxes;
  for (int g = 0; g < kStrGroups; ++g)
    std::sort(g_stage.items + off[g], g_stage.items + off[g + 1],
              [bx](const TileRef &a, const TileRef &b) {
                const int pa = planes_of(bx[a.box], a.tz), pb = planes_of(bx[b.box], b.tz);
                if (pa != pb)
                  return pa > pb;
                if (a.box != b.box)
                  return a.box < b.box;
                if (a.comp != b.comp)
                  return a.comp < b.comp;
                if (a.tz != b.tz)
                  return a.tz < b.tz;
                if (a.tx != b.tx)
                  return a.tx < b.tx;
                return a.ty < b.ty;
              });
  const int nitems = off[kStrGroups];
  // copy the work list into the device scratch (pageable source: the copy
  // has consumed g_stage when cudaMemcpyAsync returns)
  cudaError_t e = cudaSuccess;
  if (nb > 0)
    e = cudaMemcpyAsync(dev->boxes, g_stage.boxes, sizeof(BoxDesc) * nb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nitems > 0)
    e = cudaMemcpyAsync(dev->items, g_stage.items, sizeof(TileRef) * nitems,
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess && nitems > 0)
    e = cudaMemsetAsync(dev->counters, 0, sizeof(int) * kStrGroups, s);
  for (int g = 0; e == cudaSuccess && g < kStrGroups; ++g) {
    const int n = off[g + 1] - off[g];
    if (n > 0)
      e = launch_stream_level(g, stream_sched(g), dev->boxes, dev->items + off[g], n, stream_level_grid(g, stream_sched(g)),
                              dev->counters + g, s, false);
  }
  for (int id = 0; e == cudaSuccess && id < nb; ++id)
    if (point[id])
      e = launch_point_box(g_stage.boxes[id], per_group, nullptr, nullptr, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return record_failure(CX_ECUDA, cudaGetErrorString(e));
  }
  return CX_OK;
}
