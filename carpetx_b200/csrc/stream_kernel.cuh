// Separable prolongation, column-streaming kernel (all linear families and
// minmod), templated on the operator's pair of 1-D stencil kinds: KV for its
// vertex-centred directions, KC for its cell-centred ones, and on the
// operator's centring CM = (cx << 2) | (cy << 1) | cz (1: cell centred), so
// every pass has a single stencil and the z ring holds exactly the z kind's
// window.
//
// A work item is one component of a block of up to NU fine "units" of a box
// over a chunk of fine z; a unit is a fine x with FYT fine y (FYT / 2
// coarse y centres, whose y windows overlap), units are numbered x fastest
// over the box's x chunk (any width up to WFMAX), so every lane works on a
// real fine point whatever the box shape.  The CTA streams the coarse z
// planes of the block's window through a ring of shared-memory planes:
//   load    the producer warp copies plane c of the coarse window into a
//           free slot of the ring, up to NRING planes ahead: one bulk copy
//           (cp.async.bulk, no multicast) per window row, completing on the
//           slot's mbarrier; only the coarse points the operator reads are
//           copied;
//   x pass  X[cy][fx] = interp_x(coarse row), XB fine x per task from a
//           register window, into shared memory; then the slot is released
//           to the producer (an mbarrier arrival per compute warp);
//   y pass  each compute thread computes Y for the FYT fine y of each of its
//           UPT units from a register window of X (consecutive lanes =
//           consecutive fine x);
//   z pass  each thread keeps the Y values of the last L coarse planes in a
//           register ring; once the ring holds the stencil of coarse centre
//           cc it emits fine z = 2cc and 2cc+1 straight to global memory.
//           The plane loop is unrolled by L, so the ring rotates by register
//           renaming instead of moving L - 1 entries per plane.
// Every coarse value is read from HBM once per column (plus the column's x/y
// halo, which the L2 serves), every intermediate stays on chip, and the fine
// data is written once with coalesced streaming stores.  The arithmetic of
// each 1-D result is the reference's interp1d (CarpetX/src/
// prolongate_3d_rf2_impl.hxx:396-878) and the x/y/z nesting is
// call_stencil_3d (impl.hxx:1206-1216), so the values are bit-identical to
// the reference's; only the number of times a shared 1-D result is evaluated
// changes.
//
// The body (stream_body.cuh) is compiled for two CTA sizes: namespace big
// (256 compute threads, 256 units per item) and namespace small (128 compute
// threads, 128 units) for boxes with at most 128 units per x chunk; each has
// the producer warp besides.  In a level, CTAs
// take items from a per-launch counter, and each launch after a plan's
// first is a programmatic dependent of the previous one.
#pragma once
#include "cx_async.cuh"
#include "cx_internal.h"
#include "cx_stencils.cuh"
#include <type_traits>

namespace cxb {
namespace stream {

// Set when a bounded wait gave up (read and cleared by cx_check_device);
// g_str_wait_limit: cycles a compute thread's wait for a plane's copies polls
// before giving up (kWaitCycles, about a second, unless
// cx_debug_set_wait_limit lowered it to force the give-up path in a test).
// Every translation unit that instantiates the kernels has its own copies.
namespace {
__device__ int g_str_timeout = 0;
__device__ long long g_str_wait_limit = kWaitCycles;
} // namespace

namespace big {
#define CXS_NTS kStrThreads
#include "stream_body.cuh"
#undef CXS_NTS
} // namespace big

namespace small {
#define CXS_NTS kStrThreadsSmall
#include "stream_body.cuh"
#undef CXS_NTS
} // namespace small

static_assert(small::NU == kStrSmallUnits, "the small variant holds a small box's units");

using KernelFn = void (*)(const BoxDesc, const BoxDesc *, const TileRef *, int, int *);

// The kernel of an instantiation for a CTA size and schedule (the 128-thread
// variant and the order-7 z kinds have schedule 0 only).
template <class V, class C, int CM> KernelFn pick_kernel(bool small_cta, int sched) {
  if (small_cta)
    return small::stream_kernel<V, C, CM, 0>;
  if constexpr (big::Kinds<V, C, CM>::ZHI - big::Kinds<V, C, CM>::ZLO < 7) {
    if (sched == 1)
      return big::stream_kernel<V, C, CM, 1>;
  }
  return big::stream_kernel<V, C, CM, 0>;
}
// Whether an instantiation's 256-thread kernel has schedule 1.
template <class V, class C, int CM> constexpr bool has_sched1() {
  return big::Kinds<V, C, CM>::ZHI - big::Kinds<V, C, CM>::ZLO < 7;
}

} // namespace stream
} // namespace cxb
