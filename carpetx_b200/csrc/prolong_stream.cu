// Separable prolongation, column-streaming kernel (all linear families and
// minmod).
//
// A work item is one component of an SX x SY fine column of a box, over a
// chunk of fine z.  The CTA streams the coarse z planes of the column's
// window through a ring of shared-memory planes:
//   load    plane c + DPF of the coarse window (asynchronous 8-byte copies,
//           zero-filled outside the coarse points the operator reads);
//   x pass  X[cy][fx] = interp_x(coarse row), 8 fine x per thread from a
//           register window, into shared memory;
//   y pass  each thread computes Y[fy][fx] for its FYT fine y from a register
//           window of X (consecutive lanes = consecutive fine x);
//   z pass  each thread keeps the Y values of the last L coarse planes in a
//           register ring; once the ring holds the stencil of coarse centre
//           cc it emits fine z = 2cc and 2cc+1 straight to global memory.
// Every coarse value is read from HBM once per column (plus the column's x/y
// halo, which the L2 serves), every intermediate stays on chip, and the fine
// data is written once with coalesced stores.  The arithmetic of each 1-D
// result is the reference's interp1d (CarpetX/src/prolongate_3d_rf2_impl.hxx:
// 396-878) and the x/y/z nesting is call_stencil_3d (impl.hxx:1206-1216), so
// the values are bit-identical to the reference's; only the number of times a
// shared 1-D result is evaluated changes.
#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

constexpr int SX = kStrX, SY = kStrY, FYT = kStrFY, NTS = kStrThreads;
constexpr int DPF = 3;             // coarse planes prefetched ahead
constexpr int NRING = DPF + 1;     // shared-memory plane ring
constexpr int MAXW = 8;            // largest RHI - RLO of a separable kind
constexpr int MAXWX = SX / 2 + MAXW, MAXWY = SY / 2 + MAXW;
constexpr int P0MAX = MAXWX | 1;   // odd row pitch of a coarse plane
constexpr int PLANE = P0MAX * MAXWY;
constexpr int PX = SX + 1;         // row pitch of the x-pass result
constexpr int LDMAX = (PLANE + NTS - 1) / NTS;
static_assert(SX == 32, "lanes map to fine x");
static_assert(NTS == SX * SY / FYT, "one thread per (fine x, group of FYT fine y)");
static_assert(FYT == 2, "the y pass emits 2 fine y per thread");

struct Shared {
  double s0[NRING][PLANE];
  double xs[MAXWY * PX];
};

__device__ __forceinline__ void cp_async8(double *sdst, const double *gsrc, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_dpf() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(DPF) : "memory");
}

// x pass of one coarse plane: 8 fine x (4 coarse cells) per task; task =
// seg * 16 + row, so a half warp covers 16 rows of one segment (odd pitches:
// conflict-free 8-byte accesses).
template <class K>
__device__ __forceinline__ void xpass(const double *__restrict__ S0, int P0, int Wy,
                                      double *__restrict__ xs) {
  constexpr int XB = 8, WIN = XB / 2 + K::RHI - K::RLO;
  const int seg = threadIdx.x >> 4, row = threadIdx.x & 15;
  if (seg >= SX / XB)
    return;
  for (int r = row; r < Wy; r += 16) {
    const double *src = S0 + r * P0 + seg * (XB / 2);
    double v[WIN];
#pragma unroll
    for (int i = 0; i < WIN; ++i)
      v[i] = src[i];
    double *dst = xs + r * PX + seg * XB;
#pragma unroll
    for (int f = 0; f < XB; ++f) {
      if (f & 1)
        dst[f] = K::template ap<1>(v + f / 2 - K::RLO);
      else
        dst[f] = K::template ap<0>(v + f / 2 - K::RLO);
    }
  }
}

// y pass: the 2 fine y fy0, fy0+1 of this thread's fine x share the coarse
// window starting at row fy0/2 of xs.
template <class K>
__device__ __forceinline__ void ypass(const double *__restrict__ xs, int fy0, double y[2]) {
  constexpr int W = 1 + K::RHI - K::RLO;
  double v[W];
  const double *src = xs + (fy0 >> 1) * PX + (threadIdx.x & 31);
#pragma unroll
  for (int i = 0; i < W; ++i)
    v[i] = src[i * PX];
  y[0] = K::template ap<0>(v - K::RLO);
  y[1] = K::template ap<1>(v - K::RLO);
}

template <class K> __device__ __forceinline__ void xpass_k(const double *S0, int P0, int Wy, double *xs) {
  xpass<K>(S0, P0, Wy, xs);
}
template <class K> __device__ __forceinline__ void ypass_k(const double *xs, int fy0, double *y) {
  ypass<K>(xs, fy0, y);
}

// Per-item geometry shared by all planes.
struct Item {
  const double *cbase; // coarse component base
  int64_t cplane;      // coarse z-plane stride
  int clo_z, nlo_z, nhi_z;
  int c_first, c_last; // coarse planes streamed
  int P0, Wy;
  int kx, ky, kz;
  // this thread's fine column: address of (fx, fy0) at fz = 0; fy0 + 1 is
  // fnx further; colmask bit j: fy0 + j inside the region
  double *col;
  int fnx, colmask;
  int64_t fplane;
  int zlo, zhi; // fine z emitted (inclusive)
  // this thread's share of a coarse plane load: smem offset (-1: none) and
  // offset within the coarse z plane (-1: outside the read range in x or y)
  int ld_soff[LDMAX];
  int ld_goff[LDMAX];
};

__device__ __forceinline__ void load_plane(const Item &it, int c, double *S0) {
  const bool zok = c >= it.nlo_z && c <= it.nhi_z;
  const double *pb = it.cbase + (int64_t)(c - it.clo_z) * it.cplane;
#pragma unroll
  for (int i = 0; i < LDMAX; ++i) {
    if (it.ld_soff[i] < 0)
      continue;
    const bool ok = zok && it.ld_goff[i] >= 0;
    cp_async8(S0 + it.ld_soff[i], ok ? pb + it.ld_goff[i] : it.cbase, ok ? 8 : 0);
  }
}

// z stencil of kind kz among the kinds whose window is [ZLO, ZHI].
template <int ZLO, int ZHI, int OFF> struct ZApply {
  template <class K> __device__ __forceinline__ static void one(const double *v, double &r) {
    if constexpr (K::RLO == ZLO && K::RHI == ZHI)
      r = K::template ap<OFF>(v);
  }
  __device__ __forceinline__ static double ap(int kz, const double *v) {
    double r = 0.0;
    CXB_DISPATCH_SEPARABLE(kz, one, v, r);
    return r;
  }
};

// Streams one item.  The z window [ZLO, ZHI] is compile time (it sizes the
// register ring); the x, y and z stencils are dispatched per plane.
template <int ZLO, int ZHI> __device__ __forceinline__ void stream_item(Shared &sh, const Item &it) {
  constexpr int L = ZHI - ZLO + 1;
  double ring[L][FYT];
  const int fy0 = (threadIdx.x >> 5) * FYT;
#pragma unroll
  for (int d = 0; d < DPF; ++d) {
    if (it.c_first + d <= it.c_last)
      load_plane(it, it.c_first + d, sh.s0[d]);
    cp_async_commit();
  }
  int slot = 0;
  for (int c = it.c_first; c <= it.c_last; ++c) {
    {
      int ls = slot + DPF;
      if (ls >= NRING)
        ls -= NRING;
      if (c + DPF <= it.c_last)
        load_plane(it, c + DPF, sh.s0[ls]);
      cp_async_commit();
    }
    cp_async_wait_dpf();
    __syncthreads();
    CXB_DISPATCH_SEPARABLE(it.kx, xpass_k, sh.s0[slot], it.P0, it.Wy, sh.xs);
    __syncthreads();
    double y[FYT];
    CXB_DISPATCH_SEPARABLE(it.ky, ypass_k, sh.xs, fy0, y);
#pragma unroll
    for (int i = 0; i < L - 1; ++i)
#pragma unroll
      for (int j = 0; j < FYT; ++j)
        ring[i][j] = ring[i + 1][j];
#pragma unroll
    for (int j = 0; j < FYT; ++j)
      ring[L - 1][j] = y[j];
    if (c - it.c_first >= L - 1) {
      const int cc = c - ZHI; // coarse centre whose stencil is complete
#pragma unroll
      for (int off = 0; off < 2; ++off) {
        const int fz = 2 * cc + off;
        if (fz < it.zlo || fz > it.zhi)
          continue;
#pragma unroll
        for (int j = 0; j < FYT; ++j) {
          double v[L];
#pragma unroll
          for (int i = 0; i < L; ++i)
            v[i] = ring[i][j];
          const double r = off ? ZApply<ZLO, ZHI, 1>::ap(it.kz, v - ZLO)
                               : ZApply<ZLO, ZHI, 0>::ap(it.kz, v - ZLO);
          if (it.colmask & (1 << j))
            __stcs(it.col + j * it.fnx + (int64_t)fz * it.fplane, r);
        }
      }
    }
    if (++slot == NRING)
      slot = 0;
  }
  __syncthreads(); // the next item reuses the plane ring and xs
}

// Geometry of work item (tx, ty, chunk, comp) of box b.
__device__ __forceinline__ void make_item(const BoxDesc &b, int tx, int ty, int chunk, int comp,
                                          Item &it) {
  const int kx = b.kind[0], ky = b.kind[1], kz = b.kind[2];
  it.kx = kx;
  it.ky = ky;
  it.kz = kz;
  const int ox = b.tbase[0] + tx * SX, oy = b.tbase[1] + ty * SY;
  const int oz = b.tbase[2] + chunk * b.zchunk;
  const int rlx = sep_rlo(kx), rly = sep_rlo(ky);
  const int Wx = SX / 2 + sep_rhi(kx) - rlx;
  it.Wy = SY / 2 + sep_rhi(ky) - rly;
  it.P0 = Wx | 1;
  const int cx0 = ox / 2 + rlx, cy0 = oy / 2 + rly;
  it.cbase = b.crse + comp * b.cnp;
  it.cplane = (int64_t)b.cnx * b.cny;
  it.clo_z = b.clo[2];
  it.nlo_z = b.nlo[2];
  it.nhi_z = b.nhi[2];
  const int zend = min(oz + b.zchunk - 1, b.rhi[2]);
  it.c_first = (oz >> 1) + sep_rlo(kz);
  it.c_last = (zend >> 1) + sep_rhi(kz);
  it.zlo = max(oz, b.rlo[2]);
  it.zhi = zend;
  // fine column of this thread
  const int fx = ox + (threadIdx.x & 31);
  const int fyb = oy + (threadIdx.x >> 5) * FYT;
  it.fplane = (int64_t)b.fnx * b.fny;
  it.fnx = b.fnx;
  const bool xok = fx >= b.rlo[0] && fx <= b.rhi[0];
  it.colmask = 0;
#pragma unroll
  for (int j = 0; j < FYT; ++j) {
    const int fy = fyb + j;
    if (xok && fy >= b.rlo[1] && fy <= b.rhi[1])
      it.colmask |= 1 << j;
  }
  it.col = b.fine + comp * b.fnp + (fx - b.flo[0]) + (int64_t)b.fnx * (fyb - b.flo[1]) -
           it.fplane * b.flo[2];
  // this thread's elements of a coarse plane window
  const int n = Wx * it.Wy;
#pragma unroll
  for (int i = 0; i < LDMAX; ++i) {
    const int e = threadIdx.x + i * NTS;
    if (e >= n) {
      it.ld_soff[i] = -1;
      it.ld_goff[i] = -1;
      continue;
    }
    const int x = e % Wx, y = e / Wx;
    it.ld_soff[i] = y * it.P0 + x;
    const int gx = cx0 + x, gy = cy0 + y;
    const bool ok = gx >= b.nlo[0] && gx <= b.nhi[0] && gy >= b.nlo[1] && gy <= b.nhi[1];
    it.ld_goff[i] = ok ? (gy - b.clo[1]) * b.cnx + (gx - b.clo[0]) : -1;
  }
}

template <int ZLO, int ZHI>
__device__ __forceinline__ void run_item(Shared &sh, const BoxDesc &b, int tx, int ty, int chunk,
                                         int comp) {
  Item it;
  make_item(b, tx, ty, chunk, comp, it);
  stream_item<ZLO, ZHI>(sh, it);
}

// One kernel per z window.  Box mode (items == nullptr): the items of box b
// (x tile, y tile, z chunk, component) strided over the grid.  Level mode:
// items from a device work list (sorted by cost, largest first) dealt
// round-robin to persistent CTAs; the descriptors of the next item are
// loaded into registers while the current item streams, so no global-memory
// latency sits between two items.
constexpr int BOX_WORDS = (int)(sizeof(BoxDesc) / sizeof(int));
static_assert(BOX_WORDS <= NTS, "one thread per descriptor word");

template <int ZLO, int ZHI>
__global__ void __launch_bounds__(NTS, 2)
    stream_kernel(const BoxDesc b, const BoxDesc *__restrict__ boxes,
                  const TileRef *__restrict__ items, int nitems) {
  __shared__ Shared sh;
  __shared__ BoxDesc box_s;
  if (!items) {
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const int tx = item % b.ntile[0];
      int r = item / b.ntile[0];
      const int ty = r % b.ntile[1];
      r /= b.ntile[1];
      const int chunk = r % b.ntile[2];
      const int comp = r / b.ntile[2];
      run_item<ZLO, ZHI>(sh, b, tx, ty, chunk, comp);
    }
    return;
  }
  int cur = blockIdx.x;
  if (cur >= nitems)
    return;
  TileRef t_cur = items[cur];
  int w_cur =
      threadIdx.x < BOX_WORDS ? reinterpret_cast<const int *>(boxes + t_cur.box)[threadIdx.x] : 0;
  TileRef t_next = t_cur;
  if (cur + (int)gridDim.x < nitems)
    t_next = items[cur + gridDim.x];
  while (true) {
    if (threadIdx.x < BOX_WORDS)
      reinterpret_cast<int *>(&box_s)[threadIdx.x] = w_cur;
    __syncthreads();
    // prefetch: descriptor word of the next item, work-list entry of the one after
    const int nxt = cur + gridDim.x;
    int w_next = 0;
    TileRef t_next2 = t_next;
    if (nxt < nitems) {
      if (threadIdx.x < BOX_WORDS)
        w_next = reinterpret_cast<const int *>(boxes + t_next.box)[threadIdx.x];
      if (nxt + (int)gridDim.x < nitems)
        t_next2 = items[nxt + gridDim.x];
    }
    run_item<ZLO, ZHI>(sh, box_s, t_cur.tx, t_cur.ty, t_cur.tz, t_cur.comp);
    if (nxt >= nitems)
      break;
    cur = nxt;
    t_cur = t_next;
    t_next = t_next2;
    w_cur = w_next;
  }
}

// The z windows [sep_rlo, sep_rhi] of the separable kinds.
#define CXB_ZGROUPS(X)                                                         \
  X(0, 0, 0) X(1, 0, 1) X(2, -1, 2) X(3, -2, 3) X(4, -3, 4) X(5, -1, 1)       \
      X(6, -2, 2) X(7, -3, 3) X(8, -4, 4)

using KernelFn = void (*)(const BoxDesc, const BoxDesc *, const TileRef *, int);

KernelFn kernel_for_group(int g) {
  switch (g) {
#define CXB_KCASE(G, LO, HI)                                                   \
  case G:                                                                      \
    return stream_kernel<LO, HI>;
    CXB_ZGROUPS(CXB_KCASE)
#undef CXB_KCASE
  default:
    return nullptr;
  }
}

int g_sms = 0;
int sms() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  return g_sms;
}

} // namespace

void stream_tiling(BoxDesc &b) {
  const int T[2] = {SX, SY};
  for (int d = 0; d < 3; ++d)
    b.tbase[d] = b.rlo[d] & ~1;
  for (int d = 0; d < 2; ++d)
    b.ntile[d] = (b.rhi[d] - b.tbase[d] + T[d]) / T[d];
  // fine z per item: whole columns up to 96 fine points, else near-equal
  // even chunks of at most 96 (the z halo costs RHI - RLO extra planes per
  // chunk)
  const int E = b.rhi[2] - b.tbase[2] + 1;
  const int nch = (E + 95) / 96;
  int zc = (E + nch - 1) / nch;
  zc += zc & 1;
  b.zchunk = zc;
  b.ntile[2] = (E + zc - 1) / zc;
}

int stream_zgroup(int kz) {
  const int lo = sep_rlo(kz), hi = sep_rhi(kz);
#define CXB_GCASE(G, LO, HI)                                                   \
  if (lo == LO && hi == HI)                                                    \
    return G;
  CXB_ZGROUPS(CXB_GCASE)
#undef CXB_GCASE
  return -1;
}

int stream_level_grid(int group) {
  KernelFn k = kernel_for_group(group);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NTS, 0);
  return sms() * (per_sm > 0 ? per_sm : 1);
}

cudaError_t launch_stream_box(const BoxDesc &b, cudaStream_t s) {
  const int64_t n64 = (int64_t)b.ntile[0] * b.ntile[1] * b.ntile[2] * b.ncomp;
  if (n64 <= 0)
    return cudaSuccess;
  if (n64 > INT32_MAX)
    return cudaErrorInvalidValue;
  const int g = stream_zgroup(b.kind[2]);
  KernelFn k = kernel_for_group(g);
  if (!k)
    return cudaErrorInvalidValue;
  const int n = (int)n64;
  const int cap = stream_level_grid(g);
  k<<<n < cap ? n : cap, NTS, 0, s>>>(b, nullptr, nullptr, n);
  return cudaGetLastError();
}

cudaError_t launch_stream_level(int group, const BoxDesc *d_boxes, const TileRef *d_items,
                                int nitems, int grid, cudaStream_t s) {
  if (nitems <= 0)
    return cudaSuccess;
  KernelFn k = kernel_for_group(group);
  if (!k)
    return cudaErrorInvalidValue;
  BoxDesc unused{};
  k<<<grid < nitems ? grid : nitems, NTS, 0, s>>>(unused, d_boxes, d_items, nitems);
  return cudaGetLastError();
}

} // namespace cxb
