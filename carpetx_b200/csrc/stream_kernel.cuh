// Separable prolongation, column-streaming kernel (all linear families and
// minmod), templated on the operator's pair of 1-D stencil kinds: KV for its
// vertex-centred directions, KC for its cell-centred ones.
//
// A work item is one component of an SX x SY fine column of a box, over a
// chunk of fine z.  The CTA streams the coarse z planes of the column's
// window through a ring of shared-memory planes:
//   load    plane c + DPF of the coarse window (asynchronous 8-byte copies,
//           zero-filled outside the coarse points the operator reads);
//   x pass  X[cy][fx] = interp_x(coarse row), 4 fine x per thread from a
//           register window, into shared memory;
//   y pass  each thread computes Y[fy][fx] for its FYT fine y from a register
//           window of X (consecutive lanes = consecutive fine x);
//   z pass  each thread keeps the Y values of the last L coarse planes in a
//           register ring; once the ring holds the stencil of coarse centre
//           cc it emits fine z = 2cc and 2cc+1 straight to global memory.
// Every coarse value is read from HBM once per column (plus the column's x/y
// halo, which the L2 serves), every intermediate stays on chip, and the fine
// data is written once with coalesced streaming stores.  The arithmetic of
// each 1-D result is the reference's interp1d (CarpetX/src/
// prolongate_3d_rf2_impl.hxx:396-878) and the x/y/z nesting is
// call_stencil_3d (impl.hxx:1206-1216), so the values are bit-identical to
// the reference's; only the number of times a shared 1-D result is evaluated
// changes.
#pragma once
#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace stream {

constexpr int SX = kStrX, SY = kStrY, FYT = kStrFY, NTS = kStrThreads;
constexpr int DPF = 3;         // coarse planes prefetched ahead
constexpr int NRING = DPF + 1; // shared-memory plane ring
constexpr int MAXW = 8;        // largest RHI - RLO of a separable kind
constexpr int MAXWX = SX / 2 + MAXW, MAXWY = SY / 2 + MAXW;
constexpr int P0MAX = MAXWX | 1; // odd row pitch of a coarse plane
constexpr int PLANE = P0MAX * MAXWY;
constexpr int PX = SX + 1; // row pitch of the x-pass result
constexpr int LDMAX = (PLANE + NTS - 1) / NTS;
constexpr int XB = 4;                   // fine x per x-pass task
constexpr int XSEG = SX / XB;           // x-pass tasks per row
static_assert(SX == 32, "lanes map to fine x");
static_assert(NTS == SX * SY / FYT, "one thread per (fine x, group of FYT fine y)");
static_assert(FYT == 2, "the y pass emits 2 fine y per thread");
static_assert(XSEG * 16 <= NTS && MAXWY <= 16, "x pass: 16 rows per segment");

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

// x pass of one coarse plane: XB fine x per task; task = seg * 16 + row, so
// a half warp covers 16 rows of one segment (odd pitches: conflict-free
// 8-byte accesses).
template <class K>
__device__ __forceinline__ void xpass(const double *__restrict__ S0, int P0, int Wy,
                                      double *__restrict__ xs) {
  constexpr int WIN = XB / 2 + K::RHI - K::RLO;
  const int seg = threadIdx.x >> 4, row = threadIdx.x & 15;
  if (seg >= XSEG || row >= Wy)
    return;
  const double *src = S0 + row * P0 + seg * (XB / 2);
  double v[WIN];
#pragma unroll
  for (int i = 0; i < WIN; ++i)
    v[i] = src[i];
  double *dst = xs + row * PX + seg * XB;
#pragma unroll
  for (int f = 0; f < XB; ++f) {
    if (f & 1)
      dst[f] = K::template ap<1>(v + f / 2 - K::RLO);
    else
      dst[f] = K::template ap<0>(v + f / 2 - K::RLO);
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

// Per-item geometry shared by all planes.
struct Item {
  const double *cbase; // coarse component base
  int64_t cplane;      // coarse z-plane stride
  int clo_z, nlo_z, nhi_z;
  int c_first, c_last; // coarse planes streamed
  int P0, Wy;
  int ccx, ccy, ccz; // 1: the direction is cell centred (KC), 0: vertex (KV)
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

template <class KV, class KC> struct PairInfo {
  static constexpr int ZLO = KV::RLO < KC::RLO ? KV::RLO : KC::RLO;
  static constexpr int ZHI = KV::RHI > KC::RHI ? KV::RHI : KC::RHI;
};

// Streams one item.  The ring covers the union of the two kinds' z windows
// [ZLO, ZHI]; planes outside the z kind's read range are zero-filled and do
// not reach its stencil.
template <class KV, class KC> __device__ __forceinline__ void stream_item(Shared &sh, const Item &it) {
  constexpr int ZLO = PairInfo<KV, KC>::ZLO, ZHI = PairInfo<KV, KC>::ZHI;
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
    if (it.ccx)
      xpass<KC>(sh.s0[slot], it.P0, it.Wy, sh.xs);
    else
      xpass<KV>(sh.s0[slot], it.P0, it.Wy, sh.xs);
    __syncthreads();
    double y[FYT];
    if (it.ccy)
      ypass<KC>(sh.xs, fy0, y);
    else
      ypass<KV>(sh.xs, fy0, y);
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
          double r;
          if (it.ccz)
            r = off ? KC::template ap<1>(v - ZLO) : KC::template ap<0>(v - ZLO);
          else
            r = off ? KV::template ap<1>(v - ZLO) : KV::template ap<0>(v - ZLO);
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

// Geometry of work item (tx, ty, chunk, comp) of box b; [zlo, zhi] is the
// streaming window of the pair.
__device__ __forceinline__ void make_item(const BoxDesc &b, int tx, int ty, int chunk, int comp,
                                          int zwlo, int zwhi, Item &it) {
  const int kx = b.kind[0], ky = b.kind[1];
  it.ccx = kind_info(kx).cent;
  it.ccy = kind_info(ky).cent;
  it.ccz = kind_info(b.kind[2]).cent;
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
  it.c_first = (oz >> 1) + zwlo;
  it.c_last = (zend >> 1) + zwhi;
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

template <class KV, class KC>
__device__ __forceinline__ void run_item(Shared &sh, const BoxDesc &b, int tx, int ty, int chunk,
                                         int comp) {
  Item it;
  make_item(b, tx, ty, chunk, comp, PairInfo<KV, KC>::ZLO, PairInfo<KV, KC>::ZHI, it);
  stream_item<KV, KC>(sh, it);
}

constexpr int BOX_WORDS = (int)(sizeof(BoxDesc) / sizeof(int));
static_assert(BOX_WORDS <= NTS, "one thread per descriptor word");

// Box mode (items == nullptr): the items of box b (x tile, y tile, z chunk,
// component) strided over the grid.  Level mode: items from a device work
// list (sorted by cost, largest first) dealt round-robin to persistent CTAs;
// the descriptors of the next item are loaded into registers while the
// current item streams, so no global-memory latency sits between two items.
template <class KV, class KC>
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
      run_item<KV, KC>(sh, b, tx, ty, chunk, comp);
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
    run_item<KV, KC>(sh, box_s, t_cur.tx, t_cur.ty, t_cur.tz, t_cur.comp);
    if (nxt >= nitems)
      break;
    cur = nxt;
    t_cur = t_next;
    t_next = t_next2;
    w_cur = w_next;
  }
}

using KernelFn = void (*)(const BoxDesc, const BoxDesc *, const TileRef *, int);

} // namespace stream
} // namespace cxb
