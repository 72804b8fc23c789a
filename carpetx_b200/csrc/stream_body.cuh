// Body of the streaming kernel, included once per CTA size (stream_kernel.cuh
// defines CXS_NTS and the enclosing namespace): 256 threads for items of up
// to 256 column units, 128 threads for the items of boxes with at most 128
// units per x chunk, so that a small box does not run with half of its
// threads idle.  No include guard: included twice on purpose.


constexpr int NTS = CXS_NTS;    // threads per CTA (256, or 128 for small items)
constexpr int UPT = kStrUnitsPerThread; // column units per thread
constexpr int NU = NTS * UPT;    // column units per item
constexpr int FYT = kStrFineYPerUnit; // fine y per unit
constexpr int CYU = FYT / 2;     // coarse y centres per unit
constexpr int PRMAX = kStrUnitRows; // rows of units per item at most
constexpr int WFMAX = kStrMaxWidth; // fine x per x chunk at most
constexpr int NRING = 4;         // shared-memory plane ring: planes are copied NRING ahead
constexpr int MAXW = 8;          // largest RHI - RLO of a separable kind
constexpr int XB = 4;            // fine x per x-pass task

// Geometry of an item whose x chunk is W fine points wide (worst case over
// the stencil kinds): rows of the coarse window / x-pass result, their
// pitches, x-pass tasks.
// coarse y centres an item of W-wide unit rows spans at most
__host__ __device__ constexpr int span_rows(int W) {
  return CYU * (PRMAX < (NU - 1) / W + 2 ? PRMAX : (NU - 1) / W + 2);
}
__host__ __device__ constexpr int nseg_of(int W) { return (W + XB - 1) / XB; }
// Odd pitch of a coarse window row of an x kind with spread wx, for copies
// of single rows: the row's Wx = (W - 1) / 2 + 1 + wx points start at column
// 1, 2 or 3 (a shift of 0 or 1 that matches the parity of the row's global
// address at the item's first plane, plus 1 on planes where that parity
// flips, so that a bulk copy's 16-byte aligned ends fall on 16-byte aligned
// shared addresses), a copy may write one column before and one after them,
// and the x-pass tasks read up to column nseg * 2 + wx + 2.
__host__ __device__ constexpr int p0_of(int W, int wx) { return (nseg_of(W) * XB / 2 + wx + 4) | 1; }
__host__ __device__ constexpr int pxw_of(int W) { return (nseg_of(W) * XB) | 1; }
__host__ __device__ constexpr int max_over_w(int what) {
  int m = 0;
  for (int W = 1; W <= WFMAX; ++W) {
    const int nr = span_rows(W) + MAXW;
    const int v = what == 0   ? nr * p0_of(W, MAXW)
                  : what == 1 ? nr * pxw_of(W)
                  : what == 2 ? nr * nseg_of(W)
                              : nr;
    m = v > m ? v : m;
  }
  return m;
}
constexpr int PLANE = (max_over_w(0) + 1) & ~1; // coarse plane window (doubles; even: 16-byte slots)
constexpr int XBUF = max_over_w(1);             // x-pass result (doubles)
constexpr int XTMAX = (max_over_w(2) + NTS - 1) / NTS;
static_assert(NU % 32 == 0, "whole warps");
static_assert(XTMAX <= 31, "x-task parity bits");
static_assert(max_over_w(3) <= NTS, "one window row per thread");

struct Shared {
  double s0[NRING][PLANE];
  double xs[2][XBUF];     // x-pass results of even / odd planes
  uint64_t full[NRING];   // plane in slot: thread 0's arrival + the copies' bytes
  int64_t rlen[2];        // bytes a plane's copies carry, by parity flip
  int fail;               // a bounded wait gave up: no further copies, the CTA stops
};

// The slow path of a compute thread's wait for a plane (its first poll
// failed): polls bounded by `limit` cycles, giving up at once when another
// thread of the CTA has given up or the limit is 0 (tests force the give-up
// path so).  On giving up it records the failure for the CTA (no further
// copies are issued) and for cx_check_device.
static __device__ __noinline__ void wait_plane_slow(uint64_t *m, uint32_t parity, volatile int *fail,
                                             long long limit) {
  const long long t0 = clock64();
  while (limit > 0 && !*fail) {
    if (mbar_try(m, parity))
      return;
    if (clock64() - t0 > limit)
      break;
  }
  *fail = 1;
  g_str_timeout = 1;
}

// One x-pass task: XB fine x from a register window of a coarse row.
template <class K>
__device__ __forceinline__ void xtask(const double *__restrict__ src, double *__restrict__ dst) {
  constexpr int WIN = XB / 2 + K::RHI - K::RLO;
  double v[WIN];
#pragma unroll
  for (int i = 0; i < WIN; ++i)
    v[i] = src[i];
#pragma unroll
  for (int f = 0; f < XB; ++f) {
    if (f & 1)
      dst[f] = K::template ap<1>(v + f / 2 - K::RLO);
    else
      dst[f] = K::template ap<0>(v + f / 2 - K::RLO);
  }
}

// y pass of one unit: its FYT fine y (CYU coarse y centres, 2 fine y each)
// from the coarse y window starting at src (rows pxw apart).
template <class K>
__device__ __forceinline__ void ypass(const double *__restrict__ src, int pxw, double y[FYT]) {
  constexpr int W = CYU + K::RHI - K::RLO;
  double v[W];
#pragma unroll
  for (int i = 0; i < W; ++i)
    v[i] = src[i * pxw];
#pragma unroll
  for (int c = 0; c < CYU; ++c) {
    y[2 * c] = K::template ap<0>(v + c - K::RLO);
    y[2 * c + 1] = K::template ap<1>(v + c - K::RLO);
  }
}

// Per-item, per-thread geometry shared by all planes.
struct Item {
  int c_first, c_last; // coarse planes streamed
  int clo_z, cpl1;     // the item's first coarse plane, coarse z-plane stride & 1
  int pxw;             // row pitch of the x-pass result
  // this thread's units (tid and tid + NTS of the block): y window start in
  // xs (0 for a unit without a column); address of (fx, fy0) at fz = 0
  // (fy0 + 1 is fnx further); colmask bit j: fy0 + j inside the region
  int ysrc[UPT];
  double *col[UPT];
  int colmask[UPT];
  int fnx;
  int64_t fplane;
  int zlo, zhi; // fine z emitted (inclusive)
  // x-pass tasks: offsets of the task's window in a slot (on planes whose
  // parity flip is 0; one more on the others) and of its result in xs (-1:
  // none); rounds of NTS tasks the item needs
  int xt_src[XTMAX];
  int xt_dst[XTMAX];
  int nxt;
  // coarse plane copies.  Whole rows (whole = true): the window rows of the
  // read range, nearly whole rows of the coarse FAB, are one contiguous range
  // of the plane, copied by thread 0 as one bulk copy, rows cnx apart in the
  // slot; its first point lands at column MARG + rsm + flip (rsm = the
  // parity of the point's global address at the item's first plane); roff =
  // offset of that point in a plane, clen = points from the first to the
  // last.  Otherwise one copy per window row: lane l of warp w copies window
  // row r = l NW + w (NW warps), so that every warp issues about as many
  // copies (a warp's copies are issued one lane after the other); roff =
  // offset of the row's window column 0 in a plane; its column 0 lands at
  // rsm + flip, rsm = r P0 + 1 + the parity shift of the item's first plane
  // (-1: no copy).  warp_rows: the warp issues copies.  xa, xb: window
  // columns inside the read range
  const double *cbase;
  int64_t cplane;
  int nlo_z, nhi_z;
  int roff, rsm, clen;
  int xa, xb;
  bool warp_rows, whole;
};

// Column of a slot where a whole-row copy starts (even: 16-byte aligned);
// the x pass may read up to MARG columns before the first copied point.
constexpr int MARG = 16;
// a whole-row copy carries at most this many points per row outside the
// window
constexpr int WHOLE_SLACK = 8;

// The stencil kinds of an instantiation per direction; [ZLO, ZHI] is the z
// kind's window (coarse planes relative to the centre).
template <class KV, class KC, int CM> struct Kinds {
  using KX = std::conditional_t<(CM & 4) != 0, KC, KV>;
  using KY = std::conditional_t<(CM & 2) != 0, KC, KV>;
  using KZ = std::conditional_t<(CM & 1) != 0, KC, KV>;
  static constexpr int ZLO = KZ::RLO, ZHI = KZ::RHI;
};

// Bulk copy of one window row, widened to 16-byte aligned ends (at most one
// point either side, in the same 16-byte block as a point of the read
// range): window columns [xal, xend] of the row whose column 0 is at global
// g.  Returns the bytes.
__device__ __forceinline__ uint32_t row_copy_bytes(uintptr_t g, int xa, int xb, int *xal_out) {
  const int par = (int)((g >> 3) & 1);
  const int xal = xa - ((par + xa) & 1);
  const int xend = xb + 1 - ((par + xb) & 1);
  *xal_out = xal;
  return 8u * (uint32_t)(xend - xal + 1);
}

// Geometry of work item (x chunk, unit block, z chunk, comp) of box b, for
// the z kind's streaming window [zwlo, zwhi].
// The item's units are the unit block's consecutive (unit row, fine x)
// columns of the x chunk, flattened x fastest; thread t owns unit t.
// Returns false if the block holds no unit (box mode, narrow last chunk).
// Thread 0 also leaves in rlen the bytes of one plane's copies for both
// parity shifts (the caller's barrier publishes them).
__device__ __forceinline__ bool make_item(const BoxDesc &b, int xchunk, int ublock, int zchunk,
                                          int comp, int zwlo, int zwhi, Item &it,
                                          int64_t *rlen) {
  const int tid = threadIdx.x;
  const int kx = b.kind[0], ky = b.kind[1];
  const int xb = b.tbase[0] + xchunk * b.xcw;
  const int W = min(b.xcw, b.rhi[0] - xb + 1);
  const int nunits = b.npr * W;
  const int u0 = ublock * b.upi;
  if (u0 >= nunits)
    return false;
  const int uend = min(u0 + b.upi, nunits);
  const int pr_lo = u0 / W, pr_hi = (uend - 1) / W;
  const int rlx = sep_rlo(kx), rly = sep_rlo(ky);
  const int NR = (pr_hi - pr_lo + 1) * CYU + sep_rhi(ky) - rly;
  const int nseg = nseg_of(W);
  const int Wx = (W - 1) / 2 + 1 + sep_rhi(kx) - rlx;
  const int P0 = p0_of(W, sep_rhi(kx) - rlx);
  it.pxw = pxw_of(W);
  const int cxb = xb / 2 + rlx;                   // xb even
  const int cyb = b.tbase[1] / 2 + pr_lo * CYU + rly; // tbase even
  it.cbase = b.crse + comp * b.cnp;
  it.cplane = (int64_t)b.cnx * b.cny;
  it.cpl1 = (int)(it.cplane & 1);
  it.clo_z = b.clo[2];
  it.nlo_z = b.nlo[2];
  it.nhi_z = b.nhi[2];
  const int oz = b.tbase[2] + zchunk * b.zchunk;
  const int zend = min(oz + b.zchunk - 1, b.rhi[2]);
  it.c_first = (oz >> 1) + zwlo;
  it.c_last = (zend >> 1) + zwhi;
  it.zlo = max(oz, b.rlo[2]);
  it.zhi = zend;
  // this thread's units
  it.fplane = (int64_t)b.fnx * b.fny;
  it.fnx = b.fnx;
#pragma unroll
  for (int q = 0; q < UPT; ++q) {
    const int u = u0 + tid + q * NTS;
    it.colmask[q] = 0;
    it.ysrc[q] = 0; // no column: any in-bounds window of xs
    it.col[q] = b.fine;
    if (u < uend) {
      const int pr = u / W, fxl = u - pr * W;
      const int fx = xb + fxl, fy0 = b.tbase[1] + FYT * pr;
      it.ysrc[q] = (pr - pr_lo) * CYU * it.pxw + fxl;
      if (fx >= b.rlo[0]) {
#pragma unroll
        for (int j = 0; j < FYT; ++j)
          if (fy0 + j >= b.rlo[1] && fy0 + j <= b.rhi[1])
            it.colmask[q] |= 1 << j;
      }
      it.col[q] = b.fine + comp * b.fnp + (fx - b.flo[0]) + (int64_t)b.fnx * (fy0 - b.flo[1]) -
                  it.fplane * b.flo[2];
    }
  }
  // window rows and columns inside the read range
  it.xa = max(0, b.nlo[0] - cxb);
  it.xb = min(Wx - 1, b.nhi[0] - cxb);
  const int ra = max(0, b.nlo[1] - cyb), rb = min(NR - 1, b.nhi[1] - cyb);
  const int dx = sep_rhi(kx) - rlx;
  it.whole = ra <= rb && it.xa <= it.xb && it.xa <= MARG && b.cnx <= Wx + WHOLE_SLACK &&
             MARG + (rb - ra) * b.cnx + max(2 * nseg + dx, Wx) + 4 <= PLANE;
  // x-pass tasks: NR rows x nseg segments, rows fastest.  Per-row copies:
  // row r of a plane sits at r P0 + 1 + s, s = s0 + flip, s0 = (parity of
  // the global address of its window column 0 at the item's first plane +
  // r P0 + 1) & 1, flip = 1 on planes where that parity has flipped (odd
  // plane stride, odd distance from clo_z), the shift its copy uses.  Whole
  // rows: point (r, x) of the read range sits at MARG + p0 + flip +
  // (r - ra) cnx + (x - xa), p0 = the parity of the global address of point
  // (ra, xa) at the item's first plane; rows outside the read range read row
  // ra instead (their results are not stored).
  const int64_t pbase = (int64_t)((uintptr_t)it.cbase >> 3) + (int64_t)(cyb - b.clo[1]) * b.cnx +
                        (cxb - b.clo[0]) + (int64_t)(it.c_first - b.clo[2]) * it.cplane;
  const int p0 = (int)((pbase + (int64_t)ra * b.cnx + it.xa) & 1);
  // planes are counted from the item's first plane (cbase then points at
  // that plane of the component, the flip is relative to it)
  it.cbase += (int64_t)(it.c_first - b.clo[2]) * it.cplane;
  it.clo_z = it.c_first;
  const int nt = NR * nseg;
  it.nxt = (nt + NTS - 1) / NTS;
#pragma unroll
  for (int k = 0; k < XTMAX; ++k) {
    const int t = tid + k * NTS;
    it.xt_src[k] = -1;
    it.xt_dst[k] = -1;
    if (t < nt) {
      const int sg = t / NR, r = t - sg * NR;
      it.xt_dst[k] = r * it.pxw + sg * XB;
      if (it.whole) {
        const int rr = min(max(r, ra), rb);
        it.xt_src[k] = MARG + p0 + (rr - ra) * b.cnx + sg * (XB / 2) - it.xa;
      } else {
        const int rsm = r * P0 + 1;
        it.xt_src[k] = rsm + (int)((pbase + (int64_t)r * b.cnx + rsm) & 1) + sg * (XB / 2);
      }
    }
  }
  it.rsm = -1;
  it.roff = 0;
  it.clen = 0;
  if (it.whole) {
    it.warp_rows = tid < 32;
    if (tid == 0) {
      it.rsm = p0;
      it.roff = (cyb + ra - b.clo[1]) * b.cnx + (cxb + it.xa - b.clo[0]);
      it.clen = (rb - ra) * b.cnx + (it.xb - it.xa);
    }
    return true;
  }
  // this thread's window row: copied if it lies in the read range
  it.warp_rows = (tid >> 5) < NR;
  {
    const int r = (tid & 31) * (NTS / 32) + (tid >> 5), gy = cyb + r;
    if (r < NR && gy >= b.nlo[1] && gy <= b.nhi[1] && it.xa <= it.xb) {
      const int rsm = r * P0 + 1;
      it.rsm = rsm + (int)((pbase + (int64_t)r * b.cnx + rsm) & 1);
      it.roff = (gy - b.clo[1]) * b.cnx + (cxb - b.clo[0]);
    }
  }
  // bytes of a plane's copies, for both parity flips (the same rows and
  // arithmetic as the copies)
  if (tid == 0) {
    int64_t n[2] = {0, 0};
    if (it.xa <= it.xb)
      for (int r = 0; r < NR; ++r) {
        const int gy = cyb + r;
        if (gy < b.nlo[1] || gy > b.nhi[1])
          continue;
        const uintptr_t g0 =
            (uintptr_t)(it.cbase + (int64_t)(gy - b.clo[1]) * b.cnx + (cxb - b.clo[0]));
        int x;
        n[0] += row_copy_bytes(g0, it.xa, it.xb, &x);
        n[1] += row_copy_bytes(g0 + 8 * (uintptr_t)it.cplane, it.xa, it.xb, &x);
      }
    rlen[0] = n[0];
    rlen[1] = n[1];
  }
  return true;
}

// Issues the copies of coarse plane c into slot buffer S, completing on
// mbarrier m (called by the warps with copies only).  Whole rows: thread 0
// arrives expecting the copy's bytes and issues it (the range rounded out
// to 16-byte blocks: at most one point either side, in the same block as a
// point of the read range; it lands at column MARG + 2 (p0 & flip), which
// puts the first point at MARG + p0 + flip).  Per row: thread 0 arrives
// expecting the plane's bytes (rlen by the plane's parity flip) and each
// thread with a window row copies it.  Nothing is copied for a plane outside
// the read range.  Rows, columns and planes outside the read range keep
// stale data, which reaches only points that are never stored.
__device__ __forceinline__ void load_plane(const Item &it, const int64_t *rlen, int c, double *S,
                                           uint64_t *m) {
  const bool zok = c >= it.nlo_z && c <= it.nhi_z;
  const int flip = (c - it.clo_z) & it.cpl1;
  const double *pb = it.cbase + (int64_t)(c - it.clo_z) * it.cplane;
  if (it.whole) {
    if (threadIdx.x == 0) {
      if (zok) {
        const uintptr_t e0 = (uintptr_t)(pb + it.roff);
        const uintptr_t a0 = e0 & ~(uintptr_t)15, a1 = ((e0 + 8 * (uintptr_t)it.clen) | 15) + 1;
        const uint32_t nb = (uint32_t)(a1 - a0);
        mbar_arrive_expect_tx(m, nb);
        bulk_g2s(S + MARG + 2 * (it.rsm & flip), (const void *)a0, nb, m);
      } else {
        mbar_arrive_expect_tx(m, 0u);
      }
    }
    return;
  }
  if (threadIdx.x == 0)
    mbar_arrive_expect_tx(m, zok ? (uint32_t)rlen[flip] : 0u);
  if (zok && it.rsm >= 0) {
    const double *g = pb + it.roff;
    int xal;
    const uint32_t nb = row_copy_bytes((uintptr_t)g, it.xa, it.xb, &xal);
    bulk_g2s(S + it.rsm + flip + xal, g + xal, nb, m);
  }
}

// Streams one item.  The ring covers the z kind's window [ZLO, ZHI].  seq
// counts the planes this CTA has streamed: plane slot seq % NRING, mbarrier
// phase parity (seq / NRING) & 1, x-pass buffer seq & 1.  Returns false if a
// bounded wait gave up (every thread alike): the copies still in flight
// have landed (bounded) when it returns.
template <class KV, class KC, int CM, int SCHED>
__device__ __forceinline__ bool stream_item(Shared &sh, const Item &it, uint32_t &seq,
                                            long long limit) {
  using KX = typename Kinds<KV, KC, CM>::KX;
  using KY = typename Kinds<KV, KC, CM>::KY;
  using KZ = typename Kinds<KV, KC, CM>::KZ;
  constexpr int ZLO = KZ::RLO, ZHI = KZ::RHI;
  constexpr int L = ZHI - ZLO + 1;
  double ring[L][UPT][FYT];
  // planes issued by this CTA (seq of the next plane to issue); thread 0's
  // count is the one the drain uses
  uint32_t issued = seq;
  if (it.warp_rows)
    for (int d = 0; d < NRING && it.c_first + d <= it.c_last; ++d, ++issued)
      load_plane(it, sh.rlen, it.c_first + d, sh.s0[issued % NRING], &sh.full[issued % NRING]);
  for (int c0 = it.c_first; c0 <= it.c_last; c0 += L) {
#pragma unroll
    for (int ph = 0; ph < L; ++ph) {
      const int c = c0 + ph;
      if (c > it.c_last)
        break;
      const int slot = (int)(seq % NRING);
      if (!(limit > 0 && mbar_try(&sh.full[slot], (seq / NRING) & 1u)))
        wait_plane_slow(&sh.full[slot], (seq / NRING) & 1u, &sh.fail, limit);
      const double *S = sh.s0[slot] + ((c - it.clo_z) & it.cpl1);
      double *X = sh.xs[seq & 1];
      if constexpr (SCHED == 1) {
        // a rolled loop: one copy of the task body per unrolled plane keeps
        // the kernel's code small (with three CTAs per SM, instruction fetch
        // stalls otherwise cost more than the loop)
#pragma unroll 1
        for (int k = 0; k < it.nxt; ++k) {
          int src = it.xt_src[0], dst = it.xt_dst[0];
#pragma unroll
          for (int kk = 1; kk < XTMAX; ++kk)
            if (k == kk) {
              src = it.xt_src[kk];
              dst = it.xt_dst[kk];
            }
          if (src >= 0)
            xtask<KX>(S + src, X + dst);
        }
      } else {
#pragma unroll
        for (int k = 0; k < XTMAX; ++k) {
          if (k >= it.nxt)
            break;
          if (it.xt_src[k] < 0)
            continue;
          xtask<KX>(S + it.xt_src[k], X + it.xt_dst[k]);
        }
      }
      // every thread has read the slot and written its x results (the
      // other x buffer's readers, plane c - 1, are past this barrier too)
      __syncthreads();
      if (it.warp_rows && c + NRING <= it.c_last && !*(volatile int *)&sh.fail) {
        load_plane(it, sh.rlen, c + NRING, sh.s0[slot], &sh.full[slot]);
        ++issued;
      }
      ++seq;
      // ring slot ph takes plane c; logical position i (0 oldest) is slot
      // (ph + 1 + i) % L
      // (units without a column read a valid part of xs and are never
      // stored: no branch, so the compiler can interleave both units' work)
#pragma unroll
      for (int q = 0; q < UPT; ++q) {
        double y[FYT];
        ypass<KY>(X + it.ysrc[q], it.pxw, y);
#pragma unroll
        for (int j = 0; j < FYT; ++j)
          ring[ph][q][j] = y[j];
      }
      if (c - it.c_first >= L - 1) {
        const int cc = c - ZHI; // coarse centre whose stencil is complete
#pragma unroll
        for (int off = 0; off < 2; ++off) {
          // both offsets are evaluated; a fine z outside the chunk (its first
          // or last plane) is only not stored
          const int fz = 2 * cc + off;
          const bool zin = fz >= it.zlo && fz <= it.zhi;
#pragma unroll
          for (int q = 0; q < UPT; ++q)
#pragma unroll
            for (int j = 0; j < FYT; ++j) {
              double v[L];
#pragma unroll
              for (int i = 0; i < L; ++i)
                v[i] = ring[(ph + 1 + i) % L][q][j];
              const double r = off ? KZ::template ap<1>(v - ZLO) : KZ::template ap<0>(v - ZLO);
              if (zin && (it.colmask[q] & (1 << j)))
                __stcs(it.col[q] + j * it.fnx + (int64_t)fz * it.fplane, r);
            }
        }
      }
    }
  }
  __syncthreads(); // the next item reuses the plane ring and xs; publishes fail
  if (sh.fail) {
    // stop once the copies still in flight (the last NRING planes issued)
    // have landed, each wait bounded by the default
    if (threadIdx.x == 0)
      for (uint32_t q = issued > (uint32_t)NRING ? issued - NRING : 0; q < issued; ++q)
        mbar_wait_bounded(&sh.full[q % NRING], (q / NRING) & 1u);
    __syncthreads();
    return false;
  }
  return true;
}

template <class KV, class KC, int CM, int SCHED>
__device__ __forceinline__ bool run_item(Shared &sh, const BoxDesc &b, int xchunk, int ublock,
                                         int zchunk, int comp, uint32_t &seq, long long limit) {
  Item it;
  // uniform over the CTA: an empty block is skipped by every thread
  if (!make_item(b, xchunk, ublock, zchunk, comp, Kinds<KV, KC, CM>::ZLO, Kinds<KV, KC, CM>::ZHI,
                 it, sh.rlen))
    return true;
  __syncthreads(); // rlen
  return stream_item<KV, KC, CM, SCHED>(sh, it, seq, limit);
}

__device__ __forceinline__ void init_shared(Shared &sh) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < NRING; ++i)
      mbar_init(&sh.full[i], 1);
    sh.fail = 0;
    mbar_fence_init();
  }
  __syncthreads();
}

constexpr int BOX_WORDS = (int)(sizeof(BoxDesc) / sizeof(int));
static_assert(BOX_WORDS <= NTS, "one thread per descriptor word");

// Box mode (items == nullptr): the items of box b (x tile, y tile, z chunk,
// component) strided over the grid.  Level mode: items from a device work
// list (sorted by cost, largest first) taken by persistent CTAs from a
// counter;
// the descriptors of the next item are loaded into registers while the
// current item streams, so no global-memory latency sits between two items.
// Schedules (SCHED) of the 256-thread kernel, picked per instantiation by
// the tuned table (stream_tuned.h, written by carpetx_b200/tune.py):
//   0: two CTAs per SM (at most 128 registers), x-task loop unrolled;
//   1: three CTAs per SM (at most 80 registers, a few words may spill),
//      x-task loop rolled (a smaller body).
// The order-7 z kinds, whose register ring holds 8 or 9 planes, run one CTA
// per SM in both; the 128-thread variant has one schedule, four CTAs per SM
// (two for the order-7 z kinds).
template <int DZ, int SCHED> struct StreamOcc {
  static constexpr int value = NTS == 256 ? (DZ >= 7 ? 1 : SCHED == 1 ? 3 : 2) : (DZ >= 7 ? 2 : 4);
};
template <class KV, class KC, int CM, int SCHED>
__global__ void __launch_bounds__(NTS, StreamOcc<Kinds<KV, KC, CM>::ZHI - Kinds<KV, KC, CM>::ZLO, SCHED>::value)
    stream_kernel(const BoxDesc b, const BoxDesc *__restrict__ boxes,
                  const TileRef *__restrict__ items, int nitems, int *__restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[]; // sizeof(Shared) bytes
  Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
  __shared__ BoxDesc box_s;
  init_shared(sh);
  uint32_t seq = 0;
  const long long limit = g_str_wait_limit;
  if (!items) {
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const int xchunk = item % b.ntile[0];
      int r = item / b.ntile[0];
      const int ublock = r % b.ntile[1];
      r /= b.ntile[1];
      const int zchunk = r % b.ntile[2];
      const int comp = r / b.ntile[2];
      if (!run_item<KV, KC, CM, SCHED>(sh, b, xchunk, ublock, zchunk, comp, seq, limit))
        return;
    }
    return;
  }
  // Level launches after the first of a plan are programmatic dependents of
  // the previous one (they write other boxes): let the next launch start as
  // soon as every CTA of this one is running, so it fills this launch's
  // tail, and end with the wait on the previous launch, so that this
  // launch completes only after it.  Without the launch attribute both
  // instructions are no-ops.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  // Items are taken in list order (largest first): each CTA starts with item
  // blockIdx.x and then takes the next untaken one from the launch's counter
  // (zero before the launch), one item ahead of the one it streams, so a CTA
  // that started late or drew long items takes fewer.
  __shared__ int s_take;
  const int G = gridDim.x;
  int cur = blockIdx.x;
  if (cur >= nitems) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    return;
  }
  if (threadIdx.x == 0)
    s_take = G + atomicAdd(counter, 1);
  __syncthreads();
  int nxt = s_take;
  TileRef t_cur = items[cur];
  int w_cur =
      threadIdx.x < BOX_WORDS ? reinterpret_cast<const int *>(boxes + t_cur.box)[threadIdx.x] : 0;
  TileRef t_next = nxt < nitems ? items[nxt] : t_cur;
  while (true) {
    if (threadIdx.x < BOX_WORDS)
      reinterpret_cast<int *>(&box_s)[threadIdx.x] = w_cur;
    __syncthreads(); // also: every thread has read s_take
    if (threadIdx.x == 0 && nxt < nitems)
      s_take = G + atomicAdd(counter, 1);
    // prefetch: descriptor word of the next item
    int w_next = 0;
    if (nxt < nitems && threadIdx.x < BOX_WORDS)
      w_next = reinterpret_cast<const int *>(boxes + t_next.box)[threadIdx.x];
    __syncthreads();
    const int nxt2 = nxt < nitems ? s_take : nitems;
    TileRef t_next2 = t_next;
    if (nxt2 < nitems)
      t_next2 = items[nxt2]; // work-list entry of the item after next
    if (!run_item<KV, KC, CM, SCHED>(sh, box_s, t_cur.tx, t_cur.ty, t_cur.tz, t_cur.comp, seq,
                                     limit) ||
        nxt >= nitems) {
      asm volatile("griddepcontrol.wait;" ::: "memory");
      break;
    }
    cur = nxt;
    nxt = nxt2;
    t_cur = t_next;
    t_next = t_next2;
    w_cur = w_next;
  }
}
