// Body of the streaming kernel, included once per CTA size (stream_kernel.cuh
// defines CXS_NTS and the enclosing namespace): 256 threads for items of up to
// 512 column units, 128 threads for the items of boxes with at most 256
// units per x chunk, so that a small box does not run with three quarters of
// its threads idle.  No include guard: included twice on purpose.


constexpr int NTS = CXS_NTS;    // threads per CTA (256, or 128 for small items)
constexpr int UPT = kStrUnitsPerThread; // column units per thread
constexpr int NU = NTS * UPT;    // column units per item
constexpr int FYT = kStrFineYPerUnit; // fine y per unit
constexpr int CYU = FYT / 2;     // coarse y centres per unit
constexpr int PRMAX = kStrUnitRows; // rows of units per item at most
constexpr int WFMAX = kStrMaxWidth; // fine x per x chunk at most
constexpr int DPF = 3;           // coarse planes prefetched ahead
constexpr int NRING = DPF + 1;   // shared-memory plane ring
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
__host__ __device__ constexpr int p0_of(int W, int wx) { return (nseg_of(W) * XB / 2 + wx) | 1; }
__host__ __device__ constexpr int pxw_of(int W) { return (nseg_of(W) * XB) | 1; }
__host__ __device__ constexpr int max_over_w(int what) {
  int m = 0;
  for (int W = 1; W <= WFMAX; ++W) {
    const int nr = span_rows(W) + MAXW;
    const int v = what == 0 ? nr * p0_of(W, MAXW) : what == 1 ? nr * pxw_of(W) : nr * nseg_of(W);
    m = v > m ? v : m;
  }
  return m;
}
constexpr int PLANE = max_over_w(0); // coarse plane window (doubles)
constexpr int XBUF = max_over_w(1);  // x-pass result (doubles)
constexpr int LDMAX = (PLANE + NTS - 1) / NTS;
constexpr int XTMAX = (max_over_w(2) + NTS - 1) / NTS;
static_assert(NU % 32 == 0, "whole warps");

struct Shared {
  double s0[NRING][PLANE];
  double xs[XBUF];
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
  const double *cbase; // coarse component base
  int64_t cplane;      // coarse z-plane stride
  int clo_z, nlo_z, nhi_z;
  int c_first, c_last; // coarse planes streamed
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
  // coarse plane loads: smem offset (-1: none) and offset within the coarse
  // z plane (-1: outside the read range in x or y, zero-filled); rounds of
  // NTS loads the item needs (the same for every thread)
  int ld_soff[LDMAX];
  int ld_goff[LDMAX];
  int nld;
  // x-pass tasks: smem offsets into the plane and into xs (-1: none); rounds
  // of NTS tasks the item needs
  int xt_src[XTMAX];
  int xt_dst[XTMAX];
  int nxt;
};

__device__ __forceinline__ void load_plane(const Item &it, int c, double *S0) {
  const bool zok = c >= it.nlo_z && c <= it.nhi_z;
  const double *pb = it.cbase + (int64_t)(c - it.clo_z) * it.cplane;
#pragma unroll
  for (int i = 0; i < LDMAX; ++i) {
    if (i >= it.nld)
      break;
    if (it.ld_soff[i] < 0)
      continue;
    const bool ok = zok && it.ld_goff[i] >= 0;
    cp_async8(S0 + it.ld_soff[i], ok ? pb + it.ld_goff[i] : it.cbase, ok ? 8 : 0);
  }
}

// The stencil kinds of an instantiation per direction; [ZLO, ZHI] is the z
// kind's window (coarse planes relative to the centre).
template <class KV, class KC, int CM> struct Kinds {
  using KX = std::conditional_t<(CM & 4) != 0, KC, KV>;
  using KY = std::conditional_t<(CM & 2) != 0, KC, KV>;
  using KZ = std::conditional_t<(CM & 1) != 0, KC, KV>;
  static constexpr int ZLO = KZ::RLO, ZHI = KZ::RHI;
};

// Streams one item.  The ring covers the z kind's window [ZLO, ZHI].
template <class KV, class KC, int CM>
__device__ __forceinline__ void stream_item(Shared &sh, const Item &it) {
  using KX = typename Kinds<KV, KC, CM>::KX;
  using KY = typename Kinds<KV, KC, CM>::KY;
  using KZ = typename Kinds<KV, KC, CM>::KZ;
  constexpr int ZLO = KZ::RLO, ZHI = KZ::RHI;
  constexpr int L = ZHI - ZLO + 1;
  double ring[L][UPT][FYT];
#pragma unroll
  for (int d = 0; d < DPF; ++d) {
    if (it.c_first + d <= it.c_last)
      load_plane(it, it.c_first + d, sh.s0[d]);
    cp_async_commit();
  }
  int slot = 0;
  for (int c0 = it.c_first; c0 <= it.c_last; c0 += L) {
#pragma unroll
    for (int ph = 0; ph < L; ++ph) {
      const int c = c0 + ph;
      if (c > it.c_last)
        break;
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
#pragma unroll
      for (int k = 0; k < XTMAX; ++k) {
        if (k >= it.nxt)
          break;
        if (it.xt_src[k] < 0)
          continue;
        xtask<KX>(sh.s0[slot] + it.xt_src[k], sh.xs + it.xt_dst[k]);
      }
      __syncthreads();
      // ring slot ph takes plane c; logical position i (0 oldest) is slot
      // (ph + 1 + i) % L
      // (units without a column read a valid part of xs and are never
      // stored: no branch, so the compiler can interleave both units' work)
#pragma unroll
      for (int q = 0; q < UPT; ++q) {
        double y[FYT];
        ypass<KY>(sh.xs + it.ysrc[q], it.pxw, y);
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
      if (++slot == NRING)
        slot = 0;
    }
  }
  __syncthreads(); // the next item reuses the plane ring and xs
}

// Geometry of work item (x chunk, unit block, z chunk, comp) of box b, for
// the z kind's streaming window [zwlo, zwhi].
// The item's units are the unit block's consecutive (unit row, fine x)
// columns of the x chunk, flattened x fastest; thread t owns unit t.
// Returns false if the block holds no unit (box mode, narrow last chunk).
__device__ __forceinline__ bool make_item(const BoxDesc &b, int xchunk, int ublock, int zchunk,
                                          int comp, int zwlo, int zwhi, Item &it) {
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
    const int u = u0 + (int)threadIdx.x + q * NTS;
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
  // coarse plane window: NR rows x Wx columns
  const int n = NR * Wx;
  it.nld = (n + NTS - 1) / NTS;
#pragma unroll
  for (int i = 0; i < LDMAX; ++i) {
    const int e = threadIdx.x + i * NTS;
    it.ld_soff[i] = -1;
    it.ld_goff[i] = -1;
    if (e < n) {
      const int y = e / Wx, x = e - y * Wx;
      it.ld_soff[i] = y * P0 + x;
      const int gx = cxb + x, gy = cyb + y;
      if (gx >= b.nlo[0] && gx <= b.nhi[0] && gy >= b.nlo[1] && gy <= b.nhi[1])
        it.ld_goff[i] = (gy - b.clo[1]) * b.cnx + (gx - b.clo[0]);
    }
  }
  // x-pass tasks: NR rows x nseg segments, rows fastest
  const int nt = NR * nseg;
  it.nxt = (nt + NTS - 1) / NTS;
#pragma unroll
  for (int k = 0; k < XTMAX; ++k) {
    const int t = threadIdx.x + k * NTS;
    it.xt_src[k] = -1;
    it.xt_dst[k] = -1;
    if (t < nt) {
      const int sg = t / NR, r = t - sg * NR;
      it.xt_src[k] = r * P0 + sg * (XB / 2);
      it.xt_dst[k] = r * it.pxw + sg * XB;
    }
  }
  return true;
}

template <class KV, class KC, int CM>
__device__ __forceinline__ void run_item(Shared &sh, const BoxDesc &b, int xchunk, int ublock,
                                         int zchunk, int comp) {
  Item it;
  // uniform over the CTA: an empty block is skipped by every thread
  if (make_item(b, xchunk, ublock, zchunk, comp, Kinds<KV, KC, CM>::ZLO, Kinds<KV, KC, CM>::ZHI,
                it))
    stream_item<KV, KC, CM>(sh, it);
}

constexpr int BOX_WORDS = (int)(sizeof(BoxDesc) / sizeof(int));
static_assert(BOX_WORDS <= NTS, "one thread per descriptor word");

// Box mode (items == nullptr): the items of box b (x tile, y tile, z chunk,
// component) strided over the grid.  Level mode: items from a device work
// list (sorted by cost, largest first) taken by persistent CTAs from a
// counter;
// the descriptors of the next item are loaded into registers while the
// current item streams, so no global-memory latency sits between two items.
// Two CTAs of 256 threads (four of 128) per SM, at most 128 registers,
// except the order-7 z kinds whose register ring (8 or 9 planes) needs more:
// half as many.
template <class KV, class KC, int CM>
__global__ void __launch_bounds__(NTS, (Kinds<KV, KC, CM>::ZHI - Kinds<KV, KC, CM>::ZLO >= 7 ? 1 : 2) * (256 / NTS))
    stream_kernel(const BoxDesc b, const BoxDesc *__restrict__ boxes,
                  const TileRef *__restrict__ items, int nitems, int *__restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[]; // sizeof(Shared) bytes
  Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
  __shared__ BoxDesc box_s;
  if (!items) {
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const int xchunk = item % b.ntile[0];
      int r = item / b.ntile[0];
      const int ublock = r % b.ntile[1];
      r /= b.ntile[1];
      const int zchunk = r % b.ntile[2];
      const int comp = r / b.ntile[2];
      run_item<KV, KC, CM>(sh, b, xchunk, ublock, zchunk, comp);
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
    run_item<KV, KC, CM>(sh, box_s, t_cur.tx, t_cur.ty, t_cur.tz, t_cur.comp);
    if (nxt >= nitems) {
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
