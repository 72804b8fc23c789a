// Transpose of the separable linear prolongations, streaming gather form (no
// atomics).
//
// P = Pz Py Px (the x pass first) with 1-D maps P_d, so P^T = Px^T Py^T Pz^T
// and the three 1-D transposes can be applied in any order.  In 1-D, fine
// point f = 2 cc + off reads coarse cc + o with weight w(off, o), o in the
// stencil of off; so coarse point c gathers
//   crse_bar(c) = sum_{off, o} w(off, o) fine_bar(2 (c - o) + off).
// With the fine window of c starting at 2 (c - RHI), tap m = 2 (RHI - o) + off
// (0 <= m <= 2 (RHI - RLO) + 1) of that window has weight w(m & 1, RHI - m/2).
//
// A work item is a tile of up to NU coarse (x, y) columns of the coarse box
// over a chunk of coarse z, one component.  The CTA streams the fine z planes
// that reach the chunk through a ring of shared-memory buffers holding the
// tile's fine footprint (the region's fine points of it; the rest of the
// footprint is zero, set once per item):
//   load   fine plane fz + DPF (asynchronous 8-byte copies, one warp per row);
//   x^T    G(cx, fy) for the tile's coarse x and every footprint row, XB
//          coarse x per task from a register window of the fine row, into
//          shared memory (column major: the y taps of a column are adjacent);
//   y^T    each thread gathers g(cx, cy) of its UPT columns;
//   z^T    each thread accumulates w(off, o) g into the coarse planes
//          cc + o that fine plane fz = 2 cc + off reaches (a register ring of
//          L = RHI - RLO + 1 partial sums); when cc moves on, coarse plane
//          cc + RLO is complete and is stored.
// Every coarse point of the coarse box is written once (zero where no region
// point reads it); sums run in a fixed order, so results are deterministic.
// Fine data is read once per item plus the tile's footprint halo (served by
// the L2 when neighbouring tiles stream together).
#include <type_traits>

#include "cx_internal.h"
#include "cx_stencils.cuh"
#include "stream_pairs.h"

namespace cxb {
namespace {

// 1-D weight of coarse offset o for a fine point with offset off: the
// coefficient multiplying v[o] in the kind's linear form (0 outside its
// stencil).  Same stencils as cx_stencils.cuh (impl.hxx:396-878).
template <class K> struct Weight;

template <int P> struct Weight<VcPoly<P>> {
  CXB_HD static constexpr double w(int off, int o) {
    if (off == 0)
      return o == 0 ? 1.0 : 0.0;
    constexpr int i0 = (P + 1) / 2 - 1;
    if (o < -i0 || o > P - i0)
      return 0.0;
    return vc_poly_c<P>(o + i0); // symmetric pairs share c(i) = c(P - i)
  }
};
template <int P> struct Weight<CcPoly<P>> {
  CXB_HD static constexpr double w(int off, int o) {
    constexpr int I0 = (P + 1) / 2;
    if (off == 0) {
      const int i = o + I0;
      return i >= 0 && i <= P ? cc_poly_c<P>(i) : 0.0;
    }
    const int i = o + I0 - P % 2;
    return i >= 0 && i <= P ? cc_poly_c<P>(P - i) : 0.0;
  }
};
template <int P> struct Weight<CcCons<P>> {
  CXB_HD static constexpr double w(int off, int o) {
    constexpr int I0 = (P + 1) / 2;
    if constexpr (P % 2 == 0) {
      if (o == 0)
        return cc_cons_c<P>(P / 2);
      if (o < -P / 2 || o > P / 2)
        return 0.0;
      const double c = o < 0 ? cc_cons_c<P>(o + I0) : cc_cons_c<P>(P - o - I0);
      return (o < 0) == (off == 0) ? c : -c;
    } else {
      if (off == 0) {
        const int i = o + I0;
        return i >= 0 && i <= P ? cc_cons_c<P>(i) : 0.0;
      }
      const int i = (P + 1) / 2 - o;
      return i >= 0 && i <= P ? cc_cons_c<P>(i) : 0.0;
    }
  }
};
template <int P> struct Weight<VcCons<P>> {
  CXB_HD static constexpr double w(int off, int o) {
    if (off == 0)
      return o == 0 ? 1.0 : 0.0;
    if (P == 0)
      return 0.0;
    return o == 0 || o == 1 ? 0.5 : 0.0;
  }
};

// weight of tap m of a coarse point's fine window
template <class K> CXB_HD constexpr double wtap(int m) {
  return Weight<K>::w(m & 1, K::RHI - (m >> 1));
}
template <class K> constexpr int DK = K::RHI - K::RLO;

constexpr int NT = 256;        // threads per CTA
constexpr int UPT = 2;         // coarse columns per thread
constexpr int NU = NT * UPT;   // coarse columns per item at most
constexpr int TMAX = 64;       // tile extent in x or y at most
constexpr int DPF = 2;         // fine planes prefetched ahead
constexpr int NBUF = DPF + 1;  // shared fine-plane ring
constexpr int XB = 4;          // coarse x per x^T task

// Footprint of a TX x TY tile for stencil spread D (<= DM): rows, row pitch
// (odd), and x^T column pitch (odd).
CXB_HD constexpr int fp_rows(int ty, int dm) { return 2 * ty + 2 * dm; }
CXB_HD constexpr int fp_pitch(int tx, int dm) { return (2 * tx + 2 * dm) | 1; }
CXB_HD constexpr int g_pitch(int ty, int dm) { return fp_rows(ty, dm) | 1; }
CXB_HD constexpr int tile_ty(int tx) { return NU / tx < TMAX ? NU / tx : TMAX; }
CXB_HD constexpr int max_fp(int dm, int what) {
  int m = 0;
  for (int tx = 1; tx <= TMAX; ++tx) {
    const int ty = tile_ty(tx);
    const int v = what == 0 ? fp_rows(ty, dm) * fp_pitch(tx, dm) : tx * g_pitch(ty, dm);
    m = v > m ? v : m;
  }
  return m;
}

template <class KV, class KC> struct AdjPair {
  static constexpr int DM = DK<KV> > DK<KC> ? DK<KV> : DK<KC>;
  static constexpr int FP = max_fp(DM, 0); // fine footprint plane (doubles)
  static constexpr int GP = max_fp(DM, 1); // x^T result (doubles)
  static constexpr size_t SMEM = sizeof(double) * (size_t)(NBUF * FP + GP + 2 * XB);
};

__device__ __forceinline__ void cp_async8(double *sdst, const double *gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_dpf() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(DPF) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

struct AdjTiling {
  int tx, ty, tz;    // coarse tile extents (x, y) and coarse z per item
  int ntx, nty, ntz; // tiles per direction
};

// Per-item geometry.
struct AItem {
  int cx0, cy0, cz0, cz1; // tile origin (coarse, absolute), coarse z chunk
  int txe, tye;           // tile extent
  int fxo, fyo;           // footprint origin (fine, absolute)
  int fw, fh, fpw, gpw;   // footprint width, rows, row pitch; x^T column pitch
  int ax, bx, ay, by;     // region part of the footprint (local, inclusive)
  int fa, fb;             // fine planes streamed
  const double *fbase;    // fine component base at (flo)
  int fnx;
  int64_t fplane;
  int flo_z;
};

// x^T task: XB coarse x of one footprint row from a register window; only
// the first n are stored (the window of the last task of a row may run up to
// 2 (XB - 1) points past the footprint: those reach only unstored results,
// and the shared allocation is padded for them).
template <class K>
__device__ __forceinline__ void xt_task(const double *__restrict__ src, double *__restrict__ dst,
                                        int gpw, int n) {
  constexpr int D = DK<K>, WIN = 2 * XB + 2 * D;
  double v[WIN];
#pragma unroll
  for (int i = 0; i < WIN; ++i)
    v[i] = src[i];
#pragma unroll
  for (int t = 0; t < XB; ++t) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m <= 2 * D + 1; ++m) {
      const double w = wtap<K>(m);
      if (w != 0.0)
        acc = fma(w, v[2 * t + m], acc);
    }
    if (t < n)
      dst[t * gpw] = acc;
  }
}

// y^T of one column: the 2 D + 2 taps are adjacent in the x^T result.
template <class K> __device__ __forceinline__ double yt_col(const double *__restrict__ src) {
  constexpr int D = DK<K>;
  double acc = 0.0;
#pragma unroll
  for (int m = 0; m <= 2 * D + 1; ++m) {
    const double w = wtap<K>(m);
    if (w != 0.0)
      acc = fma(w, src[m], acc);
  }
  return acc;
}

template <class KV, class KC, class KZ>
__device__ __forceinline__ void adj_item(double *fbuf, double *gbuf, const BoxDesc &b,
                                         const AItem &it, double *__restrict__ out) {
  constexpr int FP = AdjPair<KV, KC>::FP;
  constexpr int L = DK<KZ> + 1;
  const int ccx = kind_info(b.kind[0]).cent, ccy = kind_info(b.kind[1]).cent;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // zero the footprint of every buffer once: points outside the region stay 0
  for (int k = 0; k < NBUF; ++k)
    for (int e = tid; e < it.fh * it.fpw; e += NT)
      fbuf[k * FP + e] = 0.0;
  __syncthreads();

  auto load = [&](int fz, int k) {
    const double *pl = it.fbase + (int64_t)(fz - it.flo_z) * it.fplane;
    double *S = fbuf + k * FP;
    for (int r = it.ay + warp; r <= it.by; r += NT / 32) {
      const double *row = pl + (int64_t)(it.fyo + r - b.flo[1]) * it.fnx + (it.fxo - b.flo[0]);
      for (int c = it.ax + lane; c <= it.bx; c += 32)
        cp_async8(S + r * it.fpw + c, row + c);
    }
  };

  // this thread's columns
  int ui[UPT], uj[UPT];
  bool act[UPT];
#pragma unroll
  for (int q = 0; q < UPT; ++q) {
    const int u = tid + q * NT;
    uj[q] = u / it.txe;
    ui[q] = u - uj[q] * it.txe;
    act[q] = uj[q] < it.tye;
  }
  double acc[UPT][L];
#pragma unroll
  for (int q = 0; q < UPT; ++q)
#pragma unroll
    for (int k = 0; k < L; ++k)
      acc[q][k] = 0.0;
  const int64_t cplane = (int64_t)b.cnx * b.cny;
  int cc = it.cz0 - KZ::RHI; // acc[q][k] <-> coarse plane cc + RLO + k
  auto advance_to = [&](int target) {
    for (; cc < target; ++cc) {
      const int cz = cc + KZ::RLO;
      if (cz >= it.cz0 && cz <= it.cz1) {
#pragma unroll
        for (int q = 0; q < UPT; ++q)
          if (act[q])
            out[(int64_t)(cz - b.clo[2]) * cplane + (int64_t)(it.cy0 + uj[q] - b.clo[1]) * b.cnx +
                (it.cx0 + ui[q] - b.clo[0])] = acc[q][0];
      }
#pragma unroll
      for (int q = 0; q < UPT; ++q) {
#pragma unroll
        for (int k = 0; k < L - 1; ++k)
          acc[q][k] = acc[q][k + 1];
        acc[q][L - 1] = 0.0;
      }
    }
  };

  const int nseg = (it.txe + XB - 1) / XB;
  const int ntask = nseg * it.fh;
#pragma unroll
  for (int d = 0; d < DPF; ++d) {
    if (it.fa + d <= it.fb)
      load(it.fa + d, d);
    cp_async_commit();
  }
  int slot = 0;
  for (int fz = it.fa; fz <= it.fb; ++fz) {
    {
      int ls = slot + DPF;
      if (ls >= NBUF)
        ls -= NBUF;
      if (fz + DPF <= it.fb)
        load(fz + DPF, ls);
      cp_async_commit();
    }
    cp_async_wait_dpf();
    __syncthreads();
    const double *S = fbuf + slot * FP;
    for (int k = tid; k < ntask; k += NT) {
      const int s = k / it.fh, r = k - s * it.fh;
      const int n = min(XB, it.txe - s * XB);
      const double *src = S + r * it.fpw + 2 * XB * s;
      double *dst = gbuf + (s * XB) * it.gpw + r;
      if (ccx)
        xt_task<KC>(src, dst, it.gpw, n);
      else
        xt_task<KV>(src, dst, it.gpw, n);
    }
    __syncthreads();
    advance_to(fz >> 1);
    const int off = fz & 1;
#pragma unroll
    for (int q = 0; q < UPT; ++q) {
      if (!act[q])
        continue;
      const double *src = gbuf + ui[q] * it.gpw + 2 * uj[q];
      const double g = ccy ? yt_col<KC>(src) : yt_col<KV>(src);
#pragma unroll
      for (int k = 0; k < L; ++k) {
        const double w0 = Weight<KZ>::w(0, KZ::RLO + k), w1 = Weight<KZ>::w(1, KZ::RLO + k);
        const double w = off ? w1 : w0;
        if (w0 != 0.0 || w1 != 0.0)
          acc[q][k] = fma(w, g, acc[q][k]);
      }
    }
    if (++slot == NBUF)
      slot = 0;
  }
  advance_to(it.cz1 - KZ::RLO + 1);
  cp_async_wait_all();
  __syncthreads(); // the next item reuses the shared buffers
}

template <class KV, class KC>
__global__ void __launch_bounds__(NT, AdjPair<KV, KC>::SMEM > 110 * 1024 ? 1 : 2)
    adjoint_kernel(const BoxDesc b, const AdjTiling t, double *crse_bar) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *fbuf = reinterpret_cast<double *>(smem_raw);
  double *gbuf = fbuf + NBUF * AdjPair<KV, KC>::FP;
  constexpr int DM = AdjPair<KV, KC>::DM;
  const int nitems = t.ntx * t.nty * t.ntz * b.ncomp;
  const int kx = b.kind[0], ky = b.kind[1];
  const bool ccz = kind_info(b.kind[2]).cent == CC;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    int r = item;
    const int xt = r % t.ntx;
    r /= t.ntx;
    const int yt = r % t.nty;
    r /= t.nty;
    const int zt = r % t.ntz;
    const int comp = r / t.ntz;
    AItem it;
    it.cx0 = b.clo[0] + xt * t.tx;
    it.cy0 = b.clo[1] + yt * t.ty;
    it.cz0 = b.clo[2] + zt * t.tz;
    const int chi0 = b.clo[0] + b.cnx - 1, chi1 = b.clo[1] + b.cny - 1;
    const int chi2 = b.clo[2] + (int)(b.cnp / ((int64_t)b.cnx * b.cny)) - 1;
    it.txe = min(t.tx, chi0 - it.cx0 + 1);
    it.tye = min(t.ty, chi1 - it.cy0 + 1);
    it.cz1 = min(it.cz0 + t.tz - 1, chi2);
    const int rhx = sep_rhi(kx), rhy = sep_rhi(ky);
    const int dx = rhx - sep_rlo(kx), dy = rhy - sep_rlo(ky);
    it.fxo = 2 * (it.cx0 - rhx);
    it.fyo = 2 * (it.cy0 - rhy);
    it.fw = 2 * it.txe + 2 * dx;
    it.fh = 2 * it.tye + 2 * dy;
    it.fpw = fp_pitch(it.txe, DM);
    it.gpw = g_pitch(it.tye, DM);
    it.ax = max(0, b.rlo[0] - it.fxo);
    it.bx = min(it.fw - 1, b.rhi[0] - it.fxo);
    it.ay = max(0, b.rlo[1] - it.fyo);
    it.by = min(it.fh - 1, b.rhi[1] - it.fyo);
    const int rlz = ccz ? KC::RLO : KV::RLO, rhz = ccz ? KC::RHI : KV::RHI;
    it.fa = max(2 * (it.cz0 - rhz), b.rlo[2]);
    it.fb = min(2 * (it.cz1 - rlz) + 1, b.rhi[2]);
    if (it.ax > it.bx || it.ay > it.by) { // no region point in the footprint
      it.fa = 1;
      it.fb = 0;
    }
    it.fbase = b.fine + comp * b.fnp;
    it.fnx = b.fnx;
    it.fplane = (int64_t)b.fnx * b.fny;
    it.flo_z = b.flo[2];
    double *out = crse_bar + comp * b.cnp;
    if (ccz)
      adj_item<KV, KC, KC>(fbuf, gbuf, b, it, out);
    else
      adj_item<KV, KC, KV>(fbuf, gbuf, b, it, out);
  }
}

using AdjFn = void (*)(const BoxDesc, const AdjTiling, double *);

// Kernel and shared-memory size of a pair (nullptr for the nonlinear ones).
template <class V, class C> AdjFn adj_fn(size_t *smem) {
  if constexpr (std::is_same_v<C, CcMinmod>) {
    return nullptr;
  } else {
    *smem = AdjPair<V, C>::SMEM;
    return adjoint_kernel<V, C>;
  }
}

AdjFn adj_kernel(int pair, size_t *smem) {
  switch (pair) {
#define CXB_ADJ_CASE(I, V, C, KVI, KCI)                                        \
  case I:                                                                      \
    return adj_fn<V, C>(smem);
    CXB_STREAM_PAIRS(CXB_ADJ_CASE)
#undef CXB_ADJ_CASE
  default:
    break;
  }
  return nullptr;
}

bool g_adj_attr[kStreamPairs] = {};
int g_adj_grid[kStreamPairs] = {};

AdjTiling adj_tiling(const BoxDesc &b, int min_items) {
  AdjTiling t;
  const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
  t.ntx = (b.cnx + TMAX - 1) / TMAX;
  t.tx = (b.cnx + t.ntx - 1) / t.ntx;
  const int tymax = tile_ty(t.tx);
  t.nty = (b.cny + tymax - 1) / tymax;
  t.ty = (b.cny + t.nty - 1) / t.nty;
  // coarse z per item: up to 48 (the z footprint costs 2 (RHI - RLO) fine
  // planes per item), shorter (down to 8) until the box fills min_items CTAs
  int maxz = 48;
  const int64_t xy = (int64_t)t.ntx * t.nty * b.ncomp;
  while (maxz > 8 && xy * ((cnz + maxz - 1) / maxz) < min_items)
    maxz /= 2;
  t.ntz = (cnz + maxz - 1) / maxz;
  t.tz = (cnz + t.ntz - 1) / t.ntz;
  t.ntz = (cnz + t.tz - 1) / t.tz;
  return t;
}

} // namespace

cudaError_t launch_prolong_adjoint_box(const BoxDesc &b, int per_group, double *crse_bar,
                                       cudaStream_t s) {
  (void)per_group; // linear operators: per-group and per-variable agree
  if (b.ncomp <= 0 || b.cnp <= 0)
    return cudaSuccess;
  const int pair = stream_pair_of(b.kind[0], b.kind[1], b.kind[2]);
  size_t smem = 0;
  AdjFn k = pair >= 0 ? adj_kernel(pair, &smem) : nullptr;
  if (!k)
    return cudaErrorInvalidValue;
  if (!g_adj_attr[pair]) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
      return e;
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem);
    g_adj_grid[pair] = sms * (per_sm > 0 ? per_sm : 1);
    g_adj_attr[pair] = true;
  }
  const AdjTiling t = adj_tiling(b, g_adj_grid[pair]);
  const int64_t n64 = (int64_t)t.ntx * t.nty * t.ntz * b.ncomp;
  if (n64 > INT32_MAX)
    return cudaErrorInvalidValue;
  const int n = (int)n64;
  k<<<n < g_adj_grid[pair] ? n : g_adj_grid[pair], NT, smem, s>>>(b, t, crse_bar);
  return cudaGetLastError();
}

} // namespace cxb
