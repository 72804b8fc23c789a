// Transpose of the separable linear prolongations, streaming gather form (no
// atomics), for one box per launch or a whole level per persistent launch.
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
// tile's fine footprint (its region points; the rest of the footprint reads
// as zero):
//   load   fine plane fz + DPF: one thread per footprint row issues one bulk
//          (TMA) copy of the row's 16-byte aligned middle, completing on the
//          buffer's mbarrier (each row is placed in shared memory with the
//          parity of its global address, so both ends of the copy are 16-byte
//          aligned); the odd first/last point of a row takes an 8-byte copy.
//          The rows are dealt across the warps: a warp's bulk copies are
//          issued one lane after the other, so spreading them shortens the
//          issue;
//   y^T    H(fx, cy) for every footprint column and the tile's coarse y,
//          YB coarse y per task from a register window down the fine column
//          (consecutive lanes read consecutive fine x of a row), into shared
//          memory split by the parity of fx; y first, because the tiles are
//          wider than tall and the first pass pays for the other direction's
//          halo at fine resolution;
//   x^T    each thread gathers g(cx, cy) of its UPT columns from H (its taps
//          are adjacent in the two parity halves);
//   z^T    each thread accumulates w(off, o) g into the coarse planes
//          cc + o that fine plane fz = 2 cc + off reaches (a register ring of
//          L = RHI - RLO + 1 partial sums); when cc moves on, coarse plane
//          cc + RLO is complete and is stored.
// Every coarse point of the coarse box is written once (zero where no region
// point reads it); sums run in a fixed order, so results are deterministic.
// Fine data is read from HBM once; the footprint halo of a tile is read again
// by its neighbours, from the L2 (tiles of a box are dealt together).
#pragma once
#include <type_traits>

#include "cx_internal.h"
#include "cx_stencils.cuh"
#include "cx_async.cuh"
#include "stream_pairs.h"

namespace cxb {
namespace adj {


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
// partial sum (0 or 1) that tap m joins: the taps of nonzero weight
// alternate, so two independent FMA chains of equal length
template <class K> CXB_HD constexpr int wchain(int m) {
  int n = 0;
  for (int i = 0; i < m; ++i)
    n += wtap<K>(i) != 0.0;
  return n & 1;
}
template <class K> constexpr int DK = K::RHI - K::RLO;

// A CTA of NT threads streams a tile of up to NT x UPT coarse columns (at
// most TMAX per direction), two planes ahead; two CTAs per SM where the
// shared memory allows (all but the order-7 pairs).  Measured on the
// differentiated level (64 boxes of 32-96 coarse points per direction), this
// beats one CTA of 512 threads with larger tiles (less footprint halo) and
// one plane ahead: the time goes into waiting for the copies, and more CTAs
// and planes in flight hide more of it.
constexpr int NT = 256;       // threads per CTA
constexpr int TMAX = 64;      // tile extent in x or y at most
constexpr int DPF = 2;        // fine planes prefetched ahead
constexpr int NBUF = DPF + 1; // shared fine-plane ring
constexpr int YB = 6;         // coarse y per y^T task

// Footprint of a TX x TY tile for stencil spread D <= DM: rows, row pitch
// (odd, one more than the widest footprint row: a row is placed at offset 0
// or 1 to match its global address parity).  The y^T result H keeps the
// even and the odd footprint columns in two halves of TY rows of TX + DM
// points; the second half starts 8 doubles past a multiple of 16, so the
// even and odd lanes of a warp's stores fall in different banks.
CXB_HD constexpr int fp_rows(int ty, int dm) { return 2 * ty + 2 * dm; }
CXB_HD constexpr int fp_pitch(int tx, int dm) { return 2 * tx + 2 * dm + 1; }
CXB_HD constexpr int h_pitch(int tx, int dm) { return tx + dm; }
CXB_HD constexpr int h_half(int tx, int ty, int dm) {
  return (ty * h_pitch(tx, dm) + 15) / 16 * 16 + 8;
}
CXB_HD constexpr int tile_ty(int tx, int nu) { return nu / tx < TMAX ? nu / tx : TMAX; }
// what: 0 footprint plane, 1 y^T result, 2 y^T tasks, 3 footprint plane plus
// the rows the last y^T window of a column may read past it
CXB_HD constexpr int max_fp(int dm, int nu, int what) {
  int m = 0;
  for (int tx = 1; tx <= TMAX; ++tx) {
    const int ty = tile_ty(tx, nu);
    const int v = what == 0   ? fp_rows(ty, dm) * fp_pitch(tx, dm)
                  : what == 1 ? 2 * h_half(tx, ty, dm)
                  : what == 2 ? (2 * tx + 2 * dm) * ((ty + YB - 1) / YB)
                              : (fp_rows(ty, dm) + 2 * YB) * fp_pitch(tx, dm);
    m = v > m ? v : m;
  }
  return m;
}
// coarse columns per thread
CXB_HD constexpr int upt_of(int) { return 2; }

template <class KV, class KC> struct AdjPair {
  static constexpr int DM = DK<KV> > DK<KC> ? DK<KV> : DK<KC>;
  static constexpr int UPT = upt_of(DM);
  static constexpr int NU = NT * UPT; // coarse columns per item at most
  static constexpr int FP = (max_fp(DM, NU, 0) + 1) & ~1; // fine footprint plane (even: 16-byte buffers)
  static constexpr int GP = max_fp(DM, NU, 1);            // y^T result
  static constexpr int XTMAX = (max_fp(DM, NU, 2) + NT - 1) / NT; // y^T tasks per thread
  // the last y^T window of a column may read up to 2 YB - 2 rows past the
  // footprint (into the next buffer, or into H for the last one; only
  // results that are not stored use them): the allocation covers them
  static constexpr int OVER = max_fp(DM, NU, 3) - FP;
  static constexpr size_t SMEM =
      sizeof(double) * (size_t)(NBUF * FP + (GP > OVER ? GP : OVER) + 2);
  static_assert(SMEM + 1024 <= 227 * 1024, "shared memory per CTA");
  static constexpr int OCC = SMEM + 2048 <= 113 * 1024 ? 2 : 1; // CTAs per SM
  static_assert(XTMAX <= 3, "y^T task registers");
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

// Set when a bounded wait gave up (read and cleared by cx_check_device);
// every translation unit that instantiates the kernels has its own copy.
// g_adj_wait_limit: cycles a wait for a plane's copies polls before giving
// up (kWaitCycles, about a second, unless cx_debug_set_wait_limit lowered it
// to force the give-up path in a test); the copies still in flight when a CTA
// gives up are always waited for with the default bound.
namespace {
__device__ int g_adj_timeout = 0;
__device__ long long g_adj_wait_limit = kWaitCycles;
}

// y^T task: YB coarse y of one footprint column from a register window
// down the column; tap i is fine row i of the window, at e + i fpw for even
// i and o + i fpw for odd i (the two row parities of the footprint).  Only
// the first n results are stored, hp apart (the window of the last task of
// a column may run past the footprint: those rows reach only unstored
// results).
template <class K>
__device__ __forceinline__ void yt_task(const double *__restrict__ e, const double *__restrict__ o,
                                        int fpw, double *__restrict__ dst, int hp, int n) {
  constexpr int D = DK<K>, WIN = 2 * YB + 2 * D;
  double v[WIN];
#pragma unroll
  for (int i = 0; i < WIN; ++i)
    v[i] = (i & 1 ? o : e)[i * fpw];
#pragma unroll
  for (int t = 0; t < YB; ++t) {
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m <= 2 * D + 1; ++m) {
      const double w = wtap<K>(m);
      if (w != 0.0)
        acc = fma(w, v[2 * t + m], acc);
    }
    if (t < n)
      dst[t * hp] = acc;
  }
}

// x^T of one column from H: tap m is in the half of parity m & 1, m / 2
// past the column's start.
template <class K>
__device__ __forceinline__ double xt_col(const double *__restrict__ h0,
                                         const double *__restrict__ h1) {
  constexpr int D = DK<K>;
  double acc = 0.0;
#pragma unroll
  for (int m = 0; m <= 2 * D + 1; ++m) {
    const double w = wtap<K>(m);
    if (w != 0.0)
      acc = fma(w, (m & 1 ? h1 : h0)[m >> 1], acc);
  }
  return acc;
}

// z^T: fine plane with offset OFF adds w(OFF, RLO + k) g to partial sum k.
template <class K, int OFF, int L>
__device__ __forceinline__ void zt_add(double (&acc)[L], double g) {
#pragma unroll
  for (int k = 0; k < L; ++k) {
    const double w = Weight<K>::w(OFF, K::RLO + k);
    if (w != 0.0)
      acc[k] = fma(w, g, acc[k]);
  }
}

// One item: coarse tile (xt, yt), coarse z chunk zt, component comp of box b,
// for stencil kinds KX, KY, KZ per direction (buffers sized for the pair).
// Returns false if a bounded wait gave up (the CTA then stops).
template <class KV, class KC, class KX, class KY, class KZ>
__device__ __forceinline__ bool adj_item(long long limit, double *fbuf, double *gbuf, uint64_t *mbar,
                                         int *s_fail,
                                         uint32_t &phase, const BoxDesc &bd, int xt, int yt, int zt,
                                         int comp) {
  constexpr int FP = AdjPair<KV, KC>::FP, DM = AdjPair<KV, KC>::DM;
  constexpr int UPT = AdjPair<KV, KC>::UPT, XTMAX = AdjPair<KV, KC>::XTMAX;
  constexpr int L = DK<KZ> + 1;
  const int tid = threadIdx.x;
  // the descriptor fields used below, in registers
  const int cnx = bd.cnx, cny = bd.cny, fnx = bd.fnx;
  const int64_t cplane = (int64_t)cnx * cny, fplane = (int64_t)fnx * bd.fny;
  const int cnz = (int)(bd.cnp / cplane);
  const int clo0 = bd.clo[0], clo1 = bd.clo[1], clo2 = bd.clo[2];
  const int cx0 = clo0 + xt * bd.at[0], cy0 = clo1 + yt * bd.at[1], cz0 = clo2 + zt * bd.at[2];
  const int txe = min(bd.at[0], clo0 + cnx - cx0), tye = min(bd.at[1], clo1 + cny - cy0);
  const int cz1 = min(cz0 + bd.at[2] - 1, clo2 + cnz - 1);
  constexpr int rhx = KX::RHI, dx = DK<KX>;
  constexpr int rhy = KY::RHI, dy = DK<KY>;
  const int fxo = 2 * (cx0 - rhx), fyo = 2 * (cy0 - rhy);
  const int fw = 2 * txe + 2 * dx, fh = 2 * tye + 2 * dy;
  const int fpw = fp_pitch(txe, DM), hp = h_pitch(txe, DM), hoff = h_half(txe, tye, DM);
  const int ax = max(0, bd.rlo[0] - fxo), bx = min(fw - 1, bd.rhi[0] - fxo);
  const int ay = max(0, bd.rlo[1] - fyo), by = min(fh - 1, bd.rhi[1] - fyo);
  int fa = max(2 * (cz0 - KZ::RHI), bd.rlo[2]);
  int fb = min(2 * (cz1 - KZ::RLO) + 1, bd.rhi[2]);
  if (ax > bx || ay > by) { // no region point in the footprint
    fa = 1;
    fb = 0;
  }
  const double *fcomp = bd.fine + comp * bd.fnp; // fine_bar component
  const uint64_t fcomp8 = (uint64_t)(uintptr_t)fcomp >> 3;
  // element offset of footprint point (0, 0) of fine plane fz in the component
  const int64_t org = (int64_t)(fyo - bd.flo[1]) * fnx + (fxo - bd.flo[0]) - (int64_t)bd.flo[2] * fplane;
  const int dpar = (fnx + fpw) & 1; // row r sits at r fpw + ((parity of plane) + r dpar) % 2
  const bool edge = ax > 0 || bx < fw - 1; // region rows have columns outside the region
  double *out = bd.cbar + comp * bd.cnp;

  // this thread's columns: x^T source in H (-1: none), output offset
  int hsrc[UPT], cofs[UPT];
#pragma unroll
  for (int q = 0; q < UPT; ++q) {
    const int u = tid + q * NT;
    const int uj = u / txe, ui = u - uj * txe;
    hsrc[q] = uj < tye ? uj * hp + ui : -1;
    cofs[q] = (cy0 + uj - clo1) * cnx + (cx0 + ui - clo0);
  }
  // this thread's y^T tasks: (footprint column c, group g of YB coarse y),
  // columns fastest; source offset of the window's first row (before the
  // plane's row shift), destination in H, results to store (0: none)
  int ysrc[XTMAX], ydst[XTMAX], yn[XTMAX];
  const int ngrp = (tye + YB - 1) / YB;
#pragma unroll
  for (int k = 0; k < XTMAX; ++k) {
    const int t = tid + k * NT;
    const int g = t / fw, c = t - g * fw;
    yn[k] = g < ngrp ? min(YB, tye - g * YB) : 0;
    ysrc[k] = 2 * YB * g * fpw + c;
    ydst[k] = (c & 1) * hoff + g * YB * hp + (c >> 1);
  }

  // zero every buffer's footprint once: rows outside the region and the
  // columns of region rows outside the region stay zero, except the one
  // column at each end that a copy placed with the other parity wrote (see
  // load)
  for (int k = 0; k < NBUF; ++k)
    for (int e = tid; e < fh * fpw; e += NT)
      fbuf[k * FP + e] = 0.0;
  fence_proxy_async();
  __syncthreads();

  // this thread's footprint row (rows are dealt across the warps: a warp's
  // bulk copies are issued one lane after the other) and its element offset
  // and address parity at fine plane 0
  const int lr = ay + (tid & 31) * (NT / 32) + (tid >> 5); // footprint rows <= NT
  const bool has_row = lr <= by;
  const int64_t rofs0 = org + (int64_t)lr * fnx;
  const int rpar0 = (int)((fcomp8 + (uint64_t)rofs0) & 1);
  const int fpl_odd = (int)(fplane & 1);
  const int rbase = lr * fpw;

  // issue the copies of fine plane fz into buffer k (the buffer's mbarrier
  // receives the bulk bytes; thread 0 arrives once every thread has issued)
  auto load = [&](int fz, int k) {
    double *S = fbuf + k * FP;
    if (has_row) {
      const int par = rpar0 ^ (fz & fpl_odd);
      const int rb = rbase + ((par + rbase) & 1); // same parity as the row's address
      const double *rowg = fcomp + rofs0 + (int64_t)fz * fplane;
      const int c0 = ax + ((par + ax) & 1); // first column with a 16-byte aligned address
      const int nch = (bx - c0 + 1) >> 1;
      if (nch > 0) {
        mbar_expect_tx(mbar + k, 16u * (uint32_t)nch);
        bulk_g2s(S + rb + c0, rowg + c0, 16u * (uint32_t)nch, mbar + k);
      }
      if (c0 > ax)
        cp_async8(S + rb + ax, rowg + ax);
      const int cl = c0 + 2 * nch;
      if (cl <= bx)
        cp_async8(S + rb + cl, rowg + cl);
      if (edge) {
        // a row sits at r fpw + s + c, s = 0 or 1 by plane; copies write
        // c in [ax, bx] only, so with s = 1 the column ax - 1 holds what a
        // plane with s = 0 put at ax, and with s = 0 the column bx + 1 holds
        // what a plane with s = 1 put at bx; every other column outside the
        // region keeps the zero of the item's start
        if (ax > 0)
          S[rb + ax - 1] = 0.0;
        if (bx < fw - 1)
          S[rb + bx + 1] = 0.0;
        fence_proxy_async();
      }
    }
  };

  double acc[UPT][L];
#pragma unroll
  for (int q = 0; q < UPT; ++q)
#pragma unroll
    for (int k = 0; k < L; ++k)
      acc[q][k] = 0.0;
  int cc = cz0 - KZ::RHI; // acc[q][k] <-> coarse plane cc + RLO + k
  auto advance_to = [&](int target) {
    for (; cc < target; ++cc) {
      const int cz = cc + KZ::RLO;
      if (cz >= cz0 && cz <= cz1) {
        double *o = out + (int64_t)(cz - clo2) * cplane;
#pragma unroll
        for (int q = 0; q < UPT; ++q)
          if (hsrc[q] >= 0)
            o[cofs[q]] = acc[q][0];
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

#pragma unroll
  for (int d = 0; d < DPF; ++d) {
    if (fa + d <= fb)
      load(fa + d, d);
    cp_async_commit();
  }
  __syncthreads();
  if (tid == 0)
    for (int d = 0; d < DPF; ++d)
      if (fa + d <= fb)
        mbar_arrive(mbar + d);
  int slot = 0;
  for (int fz = fa; fz <= fb; ++fz) {
    int ls = slot + DPF;
    if (ls >= NBUF)
      ls -= NBUF;
    const bool more = fz + DPF <= fb;
    if (more)
      load(fz + DPF, ls);
    cp_async_commit();
    cp_async_wait_dpf();
    const uint32_t par = (phase >> slot) & 1u;
    // the limit is read once per kernel; a first poll needs no clock
    if (tid == 0 && !(limit > 0 && mbar_try(mbar + slot, par)) &&
        !mbar_wait_bounded(mbar + slot, par, limit)) {
      *s_fail = 1;
      g_adj_timeout = 1;
    }
    __syncthreads();
    if (*s_fail) {
      // stop, once every copy still in flight into this CTA's buffers has
      // landed (each wait bounded by the default): planes fz .. fz + DPF - 1
      // were issued and arrived on earlier, plane fz + DPF was issued just
      // now and is arrived on here; then the 8-byte copies
      if (tid == 0) {
        if (more)
          mbar_arrive(mbar + ls);
        for (int d = 0; d <= DPF && fz + d <= fb; ++d) {
          int k = slot + d;
          if (k >= NBUF)
            k -= NBUF;
          mbar_wait_bounded(mbar + k, (phase >> k) & 1u, kWaitCycles);
        }
      }
      cp_async_wait_all();
      __syncthreads();
      return false;
    }
    if (tid == 0 && more)
      mbar_arrive(mbar + ls); // every thread issued its copies before the barrier
    mbar_try(mbar + slot, par); // completed: acquires the bulk data for this thread
    phase ^= 1u << slot;
    const double *S = fbuf + slot * FP;
    // row shifts of the plane: row r sits at r fpw + (p0 + r dpar) % 2
    const int p0 = (int)((fcomp8 + (uint64_t)(org + (int64_t)fz * fplane)) & 1);
    const int se = p0, so = (p0 + dpar) & 1;
#pragma unroll
    for (int k = 0; k < XTMAX; ++k) {
      if (yn[k] <= 0)
        continue;
      const double *src = S + ysrc[k];
      yt_task<KY>(src + se, src + so, fpw, gbuf + ydst[k], hp, yn[k]);
    }
    __syncthreads();
    advance_to(fz >> 1);
#pragma unroll
    for (int q = 0; q < UPT; ++q) {
      if (hsrc[q] < 0)
        continue;
      const double g = xt_col<KX>(gbuf + hsrc[q], gbuf + hoff + hsrc[q]);
      if (fz & 1)
        zt_add<KZ, 1, L>(acc[q], g);
      else
        zt_add<KZ, 0, L>(acc[q], g);
    }
    if (++slot == NBUF)
      slot = 0;
  }
  advance_to(cz1 - KZ::RLO + 1);
  cp_async_wait_all();
  __syncthreads(); // the next item reuses the shared buffers
  return true;
}

constexpr int BOX_WORDS = (int)(sizeof(BoxDesc) / sizeof(int));
static_assert(BOX_WORDS <= NT, "one thread per descriptor word");

// Box mode (items == nullptr): the items of box b strided over the grid.
// Level mode: items of a device work list (sorted by cost, the tiles of a box
// together) taken by persistent CTAs from a counter.  One instantiation per stencil pair
// and centring CM = (cx << 2) | (cy << 1) | cz (1: cell centred).
template <class KV, class KC, int CM>
__global__ void __launch_bounds__(NT, AdjPair<KV, KC>::OCC)
    adjoint_kernel(const __grid_constant__ BoxDesc b, const BoxDesc *__restrict__ boxes,
                   const TileRef *__restrict__ items, int nitems, int *__restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ BoxDesc box_s;
  __shared__ uint64_t mbar[NBUF];
  __shared__ int s_fail;
  __shared__ int s_take;
  double *fbuf = reinterpret_cast<double *>(smem_raw);
  double *gbuf = fbuf + NBUF * AdjPair<KV, KC>::FP;
  // level launches after the first of a plan start in the previous one's
  // tail and wait for it at their end (programmatic dependent launch; no-ops
  // without the launch attribute)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (threadIdx.x == 0) {
    for (int k = 0; k < NBUF; ++k)
      mbar_init(mbar + k, 1);
    mbar_fence_init();
    s_fail = 0;
  }
  __syncthreads();
  uint32_t phase = 0; // completed-phase parity per buffer
  const long long limit = g_adj_wait_limit;
  // level mode: after item blockIdx.x, a CTA takes the next untaken item of
  // the list (sorted by cost) from the launch's counter (zero before it)
  for (int item = blockIdx.x; item < nitems;) {
    const BoxDesc *bp = &b;
    int xt, yt, zt, comp;
    if (items) {
      const TileRef t = items[item];
      if (threadIdx.x < BOX_WORDS)
        reinterpret_cast<int *>(&box_s)[threadIdx.x] =
            reinterpret_cast<const int *>(boxes + t.box)[threadIdx.x];
      __syncthreads();
      bp = &box_s;
      xt = t.tx;
      yt = t.ty;
      zt = t.tz;
      comp = t.comp;
    } else {
      int r = item;
      xt = r % b.ant[0];
      r /= b.ant[0];
      yt = r % b.ant[1];
      r /= b.ant[1];
      zt = r % b.ant[2];
      comp = r / b.ant[2];
    }
    using KX = std::conditional_t<(CM & 4) != 0, KC, KV>;
    using KY = std::conditional_t<(CM & 2) != 0, KC, KV>;
    using KZ = std::conditional_t<(CM & 1) != 0, KC, KV>;
    const bool ok =
        adj_item<KV, KC, KX, KY, KZ>(limit, fbuf, gbuf, mbar, &s_fail, phase, *bp, xt, yt, zt, comp);
    if (!ok)
      break;
    // adj_item ends with a barrier: box_s and s_take may be overwritten
    if (items) {
      if (threadIdx.x == 0)
        s_take = gridDim.x + atomicAdd(counter, 1);
      __syncthreads();
      item = s_take;
    } else {
      item += gridDim.x;
    }
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

using AdjFn = void (*)(const BoxDesc, const BoxDesc *, const TileRef *, int, int *);

// Kernel and shared-memory size of a pair and centring (nullptr for the
// nonlinear pairs).
template <class V, class C, int CM> AdjFn adj_fn(size_t *smem) {
  if constexpr (std::is_same_v<C, CcMinmod>) {
    return nullptr;
  } else {
    *smem = AdjPair<V, C>::SMEM;
    return adjoint_kernel<V, C, CM>;
  }
}

// Instantiations of centring CM (one file each), and the reading and
// clearing of that file's timeout flag.
AdjFn adj_kernel_part0(int pair, size_t *smem);
AdjFn adj_kernel_part1(int pair, size_t *smem);
AdjFn adj_kernel_part2(int pair, size_t *smem);
AdjFn adj_kernel_part3(int pair, size_t *smem);
AdjFn adj_kernel_part4(int pair, size_t *smem);
AdjFn adj_kernel_part5(int pair, size_t *smem);
AdjFn adj_kernel_part6(int pair, size_t *smem);
AdjFn adj_kernel_part7(int pair, size_t *smem);
// Sets that file's wait limit (cycles); 0 on success, -1 on a CUDA error.
int adj_set_wait_limit_part0(long long cycles);
int adj_set_wait_limit_part1(long long cycles);
int adj_set_wait_limit_part2(long long cycles);
int adj_set_wait_limit_part3(long long cycles);
int adj_set_wait_limit_part4(long long cycles);
int adj_set_wait_limit_part5(long long cycles);
int adj_set_wait_limit_part6(long long cycles);
int adj_set_wait_limit_part7(long long cycles);
int adj_timeout_part0();
int adj_timeout_part1();
int adj_timeout_part2();
int adj_timeout_part3();
int adj_timeout_part4();
int adj_timeout_part5();
int adj_timeout_part6();
int adj_timeout_part7();

} // namespace adj
} // namespace cxb
