// ENO prolongation per coarse cell, for operators whose three directions are
// all CC ENO 2 and whose linear fallback is inactive (the "eno" family at
// indextype 7, per var or per group).
//
// The reference chooses the stencil shift of every fine point
// (CarpetX/src/prolongate_3d_rf2_impl.hxx:1415-1517 per var, 1857-1965 per
// group): over the 27 shifts s (z outer, x inner) it takes
//   dd(s) = (1 + sqrt(eps) |s|_1) * max(ddx, ddy, ddz),
//   ddx = max over the 3 x 3 lines (j, k) around (cc + s) of
//         |undivided difference in x at cc + s|, ddy and ddz alike,
// and keeps the first minimum.  For ENO directions the line windows do not
// depend on the fine offset, so the 8 children of a coarse cell share the
// choice, and every term is a maximum of per-point |differences| D_d(p):
//   max(ddx, ddy, ddz)(s) = M(cc + s),
//   M(p) = max_d (max of D_d over the 3 x 3 window of p across d).
// fmax is exact, so M and the choice equal the reference's bit for bit (for
// NaN-free data).  The kernel computes D and M once per tile of coarse cells
// in shared memory, searches the shift once per cell, and evaluates the 8
// children with interp1d<CC,ENO,2> (impl.hxx:806-841) in call_stencil_3d's
// order (x lines, then y, then z), sharing the x and y results between the
// children: 38 1-D evaluations per cell instead of 8 x 13.
#include <atomic>
#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

constexpr int ET = 8;           // coarse cells per tile edge
constexpr int EW = ET + 4;      // window edge: tile plus 2 cells each side
constexpr int EW3 = EW * EW * EW;
constexpr int ENT = 256;        // threads per CTA
constexpr int ECPT = ET * ET * ET / ENT; // cells per thread
constexpr int NWIN = (EW3 + ENT - 1) / ENT; // window points per thread

// Guard points before the first and after the last window array: the
// passes below evaluate every window point with neighbours up to EW^2 away,
// without bounds tests; the values at the window's faces that read across
// an array end are garbage, and they reach no M(p) with p in [1, EW - 2]^3
// (the only points the search reads).
constexpr int EPAD = EW * EW + EW + 1;

struct EnoShared {
  double pad0[EPAD];
  double c[EW3];    // coarse window of one component
  double d[3][EW3]; // |undivided differences| per direction (max over the block's
                    // components); then, in place, A = W_z(D_x) over d[0],
                    // B = max(W_z(D_y), W_y(D_z)) over d[1] and M over d[2]
  double p[EW3];    // the other coarse window buffer (the next item's, prefetched)
  double pad1[EPAD];
};

__device__ __forceinline__ int widx(int i, int j, int k) { return (k * EW + j) * EW + i; }

// undivided_difference_1d<CC,ENO,2> (impl.hxx:751-773): -2 c0 + (c- + c+).
__device__ __forceinline__ double undiv2(double cm, double c0, double cp) {
  return fadd(fmul(-2.0, c0), fmul(1.0, fadd(cm, cp)));
}

// The three coefficients of interp1d<CC,ENO,2> for (shift, off), in tap order:
// row m = shift + 1 (off 0) or 1 - shift (off 1), reversed for off 1.
__device__ __forceinline__ void eno2_coeffs(int shift, int off, double w[3]) {
  const int m = off == 0 ? shift + 1 : 1 - shift;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int j = off == 0 ? i : 2 - i;
    w[i] = m == 0 ? cc_eno2_c(0, j) : m == 1 ? cc_eno2_c(1, j) : cc_eno2_c(2, j);
  }
}
// The reference's sum from 0 (impl.hxx:820-841), taps at shift - 1 .. shift + 1.
__device__ __forceinline__ double eno2_apply(const double w[3], double t0, double t1, double t2) {
  return fadd(fadd(fadd(0.0, fmul(w[0], t0)), fmul(w[1], t1)), fmul(w[2], t2));
}

struct EnoTiling {
  int clo[3];   // first coarse cell of the region (rlo >> 1)
  int nc[3];    // coarse cells with children in the region, per direction
  int nt[3];    // tiles per direction
  int nblk;     // component blocks: ncomp (per var) or 1 (per group)
};

// cshift (decisions for the adjoint, or null): the chosen shift of every
// coarse cell with children in the region, per component block, one byte
// (sx + 1) + 3 (sy + 1) + 9 (sz + 1), cells x fastest over t.nc; with it the
// children are not evaluated.
template <bool DECIDE>
// Two CTAs per SM evaluating children (124 registers); three deciding only
// (no child evaluation: 72 registers, and the shared arrays fit three).
__global__ void __launch_bounds__(ENT, DECIDE ? 3 : 2)
    eno_cell_kernel(const __grid_constant__ BoxDesc b, const EnoTiling t, int per_group,
                    signed char *shifts, unsigned char *fallback, unsigned char *cshift) {
  // the launches of a level's boxes after its first start in the previous
  // launch's tail and wait for it at their end (programmatic dependent
  // launch; no-ops without the launch attribute)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the window arrays (EnoShared) as one run of doubles, guards included, for the
  // neighbour reads across array ends
  double *const wbuf = reinterpret_cast<double *>(smem_raw);
  double *const C = wbuf + EPAD;
  double *const D0 = C + EW3, *const D1 = D0 + EW3, *const D2 = D1 + EW3;
  double *const A = D0, *const B = D1, *const Mw = D2;
  // the coarse window alternates between c and p: while an item evaluates
  // its children, the first window of the next item is copied into the other
  // buffer with cp.async
  double *Cc = C, *Cn = D2 + EW3;
  const int tid = threadIdx.x;
  const int rnx = b.rhi[0] - b.rlo[0] + 1, rny = b.rhi[1] - b.rlo[1] + 1;
  const int64_t rnp = (int64_t)rnx * rny * (b.rhi[2] - b.rlo[2] + 1);
  const int64_t cplane = (int64_t)b.cnx * b.cny, fplane = (int64_t)b.fnx * b.fny;
  const int ntiles = t.nt[0] * t.nt[1] * t.nt[2];
  // this thread's window points e = tid + n ENT: (i, j, k) packed 8 bits
  // each (-1: none), decoded once
  int wpt[NWIN];
#pragma unroll
  for (int n = 0; n < NWIN; ++n) {
    const int e = tid + n * ENT;
    wpt[n] = e < EW3 ? (e % EW) | ((e / EW) % EW) << 8 | (e / (EW * EW)) << 16 : -1;
  }
  const int nitems = ntiles * t.nblk;
  // window origin (coarse index of local 0) and first component of an item
  auto origin = [&](int item, int &o0, int &o1, int &o2, int &blk) {
    const int tile = item % ntiles;
    blk = item / ntiles;
    const int tx = tile % t.nt[0], ty = (tile / t.nt[0]) % t.nt[1], tz = tile / (t.nt[0] * t.nt[1]);
    o0 = t.clo[0] + tx * ET - 2;
    o1 = t.clo[1] + ty * ET - 2;
    o2 = t.clo[2] + tz * ET - 2;
  };
  // copy the window at origin (o0, o1, o2) of component comp into W: the
  // coarse points the operator reads (the rest of the window reaches only
  // cells outside the region); asynchronous (cp.async) or plain loads
  auto load = [&](double *W, int o0, int o1, int o2, int comp, bool async) {
    const double *cb = b.crse + comp * b.cnp;
#pragma unroll
    for (int n = 0; n < NWIN; ++n) {
      if (wpt[n] < 0)
        continue;
      const int e = tid + n * ENT;
      const int i = wpt[n] & 255, j = (wpt[n] >> 8) & 255, k = wpt[n] >> 16;
      const int gi = o0 + i, gj = o1 + j, gk = o2 + k;
      if (gi >= b.nlo[0] && gi <= b.nhi[0] && gj >= b.nlo[1] && gj <= b.nhi[1] &&
          gk >= b.nlo[2] && gk <= b.nhi[2]) {
        const double *src =
            cb + (gi - b.clo[0]) + (int64_t)b.cnx * (gj - b.clo[1]) + cplane * (gk - b.clo[2]);
        if (async)
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                           (unsigned)__cvta_generic_to_shared(W + e)),
                       "l"(src)
                       : "memory");
        else
          W[e] = __ldg(src);
      }
    }
  };
  if (blockIdx.x < nitems) {
    int o0, o1, o2, blk;
    origin(blockIdx.x, o0, o1, o2, blk);
    load(Cc, o0, o1, o2, per_group ? 0 : blk, true);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    int o0, o1, o2, blk;
    origin(item, o0, o1, o2, blk);
    const int c0 = per_group ? 0 : blk, c1 = per_group ? b.ncomp : blk + 1;
    // the first window of this item was copied into Cc by the previous item
    asm volatile("cp.async.wait_all;\n" ::: "memory");

    // D_d = max over the block's components of |undivided difference in d|
    // (valid where the difference's three points are in the window)
    for (int comp = c0; comp < c1; ++comp) {
      if (comp != c0) {
        __syncthreads();
        load(Cc, o0, o1, o2, comp, false);
      }
      __syncthreads();
#pragma unroll
      for (int n = 0; n < NWIN; ++n) {
        const int e = tid + n * ENT;
        if (e >= EW3)
          break;
        const double cx = fabs(undiv2(Cc[e - 1], Cc[e], Cc[e + 1]));
        const double cy = fabs(undiv2(Cc[e - EW], Cc[e], Cc[e + EW]));
        const double cz = fabs(undiv2(Cc[e - EW * EW], Cc[e], Cc[e + EW * EW]));
        if (comp == c0) {
          D0[e] = cx;
          D1[e] = cy;
          D2[e] = cz;
        } else {
          D0[e] = fmax(D0[e], cx);
          D1[e] = fmax(D1[e], cy);
          D2[e] = fmax(D2[e], cz);
        }
      }
    }
    __syncthreads();
    // M(p) = max over d of the 3 x 3 window maximum of D_d across d
    //      = max(W_y(A), W_x(B)),  A = W_z(D_x),  B = max(W_z(D_y), W_y(D_z)),
    // with W_a the maximum over a -1, 0, +1 along axis a (fmax is exact, so
    // the regrouping gives the same value); valid for p in [1, EW - 2]^3
    // (three arrays in place, so that three CTAs fit an SM): W_z of D_x
    // and D_y down each (x, y) column, the column's values held in
    // registers; then B over D_y; then M over D_z
    for (int tc = tid; tc < 2 * EW * EW; tc += ENT) {
      constexpr int Z = EW * EW;
      double *const col = (tc < Z ? D0 : D1) + tc % Z;
      double vm = col[0], v0 = col[0]; // the ends reach no M(p) the search reads
#pragma unroll
      for (int k = 0; k < EW; ++k) {
        const double vp = k + 1 < EW ? col[(k + 1) * Z] : v0;
        col[k * Z] = fmax(fmax(vm, v0), vp);
        vm = v0;
        v0 = vp;
      }
    }
    __syncthreads();
#pragma unroll
    for (int n = 0; n < NWIN; ++n) {
      const int e = tid + n * ENT;
      if (e >= EW3)
        break;
      B[e] = fmax(B[e], fmax(fmax(D2[e - EW], D2[e]), D2[e + EW]));
    }
    __syncthreads();
#pragma unroll
    for (int n = 0; n < NWIN; ++n) {
      const int e = tid + n * ENT;
      if (e >= EW3)
        break;
      Mw[e] = fmax(fmax(fmax(A[e - EW], A[e]), A[e + EW]),
                   fmax(fmax(B[e - 1], B[e]), B[e + 1]));
    }
    __syncthreads();

    // shift search per cell: first minimum in the reference's order
    int cell[ECPT], shx[ECPT], shy[ECPT], shz[ECPT];
#pragma unroll
    for (int q = 0; q < ECPT; ++q) {
      const int u = tid + q * ENT;
      const int ci = u % ET, cj = (u / ET) % ET, ck = u / (ET * ET);
      cell[q] = widx(ci + 2, cj + 2, ck + 2);
      double min_dd = __longlong_as_double(0x7ff0000000000000LL); // +inf
      int best = 13; // candidate (si + 1) + 3 (sj + 1) + 9 (sk + 1); 13 = no shift
#pragma unroll
      for (int sk = -1; sk <= 1; ++sk)
#pragma unroll
        for (int sj = -1; sj <= 1; ++sj)
#pragma unroll
          for (int si = -1; si <= 1; ++si) {
            // 1 + sqrt(DBL_EPSILON) * |s|_1 with sqrt(2^-52) = 2^-26: exact
            // for |s|_1 <= 3, a constant per candidate
            const int n1 = (si != 0) + (sj != 0) + (sk != 0);
            const double pen = 1.0 + 0x1p-26 * n1;
            const double mv = Mw[cell[q] + si + EW * sj + EW * EW * sk];
            const double dd = n1 == 0 ? mv : fmul(pen, mv); // 1 * m is exact
            if (dd < min_dd) {
              min_dd = dd;
              best = (si + 1) + 3 * (sj + 1) + 9 * (sk + 1);
            }
          }
      shx[q] = best % 3 - 1;
      shy[q] = (best / 3) % 3 - 1;
      shz[q] = best / 9 - 1;
      if constexpr (DECIDE) {
        const int lx = o0 + 2 + ci - t.clo[0], ly = o1 + 2 + cj - t.clo[1],
                  lz = o2 + 2 + ck - t.clo[2];
        if (lx < t.nc[0] && ly < t.nc[1] && lz < t.nc[2])
          cshift[(int64_t)blk * t.nc[0] * t.nc[1] * t.nc[2] + lx +
                 (int64_t)t.nc[0] * (ly + (int64_t)t.nc[1] * lz)] = (unsigned char)best;
      }
    }
    if constexpr (DECIDE) { // decisions only: no children to evaluate
      if (item + (int)gridDim.x < nitems) {
        int p0, p1, p2, pblk;
        origin(item + gridDim.x, p0, p1, p2, pblk);
        load(Cn, p0, p1, p2, per_group ? 0 : pblk, true);
      }
      asm volatile("cp.async.commit_group;\n" ::: "memory");
      __syncthreads();
      double *const t_ = Cc;
      Cc = Cn;
      Cn = t_;
      continue;
    }

    // copy the first window of this CTA's next item into the other buffer
    // while this one evaluates
    if (item + (int)gridDim.x < nitems) {
      int p0, p1, p2, pblk;
      origin(item + gridDim.x, p0, p1, p2, pblk);
      load(Cn, p0, p1, p2, per_group ? 0 : pblk, true);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");

    // evaluate the children of every cell, component by component
    for (int comp = c0; comp < c1; ++comp) {
      if (c1 - c0 > 1 || comp != c1 - 1) { // the window holds the last component loaded
        __syncthreads();
        load(Cc, o0, o1, o2, comp, false);
        __syncthreads();
      }
      double *fb = b.fine ? b.fine + comp * b.fnp : nullptr;
#pragma unroll 1
      for (int q = 0; q < ECPT; ++q) {
        const int u = tid + q * ENT;
        const int ci = u % ET, cj = (u / ET) % ET, ck = u / (ET * ET);
        const int gi = o0 + 2 + ci, gj = o1 + 2 + cj, gk = o2 + 2 + ck; // coarse cell
        const int f0x = 2 * gi, f0y = 2 * gj, f0z = 2 * gk;
        if (f0x + 1 < b.rlo[0] || f0x > b.rhi[0] || f0y + 1 < b.rlo[1] || f0y > b.rhi[1] ||
            f0z + 1 < b.rlo[2] || f0z > b.rhi[2])
          continue; // no child in the region
        double wy[2][3], wz[2][3];
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          eno2_coeffs(shy[q], o, wy[o]);
          eno2_coeffs(shz[q], o, wz[o]);
        }
        // x lines at y = cj + shy - 1 + a, z = ck + shz - 1 + g: each line's
        // three points are read once for both fine x offsets
        const int base = cell[q] + (shx[q] - 1) + EW * (shy[q] - 1) + EW * EW * (shz[q] - 1);
        double wx[2][3];
#pragma unroll
        for (int o = 0; o < 2; ++o)
          eno2_coeffs(shx[q], o, wx[o]);
        double Y[2][2][3]; // [ox][oy][g]
#pragma unroll
        for (int g = 0; g < 3; ++g) {
          double X[2][3]; // [ox][a]
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const double *v = Cc + base + EW * a + EW * EW * g;
            const double v0 = v[0], v1 = v[1], v2 = v[2];
            X[0][a] = eno2_apply(wx[0], v0, v1, v2);
            X[1][a] = eno2_apply(wx[1], v0, v1, v2);
          }
#pragma unroll
          for (int ox = 0; ox < 2; ++ox)
#pragma unroll
            for (int oy = 0; oy < 2; ++oy)
              Y[ox][oy][g] = eno2_apply(wy[oy], X[ox][0], X[ox][1], X[ox][2]);
        }
#pragma unroll
        for (int ox = 0; ox < 2; ++ox)
#pragma unroll
          for (int oy = 0; oy < 2; ++oy)
#pragma unroll
            for (int oz = 0; oz < 2; ++oz) {
              const int fx = f0x + ox, fy = f0y + oy, fz = f0z + oz;
              if (fx < b.rlo[0] || fx > b.rhi[0] || fy < b.rlo[1] || fy > b.rhi[1] ||
                  fz < b.rlo[2] || fz > b.rhi[2])
                continue;
              const double r = eno2_apply(wz[oz], Y[ox][oy][0], Y[ox][oy][1], Y[ox][oy][2]);
              if (fb) // null: decisions only (the adjoint's decision pass)
                fb[(fx - b.flo[0]) + (int64_t)b.fnx * (fy - b.flo[1]) + fplane * (fz - b.flo[2])] = r;
              if (comp == c0 && (shifts || fallback)) {
                const int64_t ridx = (fx - b.rlo[0]) + (int64_t)rnx * ((fy - b.rlo[1]) +
                                                                      (int64_t)rny * (fz - b.rlo[2]));
                if (shifts) {
                  signed char *sp = shifts + 3 * (blk * rnp + ridx);
                  sp[0] = (signed char)shx[q];
                  sp[1] = (signed char)shy[q];
                  sp[2] = (signed char)shz[q];
                }
                if (fallback)
                  fallback[blk * rnp + ridx] = 0;
              }
            }
      }
    }
    __syncthreads(); // the next item reuses the shared arrays
    double *const t_ = Cc;
    Cc = Cn;
    Cn = t_;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Per device (cache_device()): persistent grid, 0 until the kernel's dynamic
// shared memory has been allowed on that device.
std::atomic<int> g_eno_grid[kMaxDevices][2]; // [device][decisions only]

} // namespace

bool eno_cell_applies(const BoxDesc &b, int per_group) {
  return b.kind[0] == K_CC_ENO2 && b.kind[1] == K_CC_ENO2 && b.kind[2] == K_CC_ENO2 &&
         !op_fb_active(b.op, per_group);
}

cudaError_t launch_eno_cell_box(const BoxDesc &b, int per_group, signed char *shifts,
                                unsigned char *fallback, cudaStream_t s, bool after_level,
                                unsigned char *cshift) {
  if (b.ncomp <= 0)
    return cudaSuccess;
  EnoTiling t;
  for (int d = 0; d < 3; ++d) {
    if (b.rhi[d] < b.rlo[d])
      return cudaSuccess;
    t.clo[d] = b.rlo[d] >> 1;
    t.nc[d] = (b.rhi[d] >> 1) - t.clo[d] + 1;
    t.nt[d] = (t.nc[d] + ET - 1) / ET;
  }
  t.nblk = per_group ? 1 : b.ncomp;
  const int64_t n = (int64_t)t.nt[0] * t.nt[1] * t.nt[2] * t.nblk;
  if (n > INT32_MAX)
    return cudaErrorInvalidValue;
  const int dev = cache_device();
  const int dk = cshift ? 1 : 0;
  int grid = dev >= 0 ? g_eno_grid[dev][dk].load() : 0;
  if (!grid) {
    cudaError_t e = cudaFuncSetAttribute(eno_cell_kernel<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(EnoShared));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(eno_cell_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(EnoShared));
    if (e != cudaSuccess)
      return e;
    int per_sm = 0, d = 0, sms = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, dk ? eno_cell_kernel<true> : eno_cell_kernel<false>, ENT, sizeof(EnoShared));
    grid = sms * (per_sm > 0 ? per_sm : 1);
    if (dev >= 0)
      g_eno_grid[dev][dk].store(grid);
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(n < grid ? (unsigned)n : (unsigned)grid);
  cfg.blockDim = dim3(ENT);
  cfg.dynamicSmemBytes = sizeof(EnoShared);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = after_level ? 1 : 0;
  if (cshift)
    return cudaLaunchKernelEx(&cfg, eno_cell_kernel<true>, b, t, per_group, shifts, fallback,
                              cshift);
  return cudaLaunchKernelEx(&cfg, eno_cell_kernel<false>, b, t, per_group, shifts, fallback,
                            cshift);
}


namespace {

// Adjoint of the ENO-per-cell operators, linearised at the coarse input:
// fine point f = 2 p + o (o in {0,1}^3) of parent cell p with shift s reads
// coarse p + s + (a - 1) with weight wx(sx, ox, ax) wy(sy, oy, ay)
// wz(sz, oz, az) (interp1d<CC,ENO,2>'s row, impl.hxx:806-841), so parent p
// adds to coarse q = p + s + a - 1 its tap contribution
//   W(p, a) = sum_o wz(sz, oz, az) wy(sy, oy, ay) wx(sx, ox, ax) fbar(2 p + o),
// fine points outside the region counting as 0, and
//   crse_bar(q) = sum over parents p with a = q - p - s + 1 in [0, 2]^3 of W(p, a).
// A CTA takes a tile of AX x AY x AZ coarse points of the coarse box (one
// thread each), stages the shift codes of the parents within 2 cells (the
// decision pass's cshift) once, and walks the parents' z planes: per plane it
// stages the two fine planes of the children, every parent of the plane
// computes its 27 contributions (x, then y, then z contraction) into shared
// memory, and every coarse point within two planes adds those of its
// matching candidate parents (25 per plane, one mask test each).  The order
// of the sums is fixed (no atomics, deterministic); every coarse point of
// the box is written, zero where no region point reads it.
constexpr int AX = 8, AY = 8, AZ = 4;
constexpr int PWX = AX + 4, PWY = AY + 4, PWZ = AZ + 4; // parent window
constexpr int PWXY = PWX * PWY;
constexpr int FWX = 2 * PWX, FWY = 2 * PWY;             // the children of a parent plane
constexpr int ANT = AX * AY * AZ;

struct EnoAdjShared {
  double f[2][2][FWY * FWX]; // fine_bar of a parent plane's children [buffer][oz][fy][fx]
  double w[27][PWXY];      // W(p, a) of the plane's parents [a][parent]
  double tw[3][2][3];      // interp1d<CC,ENO,2> weights [shift + 1][off][tap]
  // per parent: the offsets d = p - q it serves, bit d_x + 2, d_y + 7,
  // d_z + 12 (d_i + s_i in [-1, 1]: three consecutive bits from 1 - s_i per
  // direction, so s_i = 1 - (lowest set bit of its field)); 0: no children
  // in the region
  unsigned short code[PWZ * PWXY];
};

__constant__ double c_eno_w[3][2][3]; // [shift + 1][off][tap]

__global__ void __launch_bounds__(ANT, 4)
    eno_adjoint_kernel(const __grid_constant__ BoxDesc b, const EnoTiling t, int per_group,
                       const unsigned char *__restrict__ cshift, double *__restrict__ cbar,
                       int ntx, int nty) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  EnoAdjShared &sh = *reinterpret_cast<EnoAdjShared *>(smem_raw);
  const int tid = threadIdx.x;
  const int blk = blockIdx.y;
  const int tile = blockIdx.x;
  const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
  const int q0x = b.clo[0] + (tile % ntx) * AX, q0y = b.clo[1] + ((tile / ntx) % nty) * AY,
            q0z = b.clo[2] + (tile / (ntx * nty)) * AZ;
  const int64_t ncell = (int64_t)t.nc[0] * t.nc[1] * t.nc[2];
  if (tid < 18)
    (&sh.tw[0][0][0])[tid] = (&c_eno_w[0][0][0])[tid];
  // parents p = q0 - 2 + (i, j, k)
  for (int e = tid; e < PWX * PWY * PWZ; e += ANT) {
    const int i = e % PWX, j = (e / PWX) % PWY, k = e / PWXY;
    const int lx = q0x - 2 + i - t.clo[0], ly = q0y - 2 + j - t.clo[1], lz = q0z - 2 + k - t.clo[2];
    unsigned int w = 0;
    if (lx >= 0 && lx < t.nc[0] && ly >= 0 && ly < t.nc[1] && lz >= 0 && lz < t.nc[2]) {
      const int c = cshift[blk * ncell + lx + (int64_t)t.nc[0] * (ly + (int64_t)t.nc[1] * lz)];
      const int sx = c % 3 - 1, sy = (c / 3) % 3 - 1, sz = c / 9 - 1;
      w = (7u << (1 - sx)) | (7u << (6 - sy)) | (7u << (11 - sz));
    }
    sh.code[e] = (unsigned short)w;
  }
  const int ix = tid % AX, iy = (tid / AX) % AY, iz = tid / (AX * AY);
  const int qx = q0x + ix, qy = q0y + iy, qz = q0z + iz;
  const bool mine = qx < b.clo[0] + b.cnx && qy < b.clo[1] + b.cny && qz < b.clo[2] + cnz;
  const int c0 = per_group ? 0 : blk, c1 = per_group ? b.ncomp : blk + 1;
  const int64_t fplane = (int64_t)b.fnx * b.fny;
  const int fx0 = 2 * (q0x - 2), fy0 = 2 * (q0y - 2);
  // the children of parent plane k of component comp into buffer buf:
  // asynchronous 8-byte copies, zero outside the region
  auto stage = [&](int comp, int k, int buf) {
    const double *fb = b.fine + comp * b.fnp;
    for (int e = tid; e < 2 * FWX * FWY; e += ANT) {
      const int i = e % FWX, j = (e / FWX) % FWY, oz = e / (FWX * FWY);
      const int fx = fx0 + i, fy = fy0 + j, fz = 2 * (q0z - 2 + k) + oz;
      const bool ok = fx >= b.rlo[0] && fx <= b.rhi[0] && fy >= b.rlo[1] && fy <= b.rhi[1] &&
                      fz >= b.rlo[2] && fz <= b.rhi[2];
      const double *src =
          ok ? fb + (fx - b.flo[0]) + (int64_t)b.fnx * (fy - b.flo[1]) + fplane * (fz - b.flo[2])
             : fb;
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                       (unsigned)__cvta_generic_to_shared(&sh.f[buf][oz][j * FWX + i])),
                   "l"(src), "r"(ok ? 8 : 0)
                   : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const int nit = (c1 - c0) * PWZ; // (component, parent plane) steps
  stage(c0, 0, 0);
  double acc = 0.0;
  for (int it = 0; it < nit; ++it) {
    const int comp = c0 + it / PWZ, k = it % PWZ, buf = it & 1; // parent plane q0z - 2 + k
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads(); // this plane's children are in; the previous plane is consumed
    if (it + 1 < nit)
      stage(c0 + (it + 1) / PWZ, (it + 1) % PWZ, buf ^ 1);
    // the plane's parents: W(p, a), x then y then z contraction
    for (int e = tid; e < PWXY; e += ANT) {
      const unsigned int w = sh.code[k * PWXY + e];
      if (!w)
        continue; // no children in the region: never matched
      const int pi = e % PWX, pj = e / PWX;
      const int sx = 2 - __ffs(w & 31u), sy = 2 - __ffs((w >> 5) & 31u),
                sz = 2 - __ffs((w >> 10) & 31u);
      const double *wx = sh.tw[sx + 1][0], *wy = sh.tw[sy + 1][0], *wz = sh.tw[sz + 1][0];
      double uy[2][3][3]; // [oz][ay][ax]
#pragma unroll
      for (int oz = 0; oz < 2; ++oz) {
        double ux[2][3]; // [oy][ax]
#pragma unroll
        for (int oy = 0; oy < 2; ++oy) {
          const double *r = sh.f[buf][oz] + (2 * pj + oy) * FWX + 2 * pi;
          const double r0 = r[0], r1 = r[1];
#pragma unroll
          for (int ax = 0; ax < 3; ++ax)
            ux[oy][ax] = fma(wx[3 + ax], r1, wx[ax] * r0);
        }
#pragma unroll
        for (int ay = 0; ay < 3; ++ay)
#pragma unroll
          for (int ax = 0; ax < 3; ++ax)
            uy[oz][ay][ax] = fma(wy[3 + ay], ux[1][ax], wy[ay] * ux[0][ax]);
      }
#pragma unroll
      for (int az = 0; az < 3; ++az)
#pragma unroll
        for (int ay = 0; ay < 3; ++ay)
#pragma unroll
          for (int ax = 0; ax < 3; ++ax)
            sh.w[(az * 3 + ay) * 3 + ax][e] =
                fma(wz[3 + az], uy[1][ay][ax], wz[az] * uy[0][ay][ax]);
    }
    __syncthreads();
    const int dz = k - 2 - iz; // p_z - q_z, uniform per warp
    if (mine && dz >= -2 && dz <= 2) {
#pragma unroll 1
      for (int dy = -2; dy <= 2; ++dy)
#pragma unroll
        for (int dx = -2; dx <= 2; ++dx) {
          const int pe = (iy + 2 + dy) * PWX + (ix + 2 + dx);
          const unsigned int w = sh.code[k * PWXY + pe];
          const unsigned int want = (1u << (dx + 2)) | (1u << (dy + 7)) | (1u << (dz + 12));
          if ((w & want) != want)
            continue;
          // lowest set bit of each field: 1 - s_i; the tap a_i = 1 - s_i - d_i
          const int ax = __ffs(w & 31u) - 1 - dx, ay = __ffs((w >> 5) & 31u) - 1 - dy,
                    az = __ffs((w >> 10) & 31u) - 1 - dz;
          acc += sh.w[(az * 3 + ay) * 3 + ax][pe];
        }
    }
    if (k == PWZ - 1) { // the component's last plane: its sums are complete
      if (mine)
        cbar[comp * b.cnp + (qx - b.clo[0]) + (int64_t)b.cnx * (qy - b.clo[1]) +
             (int64_t)b.cnx * b.cny * (qz - b.clo[2])] = acc;
      acc = 0.0;
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

std::atomic<bool> g_eno_w_set[kMaxDevices];

} // namespace

size_t eno_adjoint_scratch_bytes(const BoxDesc &b, int per_group) {
  int64_t n = per_group ? 1 : b.ncomp;
  for (int d = 0; d < 3; ++d) {
    if (b.rhi[d] < b.rlo[d])
      return 0;
    n *= (b.rhi[d] >> 1) - (b.rlo[d] >> 1) + 1;
  }
  return (size_t)n;
}

cudaError_t launch_eno_adjoint_box(const BoxDesc &b, int per_group, void *scratch,
                                   double *crse_bar, cudaStream_t s) {
  if (b.ncomp <= 0 || b.cnp <= 0)
    return cudaSuccess;
  EnoTiling t;
  bool empty = false;
  for (int d = 0; d < 3; ++d) {
    empty = empty || b.rhi[d] < b.rlo[d];
    t.clo[d] = b.rlo[d] >> 1;
    t.nc[d] = empty ? 0 : (b.rhi[d] >> 1) - t.clo[d] + 1;
    t.nt[d] = 0;
  }
  t.nblk = per_group ? 1 : b.ncomp;
  unsigned char *cs = static_cast<unsigned char *>(scratch);
  const int dev = cache_device();
  if (dev < 0 || !g_eno_w_set[dev].load()) {
    double w[3][2][3];
    for (int sh = -1; sh <= 1; ++sh)
      for (int off = 0; off < 2; ++off) {
        const int m = off == 0 ? sh + 1 : 1 - sh;
        for (int i = 0; i < 3; ++i) {
          const int j = off == 0 ? i : 2 - i;
          w[sh + 1][off][i] = cc_eno2_c(m, j);
        }
      }
    cudaError_t e = cudaMemcpyToSymbol(c_eno_w, w, sizeof w);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(eno_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(EnoAdjShared));
    if (e != cudaSuccess)
      return e;
    if (dev >= 0)
      g_eno_w_set[dev].store(true);
  }
  if (!empty) {
    // the decisions: one shift code per coarse cell with children in the region
    BoxDesc d = b;
    d.fine = nullptr;
    if (cudaError_t e = launch_eno_cell_box(d, per_group, nullptr, nullptr, s, false, cs))
      return e;
  }
  const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
  const int ntx = (b.cnx + AX - 1) / AX, nty = (b.cny + AY - 1) / AY, ntz = (cnz + AZ - 1) / AZ;
  const int64_t ntiles = (int64_t)ntx * nty * ntz;
  if (ntiles > INT32_MAX)
    return cudaErrorInvalidValue;
  if (empty) // nothing reads the coarse box: zero
    return cudaMemsetAsync(crse_bar, 0, sizeof(double) * b.cnp * b.ncomp, s);
  eno_adjoint_kernel<<<dim3((unsigned)ntiles, t.nblk), ANT, sizeof(EnoAdjShared), s>>>(
      b, t, per_group, cs, crse_bar, ntx, nty);
  return cudaGetLastError();
}

} // namespace cxb
