// Pointwise prolongation kernel for the operators that are not separable:
// ENO directions (stencil shift chosen per point from undivided differences)
// and the FB_LINEAR fallback (poly-cons3lfb, poly-eno3lfb).
//
// One thread per fine point (per component in per-var mode), following the
// reference loop body (CarpetX/src/prolongate_3d_rf2_impl.hxx:1412-1669 per
// var, 1854-2146 per group) step by step: shift search, tensor evaluation,
// fallback tests, store.  Coarse values are read through the read-only data
// cache.  Stencil kinds are runtime parameters here.
#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

struct Coarse {
  const double *p; // component 0
  int64_t np;
  int lo[3];
  int nx, ny;
  __device__ __forceinline__ double operator()(int comp, int i, int j, int k) const {
    return __ldg(p + comp * np + (i - lo[0]) + (int64_t)nx * ((j - lo[1]) + (int64_t)ny * (k - lo[2])));
  }
};

// stencil_radius(shift, off) of a kind (impl.hxx:402-408, 466-476, 588-601,
// 640-649, 786-803, 850-856).
__device__ __forceinline__ void radius(int k, int shift, int off, int r[2]) {
  if (k == K_CC_ENO2) {
    r[0] = shift - 1;
    r[1] = shift + 1;
    return;
  }
  const KindInfo ki = kind_info(k);
  r[0] = off ? ki.r1lo : ki.r0lo;
  r[1] = off ? ki.r1hi : ki.r0hi;
}

// interp1d<CC,ENO,2>: row m = shift + 1 (off 0) or 1 - shift (off 1), off 1
// reverses the row (impl.hxx:806-841).
__device__ __forceinline__ double eno2(int shift, int off, const double *v) {
  const int m = off == 0 ? shift + 1 : 1 - shift;
  const int i0 = 1 - shift;
  double y = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    y = fadd(y, fmul(cc_eno2_c(m, off == 0 ? i : 2 - i), v[i - i0]));
  return y;
}

template <class K> __device__ __forceinline__ void ap_off(int off, const double *v, double &y) {
  y = off ? K::template ap<1>(v) : K::template ap<0>(v);
}

// Runtime-kind 1-D stencil; v points at coarse offset 0.
__device__ __noinline__ double ap_rt(int k, int shift, int off, const double *v) {
  if (k == K_CC_ENO2)
    return eno2(shift, off, v);
  double y = 0.0;
  CXB_DISPATCH_SEPARABLE(k, ap_off, off, v, y);
  return y;
}

// call_stencil_3d with runtime kinds (impl.hxx:1206-1216).
__device__ double eval3d(const int kind[3], const int shift[3], const int off[3], const Coarse &c,
                         int comp, const int ic[3]) {
  int r[3][2];
  for (int d = 0; d < 3; ++d)
    radius(kind[d], shift[d], off[d], r[d]);
  double Y[9], X[9], v[9];
  for (int dk = r[2][0]; dk <= r[2][1]; ++dk) {
    for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
      for (int di = r[0][0]; di <= r[0][1]; ++di)
        v[di + 4] = c(comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
      X[dj + 4] = ap_rt(kind[0], shift[0], off[0], v + 4);
    }
    Y[dk + 4] = ap_rt(kind[1], shift[1], off[1], X + 4);
  }
  return ap_rt(kind[2], shift[2], off[2], Y + 4);
}

// undivided_difference_1d<CC,ENO,2> (impl.hxx:751-773): -2*c0 + (c- + c+).
__device__ __forceinline__ double undiv2(double cm, double c0, double cp) {
  return fadd(fmul(-2.0, c0), fmul(1.0, fadd(cm, cp)));
}

// ENO shift choice (impl.hxx:1415-1517 / 1857-1965) over components c0..c1-1.
__device__ void choose_shift(const int kind[3], const int off[3], const Coarse &c, int c0, int c1,
                             const int ic[3], int shift[3]) {
  int use[3], maxs[3];
  for (int d = 0; d < 3; ++d) {
    use[d] = kind[d] == K_CC_ENO2;
    maxs[d] = use[d] ? 1 : 0;
    shift[d] = 0;
  }
  double min_dd = __longlong_as_double(0x7ff0000000000000LL); // +inf
  for (int sk = -maxs[2]; sk <= maxs[2]; ++sk)
    for (int sj = -maxs[1]; sj <= maxs[1]; ++sj)
      for (int si = -maxs[0]; si <= maxs[0]; ++si) {
        const int sh[3] = {si, sj, sk};
        int r[3][2];
        for (int d = 0; d < 3; ++d) {
          radius(kind[d], sh[d], off[d], r[d]);
          if (use[d]) {
            r[d][0] -= sh[d];
            r[d][1] -= sh[d];
          }
        }
        double ddx = 0, ddy = 0, ddz = 0;
        for (int comp = c0; comp < c1; ++comp) {
          if (use[0])
            for (int dk = r[2][0]; dk <= r[2][1]; ++dk)
              for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
                const int i = ic[0] + si, j = ic[1] + sj + dj, k = ic[2] + sk + dk;
                ddx = fmax(ddx, fabs(undiv2(c(comp, i - 1, j, k), c(comp, i, j, k), c(comp, i + 1, j, k))));
              }
          if (use[1])
            for (int dk = r[2][0]; dk <= r[2][1]; ++dk)
              for (int di = r[0][0]; di <= r[0][1]; ++di) {
                const int i = ic[0] + si + di, j = ic[1] + sj, k = ic[2] + sk + dk;
                ddy = fmax(ddy, fabs(undiv2(c(comp, i, j - 1, k), c(comp, i, j, k), c(comp, i, j + 1, k))));
              }
          if (use[2])
            for (int dj = r[1][0]; dj <= r[1][1]; ++dj)
              for (int di = r[0][0]; di <= r[0][1]; ++di) {
                const int i = ic[0] + si + di, j = ic[1] + sj + dj, k = ic[2] + sk;
                ddz = fmax(ddz, fabs(undiv2(c(comp, i, j, k - 1), c(comp, i, j, k), c(comp, i, j, k + 1))));
              }
        }
        // 1 + sqrt(DBL_EPSILON) * n, sqrt(2^-52) = 2^-26 exactly
        const double penalty = fadd(1.0, fmul(0x1p-26, (double)(abs(si) + abs(sj) + abs(sk))));
        const double dd = fmul(penalty, fmax(fmax(ddx, ddy), ddz));
        if (dd < min_dd) {
          min_dd = dd;
          shift[0] = si;
          shift[1] = sj;
          shift[2] = sk;
        }
      }
}

// Slope sign change in direction d (impl.hxx:1609-1664, 2026-2115): s0 is
// taken between offsets 0 and 1, the scan starts at radius[0] + 2.
__device__ bool slope_change(int d, const int sr[3][2], const Coarse &c, int comp, const int ic[3]) {
  const int in_d = d == 0 ? 1 : 0, out_d = d == 2 ? 1 : 2;
  bool need = false;
  for (int q = sr[out_d][0]; q <= sr[out_d][1]; ++q)
    for (int t = sr[in_d][0]; t <= sr[in_d][1]; ++t) {
      int a[3], b[3];
      a[out_d] = b[out_d] = q;
      a[in_d] = b[in_d] = t;
      a[d] = 1;
      b[d] = 0;
      const double s0 = fsub(c(comp, ic[0] + a[0], ic[1] + a[1], ic[2] + a[2]),
                             c(comp, ic[0] + b[0], ic[1] + b[1], ic[2] + b[2]));
      for (int e = sr[d][0] + 2; e <= sr[d][1]; ++e) {
        a[d] = e;
        b[d] = e - 1;
        const double s = fsub(c(comp, ic[0] + a[0], ic[1] + a[1], ic[2] + a[2]),
                              c(comp, ic[0] + b[0], ic[1] + b[1], ic[2] + b[2]));
        need |= fmul(s, s0) < 0;
      }
    }
  return need;
}

__global__ void __launch_bounds__(256)
    point_box_kernel(const BoxDesc b, int per_group, signed char *shifts, unsigned char *fallback) {
  const int rnx = b.rhi[0] - b.rlo[0] + 1, rny = b.rhi[1] - b.rlo[1] + 1;
  const int64_t rnp = (int64_t)rnx * rny * (b.rhi[2] - b.rlo[2] + 1);
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rnp)
    return;
  const int blk = blockIdx.y; // component (per var) or 0 (per group)
  const int c0 = per_group ? 0 : blk, c1 = per_group ? b.ncomp : blk + 1;
  const int ifine[3] = {b.rlo[0] + (int)(idx % rnx), b.rlo[1] + (int)((idx / rnx) % rny),
                        b.rlo[2] + (int)(idx / ((int64_t)rnx * rny))};
  Coarse c;
  c.p = b.crse;
  c.np = b.cnp;
  c.nx = b.cnx;
  c.ny = b.cny;
  int ic[3], off[3], shift[3], kind[3], lin[3];
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = b.clo[d];
    ic[d] = ifine[d] >> 1; // arithmetic shift = floor, as the reference
    off[d] = ifine[d] & 1;
    kind[d] = b.kind[d];
    const KindInfo ki = kind_info(kind[d]);
    // linear fallback stencils: impl.hxx:1547-1558 (per var: CONS and ENO
    // become CONS 1) and 2119-2121 (per group: CONS 1, ENO kept)
    if (ki.intp == CONS || (!per_group && ki.intp == ENO))
      lin[d] = K_CC_CONS1;
    else
      lin[d] = kind[d];
  }
  choose_shift(kind, off, c, c0, c1, ic, shift);
  double vals[16];
  for (int comp = c0; comp < c1; ++comp)
    vals[comp - c0] = eval3d(kind, shift, off, c, comp, ic);
  bool need = false;
  if (op_fb_active(b.op, per_group)) {
    int sr[3][2];
    for (int d = 0; d < 3; ++d)
      radius(kind[d], shift[d], off[d], sr[d]);
    double minval = __longlong_as_double(0x7ff0000000000000LL);
    double maxval = -minval;
    for (int comp = c0; comp < c1; ++comp) {
      // per group the extrema accumulate over the components (impl.hxx:
      // 2010-2024); per var there is one component
      for (int dk = sr[2][0]; dk <= sr[2][1]; ++dk)
        for (int dj = sr[1][0]; dj <= sr[1][1]; ++dj)
          for (int di = sr[0][0]; di <= sr[0][1]; ++di) {
            const double x = c(comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
            minval = fmin(minval, x);
            maxval = fmax(maxval, x);
          }
      need |= vals[comp - c0] < minval || vals[comp - c0] > maxval;
    }
    for (int d = 0; d < 3; ++d) {
      const int intp = kind_info(kind[d]).intp;
      const bool check = per_group ? intp == CONS : (intp == CONS || intp == ENO);
      if (!check)
        continue;
      for (int comp = c0; comp < c1; ++comp)
        need |= slope_change(d, sr, c, comp, ic);
    }
  }
  const int64_t fidx = (ifine[0] - b.flo[0]) +
                       (int64_t)b.fnx * ((ifine[1] - b.flo[1]) + (int64_t)b.fny * (ifine[2] - b.flo[2]));
  const int zero3[3] = {0, 0, 0};
  if (b.fine) // null: decisions only (the adjoint's decision pass)
    for (int comp = c0; comp < c1; ++comp) {
      const double res = need ? eval3d(lin, zero3, off, c, comp, ic) : vals[comp - c0];
      b.fine[comp * b.fnp + fidx] = res;
    }
  if (shifts)
    for (int d = 0; d < 3; ++d)
      shifts[3 * (blk * rnp + idx) + d] = (signed char)shift[d];
  if (fallback)
    fallback[blk * rnp + idx] = need ? 1 : 0;
}


// ---------------------------------------------------------------------------
// Adjoint of the limited operators (ENO, minmod, linear fallback), gather
// form: P^T linearised at the forward input, as the transpose of the map each
// fine point applies (the reference's choices treated as locally constant).
// A decision pass (the forward kernels with value stores off) writes every
// region point's ENO shift and fallback flag; here one thread per coarse
// point c (per component) sums, over the fine points f whose stencil can
// reach c, w(f, c) * fine_bar(f) in a fixed order (no atomics):
//   w(f, c) = wz(k) wy(j; k) wx(i; j, k),  (i, j, k) = c - cell(f),
// with each 1-D weight that of the kind f applies in that direction (its
// fallback kind if it fell back, with shift 0).  For the linear kinds the
// weights are constants of (kind, shift, off), tabulated per CTA by
// evaluating the stencil on unit vectors (the reference's arithmetic); a
// minmod direction's weights depend on the values it reads, which are
// re-evaluated (x lines from coarse data, y from the x results).

// 1-D weights of a minmod application at line values v[-1..1] (impl.hxx:
// 859-877 differentiated; fmin keeps |dm| on ties).
__device__ __forceinline__ void minmod_weights(int off, const double *v, double w[3]) {
  const double dm = v[0] - v[-1], dp = v[1] - v[0];
  const double sgn = off == 0 ? -1.0 : 1.0;
  w[0] = 0.0;
  w[1] = 1.0;
  w[2] = 0.0;
  const double f = copysign(0.125, dm) + copysign(0.125, dp);
  if (f != 0.0) {
    if (fabs(dm) <= fabs(dp)) {
      w[1] += sgn * 0.25;
      w[0] -= sgn * 0.25;
    } else {
      w[2] += sgn * 0.25;
      w[1] -= sgn * 0.25;
    }
  }
}

constexpr int AT_NT = 128; // threads per CTA

// weight table: [direction][0: kind, 1: fallback kind][shift + 1][off][o + 4]
struct AdjTable {
  double w[3][2][3][2][9];
};

__global__ void __launch_bounds__(AT_NT)
    adjoint_point_kernel(const BoxDesc b, int per_group, const signed char *shifts,
                         const unsigned char *fallback, double *crse_bar) {
  __shared__ AdjTable tab;
  int kind[3], lin[3], lo[3], hi[3];
  bool mm[3], mml[3];
  for (int d = 0; d < 3; ++d) {
    kind[d] = b.kind[d];
    const KindInfo ki = kind_info(kind[d]);
    lin[d] = (ki.intp == CONS || (!per_group && ki.intp == ENO)) ? K_CC_CONS1 : kind[d];
    mm[d] = kind[d] == K_CC_MINMOD1;
    mml[d] = lin[d] == K_CC_MINMOD1;
    // coarse offsets any fine point may read (ENO search window, both parities)
    int a, c, a1, c1;
    read_range(kind[d], 0, &a, &c);
    read_range(kind[d], 1, &a1, &c1);
    lo[d] = min(a, a1);
    hi[d] = max(c, c1);
  }
  // tabulate the linear weights (unused entries stay 0)
  for (int e = threadIdx.x; e < 3 * 2 * 3 * 2; e += blockDim.x) {
    const int off = e % 2, sh = (e / 2) % 3 - 1, which = (e / 6) % 2, d = e / 12;
    const int k = which ? lin[d] : kind[d];
    double *w = tab.w[d][which][sh + 1][off];
    for (int o = 0; o < 9; ++o)
      w[o] = 0.0;
    if (k == K_CC_MINMOD1 || (sh != 0 && k != K_CC_ENO2))
      continue;
    int r[2];
    radius(k, sh, off, r);
    for (int o = r[0]; o <= r[1]; ++o) {
      double unit[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      unit[o + 4] = 1.0;
      w[o + 4] = ap_rt(k, sh, off, unit + 4);
    }
  }
  __syncthreads();
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= b.cnp)
    return;
  const int blk = blockIdx.y; // component (per var) or 0 (per group)
  const int c0 = per_group ? 0 : blk, c1 = per_group ? b.ncomp : blk + 1;
  const int cz = b.clo[2] + (int)(idx / ((int64_t)b.cnx * b.cny));
  const int cy = b.clo[1] + (int)((idx / b.cnx) % b.cny);
  const int cx = b.clo[0] + (int)(idx % b.cnx);
  const int cc[3] = {cx, cy, cz};
  const int rnx = b.rhi[0] - b.rlo[0] + 1, rny = b.rhi[1] - b.rlo[1] + 1;
  const int64_t rnp = (int64_t)rnx * rny * (b.rhi[2] - b.rlo[2] + 1);
  const int64_t fplane = (int64_t)b.fnx * b.fny;
  Coarse crs;
  crs.p = b.crse;
  crs.np = b.cnp;
  crs.nx = b.cnx;
  crs.ny = b.cny;
  for (int d = 0; d < 3; ++d)
    crs.lo[d] = b.clo[d];
  for (int comp = c0; comp < c1; ++comp) {
    double acc = 0.0;
    for (int kz = cz - hi[2]; kz <= cz - lo[2]; ++kz)
      for (int ky = cy - hi[1]; ky <= cy - lo[1]; ++ky)
        for (int kx = cx - hi[0]; kx <= cx - lo[0]; ++kx)
          for (int o8 = 0; o8 < 8; ++o8) {
            const int ic[3] = {kx, ky, kz};
            const int off[3] = {o8 & 1, (o8 >> 1) & 1, o8 >> 2};
            const int f[3] = {2 * kx + off[0], 2 * ky + off[1], 2 * kz + off[2]};
            if (f[0] < b.rlo[0] || f[0] > b.rhi[0] || f[1] < b.rlo[1] || f[1] > b.rhi[1] ||
                f[2] < b.rlo[2] || f[2] > b.rhi[2])
              continue;
            const int64_t ridx = (f[0] - b.rlo[0]) + (int64_t)rnx * ((f[1] - b.rlo[1]) +
                                                                    (int64_t)rny * (f[2] - b.rlo[2]));
            int sh[3] = {0, 0, 0};
            int fbk = 0;
            if (shifts)
              for (int d = 0; d < 3; ++d)
                sh[d] = shifts[3 * (blk * rnp + ridx) + d];
            if (fallback)
              fbk = fallback[blk * rnp + ridx];
            int k[3], o[3], r[3][2];
            bool inside = true, anymm = false;
            for (int d = 0; d < 3; ++d) {
              if (fbk)
                sh[d] = 0;
              k[d] = fbk ? lin[d] : kind[d];
              o[d] = cc[d] - ic[d];
              radius(k[d], sh[d], off[d], r[d]);
              inside = inside && o[d] >= r[d][0] && o[d] <= r[d][1];
              anymm = anymm || (fbk ? mml[d] : mm[d]);
            }
            if (!inside)
              continue;
            double w;
            if (!anymm) {
              w = tab.w[0][fbk][sh[0] + 1][off[0]][o[0] + 4] *
                  tab.w[1][fbk][sh[1] + 1][off[1]][o[1] + 4] *
                  tab.w[2][fbk][sh[2] + 1][off[2]][o[2] + 4];
            } else {
              // re-evaluate the passes of f's stencil (call_stencil_3d order)
              double X[9][9], Y[9];
              for (int dk = r[2][0]; dk <= r[2][1]; ++dk) {
                for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
                  double v[9];
                  for (int di = r[0][0]; di <= r[0][1]; ++di)
                    v[di + 4] = crs(comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
                  X[dk + 4][dj + 4] = ap_rt(k[0], sh[0], off[0], v + 4);
                }
                Y[dk + 4] = ap_rt(k[1], sh[1], off[1], X[dk + 4] + 4);
              }
              double wz, wy, wx, t[3];
              if (k[2] == K_CC_MINMOD1) {
                minmod_weights(off[2], Y + 4, t);
                wz = t[o[2] + 1];
              } else {
                wz = tab.w[2][fbk][sh[2] + 1][off[2]][o[2] + 4];
              }
              if (k[1] == K_CC_MINMOD1) {
                minmod_weights(off[1], X[o[2] + 4] + 4, t);
                wy = t[o[1] + 1];
              } else {
                wy = tab.w[1][fbk][sh[1] + 1][off[1]][o[1] + 4];
              }
              if (k[0] == K_CC_MINMOD1) {
                double v[3];
                for (int di = -1; di <= 1; ++di)
                  v[di + 1] = crs(comp, ic[0] + di, ic[1] + o[1], ic[2] + o[2]);
                minmod_weights(off[0], v + 1, t);
                wx = t[o[0] + 1];
              } else {
                wx = tab.w[0][fbk][sh[0] + 1][off[0]][o[0] + 4];
              }
              w = wz * wy * wx;
            }
            acc = fma(w, b.fine[comp * b.fnp + (f[0] - b.flo[0]) + (int64_t)b.fnx * (f[1] - b.flo[1]) +
                                fplane * (f[2] - b.flo[2])],
                      acc);
          }
    crse_bar[comp * b.cnp + idx] = acc;
  }
}

} // namespace

cudaError_t launch_point_box(const BoxDesc &b, int per_group, signed char *shifts,
                             unsigned char *fallback, cudaStream_t s, bool after_level) {
  if (eno_cell_applies(b, per_group)) // all directions ENO, no fallback
    return launch_eno_cell_box(b, per_group, shifts, fallback, s, after_level);
  const int64_t rnp = (int64_t)(b.rhi[0] - b.rlo[0] + 1) * (b.rhi[1] - b.rlo[1] + 1) *
                      (b.rhi[2] - b.rlo[2] + 1);
  if (rnp <= 0 || b.ncomp <= 0)
    return cudaSuccess;
  const int64_t nblk = (rnp + 255) / 256;
  if (nblk > INT32_MAX)
    return cudaErrorInvalidValue;
  dim3 grid((unsigned)nblk, per_group ? 1 : b.ncomp);
  point_box_kernel<<<grid, 256, 0, s>>>(b, per_group, shifts, fallback);
  return cudaGetLastError();
}

// Scratch the adjoint of a limited operator needs on one box: the ENO shift
// (3 bytes) and fallback flag (1 byte) of every region point and component
// block, when it has ENO directions or an active linear fallback; else 0.
size_t point_adjoint_scratch_bytes(const BoxDesc &b, int per_group) {
  if (eno_cell_applies(b, per_group))
    return eno_adjoint_scratch_bytes(b, per_group);
  const int64_t rnp = (int64_t)(b.rhi[0] - b.rlo[0] + 1) * (b.rhi[1] - b.rlo[1] + 1) *
                      (b.rhi[2] - b.rlo[2] + 1);
  bool eno = false;
  for (int d = 0; d < 3; ++d)
    eno = eno || b.kind[d] == K_CC_ENO2;
  if (b.ncomp <= 0 || rnp <= 0 || !(eno || op_fb_active(b.op, per_group)))
    return 0;
  return (size_t)4 * rnp * (per_group ? 1 : b.ncomp);
}

// Adjoint of a limited operator on one box with the caller's scratch (at
// least point_adjoint_scratch_bytes): decision pass (the ENO shift and
// fallback flag of every region point, recomputed from crse), then the
// gather.  fine in b holds fine_bar.
cudaError_t launch_point_adjoint_box_scratch(const BoxDesc &b, int per_group, double *crse_bar,
                                             void *scratch, cudaStream_t s) {
  if (b.ncomp <= 0 || b.cnp <= 0)
    return cudaSuccess;
  if (eno_cell_applies(b, per_group)) // all directions ENO: per-cell shifts, tiled gather
    return launch_eno_adjoint_box(b, per_group, scratch, crse_bar, s);
  if (minmod_cell_applies(b)) // all directions minmod: tiled transposed passes
    return launch_minmod_adjoint_box(b, crse_bar, s);
  const int nblk = per_group ? 1 : b.ncomp;
  const size_t need = point_adjoint_scratch_bytes(b, per_group);
  signed char *sh = nullptr;
  unsigned char *fb = nullptr;
  cudaError_t e = cudaSuccess;
  if (need) {
    if (!scratch)
      return cudaErrorInvalidValue;
    const size_t n = need / 4;
    sh = static_cast<signed char *>(scratch);
    fb = reinterpret_cast<unsigned char *>(sh + 3 * n);
    BoxDesc d = b;
    d.fine = nullptr; // decisions only
    e = launch_point_box(d, per_group, sh, fb, s);
  }
  if (e == cudaSuccess) {
    const int64_t nb = (b.cnp + AT_NT - 1) / AT_NT;
    if (nb > INT32_MAX)
      return cudaErrorInvalidValue;
    adjoint_point_kernel<<<dim3((unsigned)nb, nblk), AT_NT, 0, s>>>(b, per_group, sh, fb,
                                                                     crse_bar);
    e = cudaGetLastError();
  }
  return e;
}

// The same for one box with stream-ordered scratch (cudaMallocAsync /
// cudaFreeAsync around the launches).
cudaError_t launch_point_adjoint_box(const BoxDesc &b, int per_group, double *crse_bar,
                                     cudaStream_t s) {
  const size_t need = point_adjoint_scratch_bytes(b, per_group);
  void *scratch = nullptr;
  if (need) {
    const cudaError_t e = cudaMallocAsync(&scratch, need, s);
    if (e != cudaSuccess)
      return e;
  }
  cudaError_t e = launch_point_adjoint_box_scratch(b, per_group, crse_bar, scratch, s);
  if (scratch) {
    const cudaError_t e2 = cudaFreeAsync(scratch, s);
    if (e == cudaSuccess)
      e = e2;
  }
  return e;
}

} // namespace cxb
