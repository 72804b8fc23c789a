/* CPU restatement of CarpetX's refinement-factor-2 prolongation operators and
 * of AMReX's average_down restriction.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, used by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.  Never linked into
 * the product.
 *
 * Reference: CarpetX/src/prolongate_3d_rf2_impl.hxx (cited per function).
 * Coefficients are derived here from exact rational interpolation (the method
 * of CarpetX/stencils/stencils.jl:36-278), independently of the product's own
 * derivation; the tests pin both against the reference build in oracle/_ref.
 * Compile with -ffp-contract=off: every `y += c * x` below must round the
 * product and the sum separately, as the reference does on the host. */
#include "cx_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Exact rationals for the coefficient derivation                            */

typedef struct {
  __int128 n, d;
} rat;

static __int128 gcd128(__int128 a, __int128 b) {
  if (a < 0)
    a = -a;
  if (b < 0)
    b = -b;
  while (b) {
    __int128 t = a % b;
    a = b;
    b = t;
  }
  return a;
}
static rat mkrat(__int128 n, __int128 d) {
  if (d < 0) {
    n = -n;
    d = -d;
  }
  __int128 g = gcd128(n, d);
  if (g == 0)
    g = 1;
  rat r = {n / g, d / g};
  return r;
}
static rat ri(long long n) { return mkrat(n, 1); }
static rat radd(rat a, rat b) { return mkrat(a.n * b.d + b.n * a.d, a.d * b.d); }
static rat rsub(rat a, rat b) { return mkrat(a.n * b.d - b.n * a.d, a.d * b.d); }
static rat rmul(rat a, rat b) { return mkrat(a.n * b.n, a.d * b.d); }
static rat rdiv(rat a, rat b) { return mkrat(a.n * b.d, a.d * b.n); }
static double rat2d(rat a) {
  /* all live coefficients are dyadic with |num| < 2^53: exact */
  return (double)(long long)a.n / (double)(long long)a.d;
}

/* Lagrange basis polynomial k over nodes xs[0..n-1], evaluated at x. */
static rat lagrange(const rat *xs, int n, int k, rat x) {
  rat r = ri(1);
  for (int m = 0; m < n; ++m)
    if (m != k)
      r = rmul(r, rdiv(rsub(x, xs[m]), rsub(xs[k], xs[m])));
  return r;
}

/* Average over [xl, xh] of the polynomial whose cell averages over the unit
 * cells centred at cells[0..n-1] (consecutive) are the data: weight of each
 * cell, via interpolation of the primitive at the n+1 cell boundaries. */
static void cons_weights(const int *cells, int n, rat xl, rat xh, rat *w) {
  rat bs[16];
  for (int k = 0; k <= n; ++k)
    bs[k] = radd(ri(cells[0]), mkrat(2 * k - 1, 2));
  for (int m = 0; m < n; ++m) {
    rat s = ri(0);
    for (int k = m + 1; k <= n; ++k)
      s = radd(s, rsub(lagrange(bs, n + 1, k, xh), lagrange(bs, n + 1, k, xl)));
    w[m] = rdiv(s, rsub(xh, xl));
  }
}

#define MAXP 11
static double vc_poly[MAXP + 1][MAXP + 1];
static double cc_poly[MAXP + 1][MAXP + 1];
static double cc_cons[MAXP + 1][MAXP + 1];
static double cc_eno2[3][3];
static double cc_eno4[5][5];
static int coeffs_ready = 0;

static void init_coeffs(void) {
  if (coeffs_ready)
    return;
  /* VC POLY p (odd): nodes i - (N/2 - 1), evaluated at the midpoint 1/2
   * (coeffs1d<VC,POLY,p>, impl.hxx:59-99) */
  for (int p = 1; p <= MAXP; p += 2) {
    const int N = p + 1, i0 = N / 2 - 1;
    rat xs[MAXP + 1];
    for (int i = 0; i < N; ++i)
      xs[i] = ri(i - i0);
    for (int i = 0; i < N; ++i)
      vc_poly[p][i] = rat2d(lagrange(xs, N, i, mkrat(1, 2)));
  }
  /* CC POLY p: cell centres i - N/2, evaluated at the left child -1/4
   * (coeffs1d<CC,POLY,p>, impl.hxx:101-186) */
  for (int p = 0; p <= MAXP; ++p) {
    const int N = p + 1, i0 = N / 2;
    rat xs[MAXP + 1];
    for (int i = 0; i < N; ++i)
      xs[i] = ri(i - i0);
    for (int i = 0; i < N; ++i)
      cc_poly[p][i] = rat2d(lagrange(xs, N, i, mkrat(-1, 4)));
  }
  /* CC CONS p: cells i - N/2, average over the left half [-1/2, 0]
   * (coeffs1d<CC,CONS,p>, impl.hxx:237-314) */
  for (int p = 0; p <= MAXP; ++p) {
    const int N = p + 1;
    int cells[MAXP + 1];
    rat w[MAXP + 1];
    for (int i = 0; i < N; ++i)
      cells[i] = i - N / 2;
    cons_weights(cells, N, mkrat(-1, 2), ri(0), w);
    for (int i = 0; i < N; ++i)
      cc_cons[p][i] = rat2d(w[i]);
  }
  /* CC ENO p (even): row m uses cells i - (N/2 - shift), shift = m - p/2
   * (coeffs1d<CC,ENO,p>, impl.hxx:316-384) */
  for (int p = 2; p <= 4; p += 2) {
    const int N = p + 1;
    for (int m = 0; m < N; ++m) {
      const int shift = m - p / 2;
      int cells[5];
      rat w[5];
      for (int i = 0; i < N; ++i)
        cells[i] = i - (N / 2 - shift);
      cons_weights(cells, N, mkrat(-1, 2), ri(0), w);
      for (int i = 0; i < N; ++i) {
        if (p == 2)
          cc_eno2[m][i] = rat2d(w[i]);
        else
          cc_eno4[m][i] = rat2d(w[i]);
      }
    }
  }
  coeffs_ready = 1;
}

__attribute__((constructor)) static void cxo_init(void) { init_coeffs(); }

int cxo_coeffs(int cent, int intp, int order, int row, double *out) {
  init_coeffs();
  const int N = order + 1;
  if (order < 0 || order > MAXP)
    return 0;
  if (cent == CXO_VC && (intp == CXO_POLY || intp == CXO_HERMITE)) {
    if (order % 2 == 0)
      return 0;
    memcpy(out, vc_poly[order], N * sizeof(double));
    return N;
  }
  if (cent == CXO_CC && intp == CXO_POLY) {
    memcpy(out, cc_poly[order], N * sizeof(double));
    return N;
  }
  if (cent == CXO_CC && intp == CXO_CONS) {
    memcpy(out, cc_cons[order], N * sizeof(double));
    return N;
  }
  if (cent == CXO_CC && intp == CXO_ENO && (order == 2 || order == 4) &&
      row >= 0 && row < N) {
    memcpy(out, order == 2 ? cc_eno2[row] : cc_eno4[row], N * sizeof(double));
    return N;
  }
  if (cent == CXO_VC && intp == CXO_CONS && (order == 0 || order == 1)) {
    /* deprecated VC CONS (impl.hxx:220-235): row 0 = on-point, row 1 =
     * midpoint */
    if (row == 0) {
      out[0] = 1.0;
      return 1;
    }
    if (order == 0)
      return 0;
    out[0] = 0.5;
    out[1] = 0.5;
    return 2;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Operator tables (prolongate_3d_rf2_impl_*.cxx, get_interpolator)          */

static void set_dirs(cxo_op *op, int indextype, int vc_intp, int vc_order,
                     int cc_intp, int cc_order, int fb) {
  for (int d = 0; d < 3; ++d) {
    op->cent[d] = (indextype >> (2 - d)) & 1;
    if (op->cent[d] == CXO_VC) {
      op->intp[d] = vc_intp;
      op->order[d] = vc_order;
    } else {
      op->intp[d] = cc_intp;
      op->order[d] = cc_order;
    }
  }
  op->fb = fb;
}

int cxo_lookup(const char *type, int o, int indextype, cxo_op *op) {
  if (!type || !op || indextype < 0 || indextype > 7)
    return -1;
  if (!strcmp(type, "interpolate")) { /* impl_poly.cxx */
    if (o != 1 && o != 3 && o != 5 && o != 7)
      return -1;
    set_dirs(op, indextype, CXO_POLY, o, CXO_POLY, o, CXO_FB_NONE);
  } else if (!strcmp(type, "conservative")) { /* impl_cons.cxx */
    if (o == 0)
      set_dirs(op, indextype, CXO_CONS, 0, CXO_CONS, 0, CXO_FB_NONE);
    else if (o == 1)
      set_dirs(op, indextype, CXO_CONS, 1, CXO_CONS, 2, CXO_FB_NONE);
    else
      return -1;
  } else if (!strcmp(type, "ddf")) { /* impl_ddf.cxx */
    if (o != 1 && o != 3 && o != 5 && o != 7)
      return -1;
    set_dirs(op, indextype, CXO_POLY, o, CXO_CONS, o - 1, CXO_FB_NONE);
  } else if (!strcmp(type, "eno")) { /* impl_eno.cxx */
    if (o != 3 && o != 5)
      return -1;
    set_dirs(op, indextype, CXO_POLY, o, CXO_ENO, 2, CXO_FB_NONE);
  } else if (!strcmp(type, "minmod")) { /* impl_minmod.cxx */
    if (o != 1 && o != 3 && o != 5)
      return -1;
    set_dirs(op, indextype, CXO_POLY, o, CXO_MINMOD, 1, CXO_FB_NONE);
  } else if (!strcmp(type, "hermite")) { /* impl_hermite.cxx */
    if (o != 1 && o != 3 && o != 5)
      return -1;
    set_dirs(op, indextype, CXO_HERMITE, o, CXO_CONS, o, CXO_FB_NONE);
  } else if (!strcmp(type, "natural")) { /* impl_natural.cxx */
    if (o != 1 && o != 3 && o != 5 && o != 7)
      return -1;
    set_dirs(op, indextype, CXO_POLY, o, CXO_CONS, o, CXO_FB_NONE);
  } else if (!strcmp(type, "poly-cons3lfb")) { /* impl_poly_cons3lfb.cxx */
    if (o != 1 && o != 3 && o != 5)
      return -1;
    set_dirs(op, indextype, CXO_POLY, o, CXO_CONS, o < 3 ? o : 3,
             CXO_FB_LINEAR);
  } else if (!strcmp(type, "poly-eno3lfb")) { /* impl_poly_eno3lfb.cxx */
    if (o == 1)
      set_dirs(op, indextype, CXO_POLY, 1, CXO_CONS, 0, CXO_FB_LINEAR);
    else if (o == 3 || o == 5)
      set_dirs(op, indextype, CXO_POLY, o, CXO_ENO, 2, CXO_FB_LINEAR);
    else
      return -1;
  } else {
    return -1;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* 1-D stencils (interp1d<...>, impl.hxx:396-878)                            */

static int req_ghosts_1d(int cent, int intp, int p) {
  if (intp == CXO_ENO)
    return p; /* impl.hxx:783 */
  if (intp == CXO_MINMOD)
    return 1; /* impl.hxx:847 */
  (void)cent;
  return (p + 1) / 2; /* impl.hxx:398,462,518,585,636 */
}

void cxo_required_ghosts(const cxo_op *op, int g[3]) {
  for (int d = 0; d < 3; ++d)
    g[d] = req_ghosts_1d(op->cent[d], op->intp[d], op->order[d]);
}

static int floor2(int i) { return i >= 0 ? i / 2 : -((-i + 1) / 2); }

void cxo_coarse_box(const cxo_op *op, const int flo[3], const int fhi[3],
                    int clo[3], int chi[3]) {
  int g[3];
  cxo_required_ghosts(op, g);
  for (int d = 0; d < 3; ++d) {
    clo[d] = floor2(flo[d]) - g[d];
    chi[d] = floor2(fhi[d]) + g[d];
  }
}

/* stencil_radius(shift, off) */
static void radius_1d(int cent, int intp, int p, int shift, int off, int r[2]) {
  const int N = p + 1;
  if (cent == CXO_VC && (intp == CXO_POLY || intp == CXO_HERMITE)) {
    /* impl.hxx:402-408, 522-531 */
    if (off == 0) {
      r[0] = 0;
      r[1] = 0;
    } else {
      const int i0 = N / 2 - off;
      r[0] = -i0;
      r[1] = p - i0;
    }
  } else if (cent == CXO_CC && intp == CXO_POLY) { /* impl.hxx:466-476 */
    const int i0 = N / 2;
    r[0] = -i0 + (off ? p % 2 : 0);
    r[1] = N - 1 - i0 + (off ? p % 2 : 0);
  } else if (cent == CXO_VC && intp == CXO_CONS) { /* impl.hxx:588-601 */
    if (off == 0) {
      const int i0 = p / 2;
      r[0] = -i0;
      r[1] = p / 2 * 2 - i0;
    } else {
      const int i0 = (p + 1) / 2 - 1;
      r[0] = -i0;
      r[1] = (p + 1) / 2 * 2 - 1 - i0;
    }
  } else if (cent == CXO_CC && intp == CXO_CONS) { /* impl.hxx:640-649 */
    if (off == 0) {
      r[0] = -((p + 1) / 2);
      r[1] = p / 2;
    } else {
      r[0] = -(p / 2);
      r[1] = (p + 1) / 2;
    }
  } else if (cent == CXO_CC && intp == CXO_ENO) { /* impl.hxx:786-803 */
    const int i0 = N / 2 - shift;
    r[0] = -i0;
    r[1] = p - i0;
  } else { /* CC MINMOD, impl.hxx:850-856 */
    r[0] = -1;
    r[1] = 1;
  }
}

/* v[o] is the value at offset o (v points at offset 0). */
static double interp_1d(int cent, int intp, int p, int shift, int off,
                        const double *v) {
  const int N = p + 1;
  double y;
  if (cent == CXO_VC && (intp == CXO_POLY || intp == CXO_HERMITE)) {
    /* impl.hxx:411-456 and 533-578: pairs of symmetric taps */
    if (off == 0)
      return v[0];
    const double *cs = vc_poly[p];
    const int i0 = N / 2 - off;
    y = 0;
    for (int i = 0; i < N / 2; ++i)
      y += cs[i] * (v[i - i0] + v[p - i - i0]);
    return y;
  }
  if (cent == CXO_CC && intp == CXO_POLY) { /* impl.hxx:478-511 */
    const double *cs = cc_poly[p];
    const int i0 = N / 2;
    y = 0;
    if (off == 0)
      for (int i = 0; i < N; ++i)
        y += cs[i] * v[i - i0];
    else
      for (int i = 0; i < N; ++i)
        y += cs[p - i] * v[i - i0 + p % 2];
    return y;
  }
  if (cent == CXO_VC && intp == CXO_CONS) { /* impl.hxx:603-630 */
    y = 0;
    if (off == 0) {
      const int i0 = p / 2;
      for (int i = 0; i < p / 2 * 2 + 1; ++i)
        y += 1.0 * v[i - i0]; /* coeffs0 = {1} for p = 0, 1 */
    } else {
      const int i0 = (p + 1) / 2 - 1;
      for (int i = 0; i < (p + 1) / 2 * 2; ++i)
        y += 0.5 * v[i - i0]; /* coeffs1 = {} (p = 0), {1/2, 1/2} (p = 1) */
    }
    return y;
  }
  if (cent == CXO_CC && intp == CXO_CONS) { /* impl.hxx:651-715 */
    const double *cs = cc_cons[p];
    const int i0 = N / 2;
    if (p % 2 == 0) {
      y = cs[p / 2] * v[p / 2 - i0];
      if (off == 0)
        for (int i = 0; i < p / 2; ++i)
          y += cs[i] * (v[i - i0] - v[p - i - i0]);
      else
        for (int i = 0; i < p / 2; ++i)
          y += cs[i] * (v[p - i - i0] - v[i - i0]);
    } else {
      y = 0;
      if (off == 0)
        for (int i = 0; i < N; ++i)
          y += cs[i] * v[i - i0];
      else
        for (int i = 0; i < N; ++i)
          y += cs[i] * v[(p + 1) / 2 - i];
    }
    return y;
  }
  if (cent == CXO_CC && intp == CXO_ENO) { /* impl.hxx:806-841 */
    const int m = off == 0 ? shift + p / 2 : p / 2 - shift;
    const double *cs = p == 2 ? cc_eno2[m] : cc_eno4[m];
    const int i0 = N / 2 - shift;
    y = 0;
    if (off == 0)
      for (int i = 0; i <= p; ++i)
        y += cs[i] * v[i - i0];
    else
      for (int i = 0; i <= p; ++i)
        y += cs[p - i] * v[i - i0];
    return y;
  }
  { /* CC MINMOD, impl.hxx:859-877 */
    const double cval = v[0], cm = v[-1], cp = v[1];
    const double dm = cval - cm, dp = cp - cval;
    const double delta =
        (copysign(0.125, dm) + copysign(0.125, dp)) * fmin(fabs(dm), fabs(dp));
    const double sign = off == 0 ? -1 : +1;
    return cval + sign * delta;
  }
}

/* Linearisation of interp_1d at v: weights w[o] (w points at offset 0) over
 * the stencil radius, zero elsewhere in [-4, 4]. */
static void weights_1d(int cent, int intp, int p, int shift, int off,
                       const double *v, double *w) {
  for (int o = -4; o <= 4; ++o)
    w[o] = 0;
  int r[2];
  radius_1d(cent, intp, p, shift, off, r);
  if (intp == CXO_MINMOD) {
    const double dm = v[0] - v[-1], dp = v[1] - v[0];
    const double sgn = off == 0 ? -1 : +1;
    w[0] = 1;
    const double f = copysign(0.125, dm) + copysign(0.125, dp);
    if (f != 0) {
      /* delta = f * min(|dm|, |dp|) = 0.25 * (chosen difference) */
      if (fabs(dm) <= fabs(dp)) { /* fmin picks dm on ties */
        w[0] += sgn * 0.25;
        w[-1] -= sgn * 0.25;
      } else {
        w[1] += sgn * 0.25;
        w[0] -= sgn * 0.25;
      }
    }
    return;
  }
  double e[9];
  for (int o = r[0]; o <= r[1]; ++o) {
    memset(e, 0, sizeof e);
    e[o + 4] = 1;
    w[o] = interp_1d(cent, intp, p, shift, off, e + 4);
  }
}

/* undivided_difference_1d<CC,ENO,p> (impl.hxx:751-773) */
static double undiv_1d(int p, const double *v) {
  static const int w3[3] = {+1, -2, +1};
  static const int w5[5] = {+1, -4, +6, -4, +1};
  const int *ws = p == 2 ? w3 : w5;
  double dd = ws[p / 2] * v[0];
  for (int i = 0; i < p / 2; ++i)
    dd += ws[i] * (v[i - p / 2] + v[p - i - p / 2]);
  return dd;
}

/* ------------------------------------------------------------------------ */
/* 3-D evaluation (call_stencil_3d, impl.hxx:1178-1216)                      */

typedef struct {
  const double *ptr; /* component 0 */
  long np;           /* component stride */
  int lo[3];
  int nx, ny;
} cbox;

static inline double cget(const cbox *c, int comp, int i, int j, int k) {
  return c->ptr[comp * c->np + (i - c->lo[0]) +
                (long)c->nx * ((j - c->lo[1]) + (long)c->ny * (k - c->lo[2]))];
}

typedef struct {
  int cent, intp, p;
} dspec;

/* z stencil over (y stencil over (x stencil)) of the coarse values around
 * ic, as in call_stencil_3d. */
static double eval3d(const dspec s[3], const int shift[3], const int off[3],
                     const cbox *c, int comp, const int ic[3]) {
  int r[3][2];
  for (int d = 0; d < 3; ++d)
    radius_1d(s[d].cent, s[d].intp, s[d].p, shift[d], off[d], r[d]);
  double Y[9];
  for (int dk = r[2][0]; dk <= r[2][1]; ++dk) {
    double X[9];
    for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
      double v[9];
      for (int di = r[0][0]; di <= r[0][1]; ++di)
        v[di + 4] = cget(c, comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
      X[dj + 4] = interp_1d(s[0].cent, s[0].intp, s[0].p, shift[0], off[0],
                            v + 4);
    }
    Y[dk + 4] =
        interp_1d(s[1].cent, s[1].intp, s[1].p, shift[1], off[1], X + 4);
  }
  return interp_1d(s[2].cent, s[2].intp, s[2].p, shift[2], off[2], Y + 4);
}

/* Gradient of eval3d with respect to the coarse values, added (times g) into
 * cbar (same layout as c). */
static void eval3d_adjoint(const dspec s[3], const int shift[3],
                           const int off[3], const cbox *c, int comp,
                           const int ic[3], double g, double *cbar) {
  int r[3][2];
  for (int d = 0; d < 3; ++d)
    radius_1d(s[d].cent, s[d].intp, s[d].p, shift[d], off[d], r[d]);
  double X[9][9], Y[9], wz[9], wy[9][9];
  for (int dk = r[2][0]; dk <= r[2][1]; ++dk) {
    for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
      double v[9];
      for (int di = r[0][0]; di <= r[0][1]; ++di)
        v[di + 4] = cget(c, comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
      X[dk + 4][dj + 4] = interp_1d(s[0].cent, s[0].intp, s[0].p, shift[0],
                                    off[0], v + 4);
    }
    Y[dk + 4] = interp_1d(s[1].cent, s[1].intp, s[1].p, shift[1], off[1],
                          X[dk + 4] + 4);
    weights_1d(s[1].cent, s[1].intp, s[1].p, shift[1], off[1], X[dk + 4] + 4,
               wy[dk + 4] + 4);
  }
  weights_1d(s[2].cent, s[2].intp, s[2].p, shift[2], off[2], Y + 4, wz + 4);
  for (int dk = r[2][0]; dk <= r[2][1]; ++dk)
    for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
      double v[9], wx[9];
      for (int di = r[0][0]; di <= r[0][1]; ++di)
        v[di + 4] = cget(c, comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
      weights_1d(s[0].cent, s[0].intp, s[0].p, shift[0], off[0], v + 4,
                 wx + 4);
      const double wzy = wz[dk + 4] * wy[dk + 4][dj + 4];
      for (int di = r[0][0]; di <= r[0][1]; ++di) {
        const long idx = comp * c->np + (ic[0] + di - c->lo[0]) +
                         (long)c->nx * ((ic[1] + dj - c->lo[1]) +
                                        (long)c->ny * (ic[2] + dk - c->lo[2]));
        cbar[idx] += wzy * wx[di + 4] * g;
      }
    }
}

/* ENO shift choice (impl.hxx:1415-1517 per var, 1857-1965 per group): the
 * candidate with the smallest penalised maximum undivided difference, first
 * minimum in (sk, sj, si) order.  Components c0..c1-1 are searched. */
static void choose_shift(const cxo_op *op, const dspec s[3], const int off[3],
                         const cbox *c, int c0, int c1, const int ic[3],
                         int shift[3]) {
  int use_shift[3], maxshift[3];
  int any = 0;
  for (int d = 0; d < 3; ++d) {
    use_shift[d] = op->intp[d] == CXO_ENO && op->order[d] > 0;
    maxshift[d] =
        use_shift[d] ? req_ghosts_1d(s[d].cent, s[d].intp, s[d].p) / 2 : 0;
    any |= use_shift[d];
    shift[d] = 0;
  }
  if (!any)
    return;
  double min_dd = 1.0 / 0.0;
  for (int sk = -maxshift[2]; sk <= maxshift[2]; ++sk)
    for (int sj = -maxshift[1]; sj <= maxshift[1]; ++sj)
      for (int si = -maxshift[0]; si <= maxshift[0]; ++si) {
        const int sh[3] = {si, sj, sk};
        int r[3][2];
        for (int d = 0; d < 3; ++d) {
          radius_1d(s[d].cent, s[d].intp, s[d].p, sh[d], off[d], r[d]);
          if (use_shift[d]) {
            r[d][0] -= sh[d];
            r[d][1] -= sh[d];
          }
        }
        double ddx = 0, ddy = 0, ddz = 0;
        for (int comp = c0; comp < c1; ++comp) {
          if (use_shift[0])
            for (int dk = r[2][0]; dk <= r[2][1]; ++dk)
              for (int dj = r[1][0]; dj <= r[1][1]; ++dj) {
                double v[9];
                for (int o = -s[0].p / 2; o <= s[0].p / 2; ++o)
                  v[o + 4] = cget(c, comp, ic[0] + si + o, ic[1] + sj + dj,
                                  ic[2] + sk + dk);
                ddx = fmax(ddx, fabs(undiv_1d(s[0].p, v + 4)));
              }
          if (use_shift[1])
            for (int dk = r[2][0]; dk <= r[2][1]; ++dk)
              for (int di = r[0][0]; di <= r[0][1]; ++di) {
                double v[9];
                for (int o = -s[1].p / 2; o <= s[1].p / 2; ++o)
                  v[o + 4] = cget(c, comp, ic[0] + si + di, ic[1] + sj + o,
                                  ic[2] + sk + dk);
                ddy = fmax(ddy, fabs(undiv_1d(s[1].p, v + 4)));
              }
          if (use_shift[2])
            for (int dj = r[1][0]; dj <= r[1][1]; ++dj)
              for (int di = r[0][0]; di <= r[0][1]; ++di) {
                double v[9];
                for (int o = -s[2].p / 2; o <= s[2].p / 2; ++o)
                  v[o + 4] = cget(c, comp, ic[0] + si + di, ic[1] + sj + dj,
                                  ic[2] + sk + o);
                ddz = fmax(ddz, fabs(undiv_1d(s[2].p, v + 4)));
              }
        }
        const double penalty =
            1 + sqrt(DBL_EPSILON) * (abs(si) + abs(sj) + abs(sk));
        const double dd = penalty * fmax(fmax(ddx, ddy), ddz);
        if (dd < min_dd) {
          min_dd = dd;
          shift[0] = si;
          shift[1] = sj;
          shift[2] = sk;
        }
      }
}

/* Slope sign-change test in direction d over the stencil (fallback condition
 * 2, impl.hxx:1609-1664 and 2026-2115).  s0 is always taken between offsets
 * 0 and 1, the loop starts at radius[0] + 2, as in the reference. */
static int slope_change(int d, const int sr[3][2], const cbox *c, int comp,
                        const int ic[3]) {
  int need = 0;
  int o1[3], o2[3];
  /* the two other directions, outer = higher index */
  int in_d = d == 0 ? 1 : 0, out_d = d == 2 ? 1 : 2;
  for (int q = sr[out_d][0]; q <= sr[out_d][1]; ++q)
    for (int t = sr[in_d][0]; t <= sr[in_d][1]; ++t) {
      o1[out_d] = q;
      o1[in_d] = t;
      o2[out_d] = q;
      o2[in_d] = t;
      o1[d] = 1;
      o2[d] = 0;
      const double s0 =
          cget(c, comp, ic[0] + o1[0], ic[1] + o1[1], ic[2] + o1[2]) -
          cget(c, comp, ic[0] + o2[0], ic[1] + o2[1], ic[2] + o2[2]);
      for (int e = sr[d][0] + 2; e <= sr[d][1]; ++e) {
        o1[d] = e;
        o2[d] = e - 1;
        const double sl =
            cget(c, comp, ic[0] + o1[0], ic[1] + o1[1], ic[2] + o1[2]) -
            cget(c, comp, ic[0] + o2[0], ic[1] + o2[1], ic[2] + o2[2]);
        need |= sl * s0 < 0;
      }
    }
  return need;
}

static int box_ok(const int lo[3], const int hi[3]) {
  return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2];
}

/* Per-point work shared by the forward operator and its adjoint: decides
 * the shift and the fallback and returns the stencil specification used. */
typedef struct {
  dspec s[3], lin[3];
  int fb_active;
} opspec;

static void make_spec(const cxo_op *op, int per_group, opspec *sp) {
  int all_off = 1;
  for (int d = 0; d < 3; ++d) {
    sp->s[d].cent = op->cent[d];
    sp->s[d].intp = op->intp[d];
    sp->s[d].p = op->order[d];
    const int is_cons_like =
        per_group ? op->intp[d] == CXO_CONS
                  : (op->intp[d] == CXO_CONS || op->intp[d] == CXO_ENO);
    if (is_cons_like && op->order[d] > 1)
      all_off = 0;
    if (per_group) { /* impl.hxx:2119-2121 */
      sp->lin[d].cent = op->cent[d];
      sp->lin[d].intp = op->intp[d];
      sp->lin[d].p = op->intp[d] == CXO_CONS ? 1 : op->order[d];
    } else { /* impl.hxx:1547-1558 */
      const int cl = op->intp[d] == CXO_CONS || op->intp[d] == CXO_ENO;
      sp->lin[d].cent = op->cent[d];
      sp->lin[d].intp = cl ? CXO_CONS : op->intp[d];
      sp->lin[d].p = cl ? 1 : op->order[d];
    }
  }
  /* impl.hxx:1535-1538 (per var), 1990-1992 (per group) */
  sp->fb_active = op->fb == CXO_FB_LINEAR && !all_off;
}

/* Decides shift and fallback for one fine point; vals[comp] are the
 * high-order values for components c0..c1-1 (filled here). */
static int decide_point(const cxo_op *op, int per_group, const opspec *sp,
                        const cbox *c, int c0, int c1, const int ic[3],
                        const int off[3], int shift[3], double *vals) {
  choose_shift(op, sp->s, off, c, c0, c1, ic, shift);
  for (int comp = c0; comp < c1; ++comp)
    vals[comp - c0] = eval3d(sp->s, shift, off, c, comp, ic);
  if (!sp->fb_active)
    return 0;
  int sr[3][2];
  for (int d = 0; d < 3; ++d)
    radius_1d(sp->s[d].cent, sp->s[d].intp, sp->s[d].p, shift[d], off[d],
              sr[d]);
  int need = 0;
  double minval = +1.0 / 0.0, maxval = -1.0 / 0.0;
  for (int comp = c0; comp < c1; ++comp) {
    if (!per_group) {
      minval = +1.0 / 0.0;
      maxval = -1.0 / 0.0;
    }
    for (int dk = sr[2][0]; dk <= sr[2][1]; ++dk)
      for (int dj = sr[1][0]; dj <= sr[1][1]; ++dj)
        for (int di = sr[0][0]; di <= sr[0][1]; ++di) {
          const double x = cget(c, comp, ic[0] + di, ic[1] + dj, ic[2] + dk);
          minval = fmin(minval, x);
          maxval = fmax(maxval, x);
        }
    need |= vals[comp - c0] < minval || vals[comp - c0] > maxval;
  }
  for (int d = 0; d < 3; ++d) {
    const int check = per_group
                          ? op->intp[d] == CXO_CONS
                          : (op->intp[d] == CXO_CONS || op->intp[d] == CXO_ENO);
    if (!check)
      continue;
    for (int comp = c0; comp < c1; ++comp)
      need |= slope_change(d, sr, c, comp, ic);
  }
  return need;
}

static int check_args(const cxo_op *op, const double *crse, const int clo[3],
                      const int chi[3], const void *fine, const int flo[3],
                      const int fhi[3], const int rlo[3], const int rhi[3],
                      int ncomp) {
  if (!op || !crse || !fine || ncomp < 0)
    return -1;
  if (!box_ok(clo, chi) || !box_ok(flo, fhi))
    return -1;
  for (int d = 0; d < 3; ++d)
    if (rlo[d] < flo[d] || rhi[d] > fhi[d])
      return -1;
  return 0;
}

int cxo_prolong(const cxo_op *op, int per_group, const double *crse,
                const int clo[3], const int chi[3], double *fine,
                const int flo[3], const int fhi[3], const int rlo[3],
                const int rhi[3], int ncomp, signed char *shifts,
                unsigned char *fallback) {
  init_coeffs();
  if (check_args(op, crse, clo, chi, fine, flo, fhi, rlo, rhi, ncomp))
    return -1;
  if (!box_ok(rlo, rhi) || ncomp == 0)
    return 0;
  if (per_group && ncomp > 16) /* impl.hxx:1707-1708 */
    return -1;
  cbox c;
  c.ptr = crse;
  c.nx = chi[0] - clo[0] + 1;
  c.ny = chi[1] - clo[1] + 1;
  c.np = (long)c.nx * c.ny * (chi[2] - clo[2] + 1);
  memcpy(c.lo, clo, sizeof c.lo);
  const long fnx = fhi[0] - flo[0] + 1, fny = fhi[1] - flo[1] + 1;
  const long fnp = fnx * fny * (fhi[2] - flo[2] + 1);
  const long rnx = rhi[0] - rlo[0] + 1, rny = rhi[1] - rlo[1] + 1;
  const long rnp = rnx * rny * (rhi[2] - rlo[2] + 1);
  opspec sp;
  make_spec(op, per_group, &sp);
  const int ngroups = per_group ? 1 : ncomp;
  for (int g = 0; g < ngroups; ++g) {
    const int c0 = per_group ? 0 : g, c1 = per_group ? ncomp : g + 1;
#pragma omp parallel for schedule(dynamic)
    for (int k = rlo[2]; k <= rhi[2]; ++k)
      for (int j = rlo[1]; j <= rhi[1]; ++j)
        for (int i = rlo[0]; i <= rhi[0]; ++i) {
          const int ifine[3] = {i, j, k};
          int ic[3], off[3], shift[3];
          for (int d = 0; d < 3; ++d) {
            ic[d] = floor2(ifine[d]);
            off[d] = ifine[d] - 2 * ic[d];
          }
          double vals[16];
          const int need =
              decide_point(op, per_group, &sp, &c, c0, c1, ic, off, shift, vals);
          const long ridx = (i - rlo[0]) + rnx * ((j - rlo[1]) + rny * (k - rlo[2]));
          const long fidx = (i - flo[0]) + fnx * ((j - flo[1]) + fny * (long)(k - flo[2]));
          for (int comp = c0; comp < c1; ++comp) {
            double res = vals[comp - c0];
            if (need)
              res = eval3d(sp.lin, (const int[3]){0, 0, 0}, off, &c, comp, ic);
            fine[comp * fnp + fidx] = res;
          }
          if (shifts)
            for (int d = 0; d < 3; ++d)
              shifts[3 * (g * rnp + ridx) + d] = (signed char)shift[d];
          if (fallback)
            fallback[g * rnp + ridx] = (unsigned char)need;
        }
  }
  return 0;
}

int cxo_prolong_adjoint(const cxo_op *op, int per_group, const double *crse,
                        const int clo[3], const int chi[3],
                        const double *fine_bar, const int flo[3],
                        const int fhi[3], const int rlo[3], const int rhi[3],
                        int ncomp, double *crse_bar) {
  init_coeffs();
  if (check_args(op, crse, clo, chi, fine_bar, flo, fhi, rlo, rhi, ncomp) ||
      !crse_bar)
    return -1;
  if (per_group && ncomp > 16)
    return -1;
  cbox c;
  c.ptr = crse;
  c.nx = chi[0] - clo[0] + 1;
  c.ny = chi[1] - clo[1] + 1;
  c.np = (long)c.nx * c.ny * (chi[2] - clo[2] + 1);
  memcpy(c.lo, clo, sizeof c.lo);
  memset(crse_bar, 0, sizeof(double) * c.np * ncomp);
  if (!box_ok(rlo, rhi) || ncomp == 0)
    return 0;
  const long fnx = fhi[0] - flo[0] + 1, fny = fhi[1] - flo[1] + 1;
  const long fnp = fnx * fny * (fhi[2] - flo[2] + 1);
  opspec sp;
  make_spec(op, per_group, &sp);
  const int ngroups = per_group ? 1 : ncomp;
  for (int g = 0; g < ngroups; ++g) {
    const int c0 = per_group ? 0 : g, c1 = per_group ? ncomp : g + 1;
    for (int k = rlo[2]; k <= rhi[2]; ++k)
      for (int j = rlo[1]; j <= rhi[1]; ++j)
        for (int i = rlo[0]; i <= rhi[0]; ++i) {
          const int ifine[3] = {i, j, k};
          int ic[3], off[3], shift[3];
          for (int d = 0; d < 3; ++d) {
            ic[d] = floor2(ifine[d]);
            off[d] = ifine[d] - 2 * ic[d];
          }
          double vals[16];
          const int need =
              decide_point(op, per_group, &sp, &c, c0, c1, ic, off, shift, vals);
          const long fidx = (i - flo[0]) + fnx * ((j - flo[1]) + fny * (long)(k - flo[2]));
          static const int zero3[3] = {0, 0, 0};
          for (int comp = c0; comp < c1; ++comp)
            eval3d_adjoint(need ? sp.lin : sp.s, need ? zero3 : shift, off, &c,
                           comp, ic, fine_bar[comp * fnp + fidx], crse_bar);
        }
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Restriction: AMReX average_down family as called by Restrict              */

static int restrict_check(const double *a, const int alo[3], const int ahi[3],
                          const double *b, const int blo[3], const int bhi[3],
                          const int rlo[3], const int rhi[3], int ncomp) {
  if (!a || !b || ncomp < 0 || !box_ok(alo, ahi) || !box_ok(blo, bhi))
    return -1;
  (void)rlo;
  (void)rhi;
  return 0;
}

int cxo_restrict(int indextype, const double *fine, const int flo[3],
                 const int fhi[3], double *crse, const int clo[3],
                 const int chi[3], const int rlo[3], const int rhi[3],
                 int ncomp) {
  if (indextype < 0 || indextype > 7 ||
      restrict_check(fine, flo, fhi, crse, clo, chi, rlo, rhi, ncomp))
    return -1;
  if (!box_ok(rlo, rhi))
    return 0;
  int cc[3], nch = 1;
  for (int d = 0; d < 3; ++d) {
    cc[d] = (indextype >> (2 - d)) & 1;
    nch *= cc[d] ? 2 : 1;
    if (rlo[d] < clo[d] || rhi[d] > chi[d] || 2 * rlo[d] < flo[d] ||
        2 * rhi[d] + cc[d] > fhi[d])
      return -1;
  }
  const double scale = 1.0 / nch;
  const long fnx = fhi[0] - flo[0] + 1, fny = fhi[1] - flo[1] + 1;
  const long fnp = fnx * fny * (fhi[2] - flo[2] + 1);
  const long cnx = chi[0] - clo[0] + 1, cny = chi[1] - clo[1] + 1;
  const long cnp = cnx * cny * (chi[2] - clo[2] + 1);
  for (int comp = 0; comp < ncomp; ++comp)
#pragma omp parallel for
    for (int k = rlo[2]; k <= rhi[2]; ++k)
      for (int j = rlo[1]; j <= rhi[1]; ++j)
        for (int i = rlo[0]; i <= rhi[0]; ++i) {
          const long cidx = comp * cnp + (i - clo[0]) +
                            cnx * ((j - clo[1]) + cny * (long)(k - clo[2]));
          const double *f = fine + comp * fnp;
#define FIDX(a, b, e)                                                         \
  ((a) - flo[0] + fnx * ((b) - flo[1] + fny * (long)((e) - flo[2])))
          if (indextype == 0) { /* average_down_nodal: injection */
            crse[cidx] = f[FIDX(2 * i, 2 * j, 2 * k)];
            continue;
          }
          double s = 0;
          for (int kr = 0; kr <= cc[2]; ++kr)
            for (int jr = 0; jr <= cc[1]; ++jr)
              for (int ir = 0; ir <= cc[0]; ++ir)
                s += f[FIDX(2 * i + ir, 2 * j + jr, 2 * k + kr)];
          crse[cidx] = s * scale;
#undef FIDX
        }
  return 0;
}

int cxo_restrict_adjoint(int indextype, const double *crse_bar,
                         const int clo[3], const int chi[3], double *fine_bar,
                         const int flo[3], const int fhi[3], const int rlo[3],
                         const int rhi[3], int ncomp) {
  if (indextype < 0 || indextype > 7 ||
      restrict_check(crse_bar, clo, chi, fine_bar, flo, fhi, rlo, rhi, ncomp))
    return -1;
  const long fnx = fhi[0] - flo[0] + 1, fny = fhi[1] - flo[1] + 1;
  const long fnp = fnx * fny * (fhi[2] - flo[2] + 1);
  const long cnx = chi[0] - clo[0] + 1, cny = chi[1] - clo[1] + 1;
  const long cnp = cnx * cny * (chi[2] - clo[2] + 1);
  memset(fine_bar, 0, sizeof(double) * fnp * ncomp);
  if (!box_ok(rlo, rhi))
    return 0;
  int cc[3], nch = 1;
  for (int d = 0; d < 3; ++d) {
    cc[d] = (indextype >> (2 - d)) & 1;
    nch *= cc[d] ? 2 : 1;
    if (rlo[d] < clo[d] || rhi[d] > chi[d] || 2 * rlo[d] < flo[d] ||
        2 * rhi[d] + cc[d] > fhi[d])
      return -1;
  }
  const double scale = 1.0 / nch;
  for (int comp = 0; comp < ncomp; ++comp)
    for (int k = rlo[2]; k <= rhi[2]; ++k)
      for (int j = rlo[1]; j <= rhi[1]; ++j)
        for (int i = rlo[0]; i <= rhi[0]; ++i) {
          const double g = crse_bar[comp * cnp + (i - clo[0]) +
                                    cnx * ((j - clo[1]) + cny * (long)(k - clo[2]))];
          for (int kr = 0; kr <= cc[2]; ++kr)
            for (int jr = 0; jr <= cc[1]; ++jr)
              for (int ir = 0; ir <= cc[0]; ++ir) {
                const int a = 2 * i + ir, b = 2 * j + jr, e = 2 * k + kr;
                fine_bar[comp * fnp + (a - flo[0]) +
                         fnx * ((b - flo[1]) + fny * (long)(e - flo[2]))] +=
                    indextype == 0 ? g : g * scale;
              }
        }
  return 0;
}

/* ---- Outer boundary conditions ------------------------------------------
 * Restates CarpetX's BoundaryCondition (boundaries.cxx:32-118,
 * boundaries_impl.hxx:28-444).  The reference visits the 26 regions of the
 * destination box outside the domain interior [imin, imax) (below, inside or
 * above it per direction) one template instantiation each; here each point
 * finds its region from its coordinates, which is the same partition. */
enum { BM_NONE, BM_DIRICHLET, BM_LINEXT, BM_NEUMANN, BM_ROBIN, BM_REFLECT, BM_BAD };

/* Condition of direction d on face f (0 lower, 1 upper), as chosen in
 * apply_on_face (boundaries_impl.hxx:71-108): periodic faces, and faces with
 * no or an inter-patch symmetry and no boundary condition, set nothing; a
 * reflection symmetry takes precedence over the group's boundary condition;
 * any other combination is an internal error there. */
static int bc_mode(const int sym[6], const int bc[6], int f, int d) {
  const int s = sym[3 * f + d], b = bc[3 * f + d];
  if (((s == 0 || s == 1) && b == 0) || s == 2)
    return BM_NONE;
  if (s == 3)
    return BM_REFLECT;
  switch (b) {
  case 2: return BM_DIRICHLET;
  case 3: return BM_LINEXT;
  case 4: return BM_NEUMANN;
  case 5: return BM_ROBIN;
  default: return BM_BAD;
  }
}

int cxo_boundary_box(const int symmetry[6], const int boundary[6],
                     const int domain_lo[3], const int domain_hi[3],
                     const double prob_lo[3], const double prob_hi[3],
                     const double dx[3], const int indextype[3], int ncomp,
                     const double *dirichlet, const double *robin,
                     const int *parity, double *data, const int lo[3],
                     const int hi[3]) {
  (void)prob_hi;
  if (ncomp < 1 || ncomp > 16 || !box_ok(lo, hi))
    return -1;
  int imin[3], imax[3], nx[3];
  double xmin[3];
  for (int d = 0; d < 3; ++d) {
    /* interior: the domain's cells, or its vertices (one more), as in the
     * constructor (boundaries.cxx:40-48); xmin as written there */
    imin[d] = domain_lo[d];
    imax[d] = domain_hi[d] + 1 + !indextype[d];
    xmin[d] = prob_lo[d] + 0.5 * indextype[d] - 1;
    nx[d] = hi[d] - lo[d] + 1;
  }
  const long np = (long)nx[0] * nx[1] * nx[2];
#define AT(c, q) data[(c) * np + ((q)[0] - lo[0]) + nx[0] * (((q)[1] - lo[1]) + nx[1] * (long)((q)[2] - lo[2]))]
  /* pass 0 checks every region; pass 1 writes.  Sources lie inside the
   * interior in every direction that has a condition, so no point read is
   * one that is written. */
  for (int pass = 0; pass < 2; ++pass)
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int p[3] = {i, j, k};
          int r[3], m[3], src[3], sp[3], delta[3] = {0, 0, 0};
          int any = 0, flags = 0;
          for (int d = 0; d < 3; ++d) {
            r[d] = p[d] < imin[d] ? -1 : p[d] >= imax[d] ? 1 : 0;
            m[d] = r[d] ? bc_mode(symmetry, boundary, r[d] > 0, d) : BM_NONE;
            if (m[d] == BM_BAD)
              return -1;
            any |= m[d] != BM_NONE;
            flags |= 1 << m[d];
          }
          if (!any)
            continue;
          for (int d = 0; d < 3; ++d) {
            const int edge = r[d] < 0 ? imin[d] : imax[d] - 1;
            src[d] = p[d];
            switch (m[d]) {
            case BM_LINEXT: src[d] = edge; delta[d] = -r[d]; break;
            case BM_NEUMANN:
            case BM_ROBIN: src[d] = edge; break;
            case BM_REFLECT:
              src[d] = (r[d] < 0 ? 2 * imin[d] - indextype[d]
                                 : 2 * (imax[d] - 1) + indextype[d]) - p[d];
              break;
            default: break;
            }
            sp[d] = src[d] + delta[d];
          }
          if (pass == 0) {
            for (int d = 0; d < 3; ++d) {
              if (m[d] == BM_NONE || m[d] == BM_DIRICHLET)
                continue;
              if (src[d] < imin[d] || src[d] >= imax[d] || src[d] < lo[d] || src[d] > hi[d] ||
                  sp[d] < imin[d] || sp[d] >= imax[d] || sp[d] < lo[d] || sp[d] > hi[d])
                return -1;
            }
            if (flags & (1 << BM_REFLECT))
              for (int c = 0; c < ncomp; ++c)
                for (int d = 0; d < 3; ++d)
                  if (m[d] == BM_REFLECT && parity[3 * c + d] != 1 && parity[3 * c + d] != -1)
                    return -1;
            continue;
          }
          for (int c = 0; c < ncomp; ++c) {
            double val;
            if (flags & (1 << BM_DIRICHLET)) {
              val = dirichlet[c];
            } else {
              val = AT(c, src);
              if (flags & (1 << BM_ROBIN))
                /* f(x') = finf + |x| / |x'| (f(x) - finf), once per Robin
                 * direction (boundaries_impl.hxx:391-408) */
                for (int d = 0; d < 3; ++d) {
                  if (m[d] != BM_ROBIN)
                    continue;
                  double sb = 0, si = 0;
                  for (int e = 0; e < 3; ++e) {
                    const double xb = xmin[e] + p[e] * dx[e];
                    const double xi = xmin[e] + src[e] * dx[e];
                    sb = sb + xb * xb;
                    si = si + xi * xi;
                  }
                  const double q = sqrt(si) / sqrt(sb);
                  val = robin[c] + q * (val - robin[c]);
                }
              if (flags & (1 << BM_LINEXT)) {
                /* slope from the two points src, src + delta; the distance
                 * ratio is an integer quotient of squared lengths, taken
                 * before the square root (boundaries_impl.hxx:409-414) */
                const double grad = val - AT(c, sp);
                int n2 = 0, d2 = 0;
                for (int d = 0; d < 3; ++d) {
                  n2 += (p[d] - src[d]) * (p[d] - src[d]);
                  d2 += delta[d] * delta[d];
                }
                val = val + sqrt((double)(n2 / d2)) * grad;
              }
              if (flags & (1 << BM_REFLECT)) {
                double par = 1;
                for (int d = 0; d < 3; ++d)
                  if (m[d] == BM_REFLECT)
                    par = par * parity[3 * c + d];
                val = val * par;
              }
            }
            AT(c, p) = val;
          }
        }
#undef AT
  return 0;
}
