// The C ABI (include/carpetx_b200.h): operator registry, argument
// validation, dispatch to the kernels, level plans.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/carpetx_b200.h"
#include "cx_internal.h"

using namespace cxb;

namespace {

thread_local std::string g_last_error;

int fail(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

int cuda_status(cudaError_t e, const char *what) {
  if (e == cudaSuccess)
    return CX_OK;
  return fail(CX_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Kinds of a family for one direction (the nine tables of
// CarpetX/src/prolongate_3d_rf2_impl_*.cxx).
int vc_poly_kind(int p) {
  return p == 1 ? K_VC_POLY1 : p == 3 ? K_VC_POLY3 : p == 5 ? K_VC_POLY5 : p == 7 ? K_VC_POLY7 : -1;
}
int cc_poly_kind(int p) {
  return p == 1 ? K_CC_POLY1 : p == 3 ? K_CC_POLY3 : p == 5 ? K_CC_POLY5 : p == 7 ? K_CC_POLY7 : -1;
}
int cc_cons_kind(int p) { return p >= 0 && p <= 7 ? K_CC_CONS0 + p : -1; }

bool lookup_kinds(const char *type, int o, int *vc, int *cc, int *fb) {
  const std::string t(type);
  *fb = 0;
  auto in = [o](std::initializer_list<int> l) { return std::find(l.begin(), l.end(), o) != l.end(); };
  if (t == "interpolate" && in({1, 3, 5, 7})) { // impl_poly.cxx:7-121
    *vc = vc_poly_kind(o);
    *cc = cc_poly_kind(o);
  } else if (t == "conservative" && in({0, 1})) { // impl_cons.cxx:7-65
    *vc = o == 0 ? K_VC_CONS0 : K_VC_CONS1;
    *cc = o == 0 ? K_CC_CONS0 : K_CC_CONS2;
  } else if (t == "ddf" && in({1, 3, 5, 7})) { // impl_ddf.cxx:7-121
    *vc = vc_poly_kind(o);
    *cc = cc_cons_kind(o - 1);
  } else if (t == "eno" && in({3, 5})) { // impl_eno.cxx:7-65
    *vc = vc_poly_kind(o);
    *cc = K_CC_ENO2;
  } else if (t == "minmod" && in({1, 3, 5})) { // impl_minmod.cxx:7-93
    *vc = vc_poly_kind(o);
    *cc = K_CC_MINMOD1;
  } else if ((t == "hermite" && in({1, 3, 5})) || (t == "natural" && in({1, 3, 5, 7}))) {
    // impl_hermite.cxx:7-96 (VC HERMITE = VC POLY arithmetic), impl_natural.cxx:7-121
    *vc = vc_poly_kind(o);
    *cc = cc_cons_kind(o);
  } else if (t == "poly-cons3lfb" && in({1, 3, 5})) { // impl_poly_cons3lfb.cxx:9-119
    *vc = vc_poly_kind(o);
    *cc = cc_cons_kind(std::min(o, 3));
    *fb = 1;
  } else if (t == "poly-eno3lfb" && in({1, 3, 5})) { // impl_poly_eno3lfb.cxx:9-119
    *vc = vc_poly_kind(o);
    *cc = o == 1 ? K_CC_CONS0 : K_CC_ENO2;
    *fb = 1;
  } else {
    return false;
  }
  return true;
}

bool valid_op(cx_op_t op) {
  for (int d = 0; d < 3; ++d)
    if (op_kind(op, d) < 0 || op_kind(op, d) >= K_COUNT)
      return false;
  return (op >> 16) == 0;
}

int floor2(int i) { return i >= 0 ? i / 2 : -((-i + 1) / 2); }

bool box_ok(const int lo[3], const int hi[3]) {
  return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2];
}

// Builds and validates the kernel descriptor of one interp() call.
// Returns CX_OK, or an error; *empty is set when there is nothing to do.
int make_box(cx_op_t op, const double *crse, const int clo[3], const int chi[3], double *fine,
             const int flo[3], const int fhi[3], const int rlo[3], const int rhi[3], int ncomp,
             int per_group, BoxDesc *b, bool *empty) {
  *empty = false;
  if (!valid_op(op))
    return fail(CX_EUNSUPPORTED, "invalid operator handle %d", (int)op);
  if (!clo || !chi || !flo || !fhi || !rlo || !rhi)
    return fail(CX_EINVAL, "null box pointer");
  if (ncomp < 0)
    return fail(CX_EINVAL, "ncomp = %d < 0", ncomp);
  if (per_group && ncomp > 16) // impl.hxx:1707-1708
    return fail(CX_EINVAL, "per-group prolongation supports at most 16 components, got %d", ncomp);
  if (!box_ok(rlo, rhi) || ncomp == 0) {
    *empty = true;
    return CX_OK;
  }
  if (!crse || !fine)
    return fail(CX_EINVAL, "null data pointer");
  if (!box_ok(flo, fhi) || !box_ok(clo, chi))
    return fail(CX_EINVAL, "empty coarse or fine FAB box");
  for (int d = 0; d < 3; ++d)
    if (rlo[d] < flo[d] || rhi[d] > fhi[d]) // impl.hxx:1300-1302
      return fail(CX_EINVAL, "fine region [%d,%d] not inside the fine box [%d,%d] in direction %d",
                  rlo[d], rhi[d], flo[d], fhi[d], d);
  std::memset(b, 0, sizeof *b);
  b->crse = crse;
  b->fine = fine;
  b->op = op;
  b->ncomp = ncomp;
  for (int d = 0; d < 3; ++d) {
    const int k = op_kind(op, d);
    b->kind[d] = k;
    b->clo[d] = clo[d];
    b->flo[d] = flo[d];
    b->rlo[d] = rlo[d];
    b->rhi[d] = rhi[d];
    // coarse points read: extreme fine points of each parity
    int nlo = INT32_MAX, nhi = INT32_MIN;
    for (int f = rlo[d]; f <= rhi[d] && f <= rlo[d] + 1; ++f) {
      int a, c;
      read_range(k, f & 1, &a, &c);
      nlo = std::min(nlo, floor2(f) + a);
    }
    for (int f = rhi[d]; f >= rlo[d] && f >= rhi[d] - 1; --f) {
      int a, c;
      read_range(k, f & 1, &a, &c);
      nhi = std::max(nhi, floor2(f) + c);
    }
    if (nlo < clo[d] || nhi > chi[d])
      return fail(CX_EINVAL,
                  "coarse box [%d,%d] does not contain the coarse points [%d,%d] the stencil "
                  "reads in direction %d",
                  clo[d], chi[d], nlo, nhi, d);
    b->nlo[d] = nlo;
    b->nhi[d] = nhi;
  }
  b->cnx = chi[0] - clo[0] + 1;
  b->cny = chi[1] - clo[1] + 1;
  b->cnp = (int64_t)b->cnx * b->cny * (chi[2] - clo[2] + 1);
  b->fnx = fhi[0] - flo[0] + 1;
  b->fny = fhi[1] - flo[1] + 1;
  b->fnp = (int64_t)b->fnx * b->fny * (fhi[2] - flo[2] + 1);
  stream_tiling(*b, 0);
  (void)per_group;
  return CX_OK;
}

// The separable operators run on the streaming kernel (pair instantiation);
// everything else on the pointwise kernel.
bool use_stream(cx_op_t op, int per_group) {
  return op_separable(op, per_group) &&
         stream_pair_of(op_kind(op, 0), op_kind(op, 1), op_kind(op, 2)) >= 0;
}

int check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(CX_ENODEVICE, "no CUDA device");
  }
  return CX_OK;
}

int64_t box_points(const int lo[3], const int hi[3]) {
  return (int64_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
}

} // namespace

struct cx_level_plan {
  int per_group = 0;
  std::vector<BoxDesc> boxes;
  std::vector<int> point_boxes; // boxes handled by the pointwise kernel
  BoxDesc *d_boxes = nullptr;
  TileRef *d_tiles = nullptr;
  int *d_counters = nullptr; // one item counter per group
  int nsep_tiles = 0;
  // items of kernel group g: [group_off[g], group_off[g + 1]) of d_tiles
  int group_off[kStrGroups + 1] = {};
  int group_grid[kStrGroups] = {};
  int group_sched[kStrGroups] = {}; // streaming groups: schedule picked at creation
  int64_t nfine = 0, bytes = 0;
  // adjoint plan: execute computes crse = P^T fine for every box; coarse
  // boxes whose region is empty are zeroed (pointer, bytes)
  bool adjoint = false;
  std::vector<std::pair<double *, size_t>> zero_boxes;
  // adjoint plan: scratch of the limited operators' decision passes (the
  // point boxes run one after the other on the stream, so one buffer of the
  // largest box's size serves them all)
  void *d_scratch = nullptr;
};

extern "C" {

const char *cx_status_string(int status) {
  switch (status) {
  case CX_OK: return "ok";
  case CX_EINVAL: return "invalid argument";
  case CX_EUNSUPPORTED: return "unsupported operator";
  case CX_ECUDA: return "CUDA error";
  case CX_ETIMEOUT: return "device wait timed out";
  case CX_ENOMEM: return "out of memory";
  case CX_ENODEVICE: return "no CUDA device";
  default: return "unknown status";
  }
}

const char *cx_last_error(void) { return g_last_error.c_str(); }

int cx_prolong_lookup(const char *type, int order, int indextype, cx_op_t *out) {
  if (!type || !out)
    return fail(CX_EINVAL, "null argument");
  if (indextype < 0 || indextype > 7)
    return fail(CX_EUNSUPPORTED, "indextype %d out of range 0..7", indextype);
  int vc, cc, fb;
  if (!lookup_kinds(type, order, &vc, &cc, &fb))
    return fail(CX_EUNSUPPORTED, "Unsupported prolongation order %d for prolongation type %s",
                order, type);
  int k[3];
  for (int d = 0; d < 3; ++d)
    k[d] = ((indextype >> (2 - d)) & 1) ? cc : vc;
  *out = op_encode(k[0], k[1], k[2], fb);
  return CX_OK;
}

int cx_prolong_required_ghosts(cx_op_t op, int ghosts[3]) {
  if (!valid_op(op) || !ghosts)
    return fail(CX_EINVAL, "invalid argument");
  for (int d = 0; d < 3; ++d)
    ghosts[d] = kind_info(op_kind(op, d)).ghosts;
  return CX_OK;
}

int cx_prolong_coarse_box(cx_op_t op, const int fine_lo[3], const int fine_hi[3], int crse_lo[3],
                          int crse_hi[3]) {
  int g[3];
  if (!fine_lo || !fine_hi || !crse_lo || !crse_hi)
    return fail(CX_EINVAL, "null argument");
  if (int e = cx_prolong_required_ghosts(op, g))
    return e;
  for (int d = 0; d < 3; ++d) {
    crse_lo[d] = floor2(fine_lo[d]) - g[d];
    crse_hi[d] = floor2(fine_hi[d]) + g[d];
  }
  return CX_OK;
}

int cx_prolong_box_diag(cx_op_t op, const double *crse, const int crse_lo[3], const int crse_hi[3],
                        double *fine, const int fine_lo[3], const int fine_hi[3],
                        const int reg_lo[3], const int reg_hi[3], int ncomp, int per_group,
                        signed char *shifts, unsigned char *fallback, cx_stream_t stream) {
  BoxDesc b;
  bool empty;
  if (int e = make_box(op, crse, crse_lo, crse_hi, fine, fine_lo, fine_hi, reg_lo, reg_hi, ncomp,
                       per_group, &b, &empty))
    return e;
  if (empty)
    return CX_OK;
  if (int e = check_device())
    return e;
  cudaStream_t s = (cudaStream_t)stream;
  // one box per launch: spread it over the GPU (z chunks sized by the grid of
  // the 256-thread variant, whichever CTA size the box then takes)
  if (use_stream(op, per_group))
    {
      const int g = stream_group_of(b.kind[0], b.kind[1], b.kind[2]);
      stream_tiling(b, stream_level_grid(g, stream_sched(g)));
    }
  if (use_stream(op, per_group) && !shifts && !fallback)
    return cuda_status(launch_stream_box(b, s), "prolongation launch");
  if (use_stream(op, per_group)) {
    // diagnostics requested for an operator without shifts or fallback:
    // values from the separable kernel, diagnostics all zero
    const int64_t nreg = box_points(reg_lo, reg_hi) * (per_group ? 1 : ncomp);
    if (shifts)
      if (int e = cuda_status(cudaMemsetAsync(shifts, 0, 3 * nreg, s), "memset"))
        return e;
    if (fallback)
      if (int e = cuda_status(cudaMemsetAsync(fallback, 0, nreg, s), "memset"))
        return e;
    return cuda_status(launch_stream_box(b, s), "prolongation launch");
  }
  return cuda_status(launch_point_box(b, per_group, shifts, fallback, s), "prolongation launch");
}

int cx_prolong_box(cx_op_t op, const double *crse, const int crse_lo[3], const int crse_hi[3],
                   double *fine, const int fine_lo[3], const int fine_hi[3], const int reg_lo[3],
                   const int reg_hi[3], int ncomp, int per_group, cx_stream_t stream) {
  return cx_prolong_box_diag(op, crse, crse_lo, crse_hi, fine, fine_lo, fine_hi, reg_lo, reg_hi,
                             ncomp, per_group, nullptr, nullptr, stream);
}

int cx_level_plan_create(const cx_box_t *boxes, int nboxes, int per_group, cx_level_plan_t *out) {
  if (!out || nboxes < 0 || (nboxes > 0 && !boxes))
    return fail(CX_EINVAL, "invalid argument");
  *out = nullptr;
  if (int e = check_device())
    return e;
  cx_level_plan *p = new cx_level_plan;
  p->per_group = per_group;
  std::vector<int> sep_ids;
  for (int i = 0; i < nboxes; ++i) {
    const cx_box_t &x = boxes[i];
    BoxDesc b;
    bool empty;
    if (int e = make_box(x.op, x.crse, x.crse_lo, x.crse_hi, x.fine, x.fine_lo, x.fine_hi,
                         x.reg_lo, x.reg_hi, x.ncomp, per_group, &b, &empty)) {
      delete p;
      return fail(e, "box %d: %s", i, g_last_error.c_str());
    }
    if (empty)
      continue;
    if (b.ntile[0] > INT16_MAX || b.ntile[1] > INT16_MAX || b.ntile[2] > INT16_MAX ||
        x.ncomp > INT16_MAX) {
      delete p;
      return fail(CX_EINVAL, "box %d: too many tiles or components for a level plan", i);
    }
    int cl[3], ch[3];
    cx_prolong_coarse_box(x.op, x.reg_lo, x.reg_hi, cl, ch);
    p->nfine += box_points(x.reg_lo, x.reg_hi) * x.ncomp;
    p->bytes += 8 * (box_points(cl, ch) + box_points(x.reg_lo, x.reg_hi)) * x.ncomp;
    const int id = (int)p->boxes.size();
    p->boxes.push_back(b);
    if (use_stream(x.op, per_group))
      sep_ids.push_back(id);
    else
      p->point_boxes.push_back(id);
  }
  // work items of the separable boxes: (box, x tile, y tile, z chunk,
  // component), grouped by kernel instantiation and sorted by streamed
  // planes, largest first; each kernel deals them round-robin to its
  // persistent CTAs
  std::vector<std::pair<int, TileRef>> keyed;
  for (int id : sep_ids) {
    const BoxDesc &b = p->boxes[id];
    const int L = sep_rhi(b.kind[2]) - sep_rlo(b.kind[2]);
    for (int c = 0; c < b.ncomp; ++c)
      for (int tz = 0; tz < b.ntile[2]; ++tz) {
        const int z0 = b.tbase[2] + tz * b.zchunk;
        const int z1 = std::min(z0 + b.zchunk - 1, b.rhi[2]);
        const int planes = (z1 >> 1) - (z0 >> 1) + 1 + L;
        for (int tx = 0; tx < b.ntile[0]; ++tx) {
          const int xb = b.tbase[0] + tx * b.xcw;
          const int W = std::min(b.xcw, b.rhi[0] - xb + 1);
          const int nub = (b.npr * W + b.upi - 1) / b.upi; // non-empty unit blocks
          for (int ub = 0; ub < nub; ++ub)
            keyed.push_back({planes, TileRef{id, (int16_t)tx, (int16_t)ub, (int16_t)tz, (int16_t)c}});
        }
      }
  }
  // by z-window group (one kernel each), then by cost, largest first
  auto group_of = [&](const TileRef &t) {
    const BoxDesc &b = p->boxes[t.box];
    return stream_group_of(b.kind[0], b.kind[1], b.kind[2]) + (b.scta ? kStrKinds : 0);
  };
  std::stable_sort(keyed.begin(), keyed.end(),
                   [&](const std::pair<int, TileRef> &a, const std::pair<int, TileRef> &b) {
                     const int ga = group_of(a.second), gb = group_of(b.second);
                     return ga != gb ? ga < gb : a.first > b.first;
                   });
  for (auto &k : keyed)
    p->group_off[group_of(k.second) + 1]++;
  for (int g = 0; g < kStrGroups; ++g)
    p->group_off[g + 1] += p->group_off[g];
  std::vector<TileRef> tiles;
  tiles.reserve(keyed.size());
  for (auto &k : keyed)
    tiles.push_back(k.second);
  if (tiles.size() > (size_t)INT32_MAX) {
    delete p;
    return fail(CX_EINVAL, "too many tiles");
  }
  p->nsep_tiles = (int)tiles.size();
  cudaError_t e = cudaSuccess;
  if (!p->boxes.empty())
    e = cudaMalloc(&p->d_boxes, sizeof(BoxDesc) * p->boxes.size());
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMalloc(&p->d_tiles, sizeof(TileRef) * tiles.size());
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMalloc(&p->d_counters, sizeof(int) * kStrGroups);
  if (e == cudaSuccess && !p->boxes.empty())
    e = cudaMemcpy(p->d_boxes, p->boxes.data(), sizeof(BoxDesc) * p->boxes.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMemcpy(p->d_tiles, tiles.data(), sizeof(TileRef) * tiles.size(),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cx_level_plan_destroy(p);
    return fail(e == cudaErrorMemoryAllocation ? CX_ENOMEM : CX_ECUDA, "level plan: %s",
                cudaGetErrorString(e));
  }
  for (int g = 0; g < kStrGroups; ++g) {
    p->group_sched[g] = stream_sched(g);
    p->group_grid[g] =
        p->group_off[g + 1] > p->group_off[g] ? stream_level_grid(g, p->group_sched[g]) : 0;
  }
  *out = p;
  return CX_OK;
}

int cx_level_plan_create_adjoint(const cx_box_t *boxes, int nboxes, int per_group,
                                 cx_level_plan_t *out) {
  return cx_level_plan_create_adjoint_at(boxes, nullptr, nboxes, per_group, out);
}

int cx_level_plan_create_adjoint_at(const cx_box_t *boxes, const double *const *crse_at,
                                    int nboxes, int per_group, cx_level_plan_t *out) {
  if (!out || nboxes < 0 || (nboxes > 0 && !boxes))
    return fail(CX_EINVAL, "invalid argument");
  *out = nullptr;
  if (int e = check_device())
    return e;
  cx_level_plan *p = new cx_level_plan;
  p->per_group = per_group;
  p->adjoint = true;
  std::vector<int> ids;
  size_t scratch = 0;
  for (int i = 0; i < nboxes; ++i) {
    const cx_box_t &x = boxes[i];
    BoxDesc b;
    bool empty;
    if (!x.crse && x.ncomp > 0) {
      delete p;
      return fail(CX_EINVAL, "box %d: null crse (the adjoint's output)", i);
    }
    if (int e = make_box(x.op, x.crse, x.crse_lo, x.crse_hi, x.fine, x.fine_lo, x.fine_hi,
                         x.reg_lo, x.reg_hi, x.ncomp, per_group, &b, &empty)) {
      delete p;
      return fail(e, "box %d: %s", i, g_last_error.c_str());
    }
    if (empty) {
      if (x.ncomp > 0 && box_ok(x.crse_lo, x.crse_hi))
        p->zero_boxes.push_back({const_cast<double *>(x.crse),
                                 sizeof(double) * box_points(x.crse_lo, x.crse_hi) * x.ncomp});
      continue;
    }
    b.cbar = const_cast<double *>(x.crse);
    if (!op_separable(x.op, per_group) || adjoint_pair_of(b) < 0) {
      // limited operators (ENO, minmod, active linear fallback): a decision
      // pass and a gather per box, after the streaming groups, linearised at
      // the box's coarse data crse_at[i] (crse is the output)
      if (!crse_at || !crse_at[i]) {
        cx_level_plan_destroy(p);
        return fail(CX_EINVAL, "box %d: the adjoint of a limited operator (ENO, minmod, linear "
                               "fallback) needs the coarse data it is linearised at "
                               "(cx_level_plan_create_adjoint_at)", i);
      }
      b.crse = crse_at[i];
      int cl[3], ch[3];
      cx_prolong_coarse_box(x.op, x.reg_lo, x.reg_hi, cl, ch);
      p->nfine += box_points(x.reg_lo, x.reg_hi) * x.ncomp;
      p->bytes += 8 * (box_points(cl, ch) + box_points(x.reg_lo, x.reg_hi)) * x.ncomp;
      scratch = std::max(scratch, point_adjoint_scratch_bytes(b, per_group));
      p->point_boxes.push_back((int)p->boxes.size());
      p->boxes.push_back(b);
      continue;
    }
    adjoint_tiling(b, 0);
    if (b.ant[0] > INT16_MAX || b.ant[1] > INT16_MAX || b.ant[2] > INT16_MAX ||
        x.ncomp > INT16_MAX) {
      delete p;
      return fail(CX_EINVAL, "box %d: too many tiles or components for a level plan", i);
    }
    int cl[3], ch[3];
    cx_prolong_coarse_box(x.op, x.reg_lo, x.reg_hi, cl, ch);
    p->nfine += box_points(x.reg_lo, x.reg_hi) * x.ncomp;
    p->bytes += 8 * (box_points(cl, ch) + box_points(x.reg_lo, x.reg_hi)) * x.ncomp;
    ids.push_back((int)p->boxes.size());
    p->boxes.push_back(b);
  }
  // work items (box, x tile, y tile, z chunk, component) grouped by kernel
  // instantiation and sorted by cost (fine planes x tile columns), largest
  // first; equal costs keep the tiles of a box together, so neighbouring
  // tiles stream at the same time and share their footprint halo in the L2
  std::vector<std::pair<int64_t, TileRef>> keyed;
  for (int id : ids) {
    const BoxDesc &b = p->boxes[id];
    const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
    const int L = sep_rhi(b.kind[2]) - sep_rlo(b.kind[2]);
    for (int c = 0; c < b.ncomp; ++c)
      for (int tz = 0; tz < b.ant[2]; ++tz) {
        const int nz = std::min(b.at[2], cnz - tz * b.at[2]);
        for (int ty = 0; ty < b.ant[1]; ++ty)
          for (int tx = 0; tx < b.ant[0]; ++tx) {
            const int w = std::min(b.at[0], b.cnx - tx * b.at[0]);
            const int h = std::min(b.at[1], b.cny - ty * b.at[1]);
            keyed.push_back({(int64_t)(2 * (nz + L)) * w * h,
                             TileRef{id, (int16_t)tx, (int16_t)ty, (int16_t)tz, (int16_t)c}});
          }
      }
  }
  auto group_of = [&](const TileRef &t) { return adjoint_group_of(p->boxes[t.box]); };
  std::stable_sort(keyed.begin(), keyed.end(),
                   [&](const std::pair<int64_t, TileRef> &a, const std::pair<int64_t, TileRef> &b) {
                     const int ga = group_of(a.second), gb = group_of(b.second);
                     return ga != gb ? ga < gb : a.first > b.first;
                   });
  for (auto &k : keyed)
    p->group_off[group_of(k.second) + 1]++;
  for (int g = 0; g < kStrGroups; ++g)
    p->group_off[g + 1] += p->group_off[g];
  std::vector<TileRef> tiles;
  tiles.reserve(keyed.size());
  for (auto &k : keyed)
    tiles.push_back(k.second);
  if (tiles.size() > (size_t)INT32_MAX) {
    delete p;
    return fail(CX_EINVAL, "too many tiles");
  }
  p->nsep_tiles = (int)tiles.size();
  cudaError_t e = cudaSuccess;
  if (!p->boxes.empty())
    e = cudaMalloc(&p->d_boxes, sizeof(BoxDesc) * p->boxes.size());
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMalloc(&p->d_tiles, sizeof(TileRef) * tiles.size());
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMalloc(&p->d_counters, sizeof(int) * kStrGroups);
  if (e == cudaSuccess && !p->boxes.empty())
    e = cudaMemcpy(p->d_boxes, p->boxes.data(), sizeof(BoxDesc) * p->boxes.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !tiles.empty())
    e = cudaMemcpy(p->d_tiles, tiles.data(), sizeof(TileRef) * tiles.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && scratch)
    e = cudaMalloc(&p->d_scratch, scratch);
  if (e != cudaSuccess) {
    cx_level_plan_destroy(p);
    return fail(e == cudaErrorMemoryAllocation ? CX_ENOMEM : CX_ECUDA, "level plan: %s",
                cudaGetErrorString(e));
  }
  for (int g = 0; g < kStrGroups; ++g)
    p->group_grid[g] = p->group_off[g + 1] > p->group_off[g] ? adjoint_level_grid(g) : 0;
  *out = p;
  return CX_OK;
}

int cx_level_plan_execute(cx_level_plan_t p, cx_stream_t stream) {
  if (!p)
    return fail(CX_EINVAL, "null plan");
  cudaStream_t s = (cudaStream_t)stream;
  if (p->adjoint) {
    for (auto &z : p->zero_boxes)
      if (int e = cuda_status(cudaMemsetAsync(z.first, 0, z.second, s), "memset"))
        return e;
    if (p->d_counters)
      if (int e = cuda_status(cudaMemsetAsync(p->d_counters, 0, sizeof(int) * kStrGroups, s),
                              "memset"))
        return e;
    bool after_level = false;
    for (int g = 0; g < kStrGroups; ++g) {
      const int n = p->group_off[g + 1] - p->group_off[g];
      if (n > 0) {
        if (int e = cuda_status(launch_adjoint_level(g, p->d_boxes, p->d_tiles + p->group_off[g],
                                                     n, p->group_grid[g], p->d_counters + g, s,
                                                     after_level),
                                "adjoint level launch"))
          return e;
        after_level = true;
      }
    }
    // the limited operators' boxes: a decision pass and a gather each
    for (int id : p->point_boxes)
      if (int e = cuda_status(launch_point_adjoint_box_scratch(p->boxes[id], p->per_group,
                                                               p->boxes[id].cbar, p->d_scratch, s),
                              "adjoint launch (limited operators)"))
        return e;
    return CX_OK;
  }
  if (p->d_counters)
    if (int e = cuda_status(cudaMemsetAsync(p->d_counters, 0, sizeof(int) * kStrGroups, s),
                            "memset"))
      return e;
  // the 128-thread groups first: their few items then run beside the
  // 256-thread groups instead of after them
  bool after_level = false;
  for (int i = 0; i < kStrGroups; ++i) {
    const int g = (i + kStrKinds) % kStrGroups;
    const int n = p->group_off[g + 1] - p->group_off[g];
    if (n > 0) {
      if (int e = cuda_status(launch_stream_level(g, p->group_sched[g], p->d_boxes,
                                                  p->d_tiles + p->group_off[g], n,
                                                  p->group_grid[g], p->d_counters + g, s,
                                                  after_level),
                              "level launch"))
        return e;
      after_level = true;
    }
  }
  for (int id : p->point_boxes) {
    if (int e = cuda_status(
            launch_point_box(p->boxes[id], p->per_group, nullptr, nullptr, s, after_level),
            "level launch (limited operators)"))
      return e;
    after_level = true;
  }
  return CX_OK;
}

int cx_check_device(void) {
  if (int e = check_device())
    return e;
  if (int e = cuda_status(cudaDeviceSynchronize(), "device work"))
    return e;
  const int ta = adjoint_take_timeout(), ts = stream_take_timeout();
  const int t = ta < 0 || ts < 0 ? -1 : ta | ts;
  if (t < 0)
    return fail(CX_ECUDA, "reading the device wait flag failed");
  if (t > 0)
    return fail(CX_ETIMEOUT, "a bounded device wait gave up (its results are not valid)");
  return CX_OK;
}

int cx_debug_stream_kind(cx_op_t op) {
  if (!valid_op(op))
    return fail(CX_EINVAL, "invalid operator handle %d", (int)op);
  if (!use_stream(op, 0))
    return -1;
  return stream_group_of(op_kind(op, 0), op_kind(op, 1), op_kind(op, 2));
}

int cx_debug_set_stream_schedule(int kind, int sched, int maxz) {
  if (stream_set_schedule(kind, sched, maxz) != 0)
    return fail(CX_EINVAL, "kind %d, schedule %d or z cap %d out of range", kind, sched, maxz);
  return CX_OK;
}

int cx_debug_set_wait_limit(long long cycles) {
  if (int e = check_device())
    return e;
  if (adjoint_set_wait_limit(cycles) != 0 || stream_set_wait_limit(cycles) != 0) {
    cudaGetLastError();
    return fail(CX_ECUDA, "setting the device wait limit failed");
  }
  return CX_OK;
}

int cx_level_plan_stats(cx_level_plan_t p, int64_t *ntiles, int64_t *nfine, int64_t *bytes) {
  if (!p)
    return fail(CX_EINVAL, "null plan");
  if (ntiles)
    *ntiles = p->nsep_tiles;
  if (nfine)
    *nfine = p->nfine;
  if (bytes)
    *bytes = p->bytes;
  return CX_OK;
}

int cx_level_plan_launches(cx_level_plan_t p, int *nlaunches) {
  if (!p || !nlaunches)
    return fail(CX_EINVAL, "invalid argument");
  int n = 0;
  for (int g = 0; g < kStrGroups; ++g)
    n += p->group_off[g + 1] > p->group_off[g];
  if (!p->adjoint)
    n += (int)p->point_boxes.size();
  else
    for (int id : p->point_boxes) // decision pass (if any) and gather
      n += 1 + (point_adjoint_scratch_bytes(p->boxes[id], p->per_group) > 0);
  *nlaunches = n;
  return CX_OK;
}

int cx_level_plan_destroy(cx_level_plan_t p) {
  if (!p)
    return CX_OK;
  cudaFree(p->d_boxes);
  cudaFree(p->d_tiles);
  cudaFree(p->d_counters);
  cudaFree(p->d_scratch);
  delete p;
  return CX_OK;
}

} // extern "C"

namespace {
// The checks of cx_restrict_box; *empty: nothing to do.
int check_restrict(int indextype, const double *fine, const int fine_lo[3], const int fine_hi[3],
                   const double *crse, const int crse_lo[3], const int crse_hi[3],
                   const int reg_lo[3], const int reg_hi[3], int ncomp, bool *empty) {
  *empty = true;
  if (indextype < 0 || indextype > 7)
    return fail(CX_EUNSUPPORTED, "indextype %d out of range 0..7", indextype);
  if (!fine_lo || !fine_hi || !crse_lo || !crse_hi || !reg_lo || !reg_hi || ncomp < 0)
    return fail(CX_EINVAL, "invalid argument");
  if (!box_ok(reg_lo, reg_hi) || ncomp == 0)
    return CX_OK;
  if (!fine || !crse || !box_ok(fine_lo, fine_hi) || !box_ok(crse_lo, crse_hi))
    return fail(CX_EINVAL, "invalid FAB");
  for (int d = 0; d < 3; ++d) {
    const int cc = (indextype >> (2 - d)) & 1;
    if (reg_lo[d] < crse_lo[d] || reg_hi[d] > crse_hi[d])
      return fail(CX_EINVAL, "coarse region not inside the coarse box in direction %d", d);
    if (2 * reg_lo[d] < fine_lo[d] || 2 * reg_hi[d] + cc > fine_hi[d])
      return fail(CX_EINVAL, "fine box does not contain the children of the region in direction %d",
                  d);
  }
  *empty = false;
  return CX_OK;
}
} // namespace

struct cx_restrict_plan {
  void *d_items[8] = {};
  int *d_first[8] = {}; // per chunk of 256 points: its first item
  int nitems[8] = {};
  int64_t npts[8] = {};
  int64_t ncoarse = 0, bytes = 0;
  int nlaunch = 0;
};

extern "C" {

int cx_restrict_box(int indextype, const double *fine, const int fine_lo[3], const int fine_hi[3],
                    double *crse, const int crse_lo[3], const int crse_hi[3], const int reg_lo[3],
                    const int reg_hi[3], int ncomp, cx_stream_t stream) {
  bool empty;
  if (int e = check_restrict(indextype, fine, fine_lo, fine_hi, crse, crse_lo, crse_hi, reg_lo,
                             reg_hi, ncomp, &empty))
    return e;
  if (empty)
    return CX_OK;
  if (int e = check_device())
    return e;
  return cuda_status(launch_restrict_box(indextype, fine, fine_lo, fine_hi, crse, crse_lo, crse_hi,
                                         reg_lo, reg_hi, ncomp, (cudaStream_t)stream),
                     "restriction launch");
}

int cx_restrict_plan_create(const cx_restrict_box_t *boxes, int nboxes, cx_restrict_plan_t *out) {
  if (!out || nboxes < 0 || (nboxes > 0 && !boxes))
    return fail(CX_EINVAL, "invalid argument");
  *out = nullptr;
  std::vector<int> ids[8];
  for (int i = 0; i < nboxes; ++i) {
    const cx_restrict_box_t &b = boxes[i];
    bool empty;
    if (int e = check_restrict(b.indextype, b.fine, b.fine_lo, b.fine_hi, b.crse, b.crse_lo,
                               b.crse_hi, b.reg_lo, b.reg_hi, b.ncomp, &empty))
      return fail(e, "box %d: %s", i, g_last_error.c_str());
    if (!empty)
      ids[b.indextype].push_back(i);
  }
  if (int e = check_device())
    return e;
  cx_restrict_plan *p = new cx_restrict_plan;
  const int64_t isz = restrict_item_bytes();
  for (int it = 0; it < 8; ++it) {
    if (ids[it].empty())
      continue;
    std::vector<char> buf(ids[it].size() * isz);
    std::vector<int64_t> starts(ids[it].size());
    int64_t start = 0;
    const int nch = (1 + ((it >> 2) & 1)) * (1 + ((it >> 1) & 1)) * (1 + (it & 1));
    for (size_t n = 0; n < ids[it].size(); ++n) {
      const cx_restrict_box_t &b = boxes[ids[it][n]];
      const int64_t pts = restrict_fill_item(buf.data(), (int)n, b.fine, b.fine_lo, b.fine_hi,
                                             b.crse, b.crse_lo, b.crse_hi, b.reg_lo, b.reg_hi,
                                             b.ncomp, start);
      if (pts > INT32_MAX) {
        cx_restrict_plan_destroy(p);
        return fail(CX_EINVAL, "box %d: more than 2^31 coarse values", ids[it][n]);
      }
      starts[n] = start;
      start += pts;
      p->bytes += 8 * pts * (nch + 1);
    }
    std::vector<int> first((start + 255) / 256);
    size_t a = 0;
    for (size_t c = 0; c < first.size(); ++c) {
      while (a + 1 < starts.size() && starts[a + 1] <= (int64_t)c * 256)
        ++a;
      first[c] = (int)a;
    }
    p->ncoarse += start;
    p->npts[it] = start;
    p->nitems[it] = (int)ids[it].size();
    ++p->nlaunch;
    cudaError_t e = cudaMalloc(&p->d_items[it], buf.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_items[it], buf.data(), buf.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMalloc(&p->d_first[it], first.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_first[it], first.data(), first.size() * sizeof(int),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cx_restrict_plan_destroy(p);
      return cuda_status(e, "restriction plan upload");
    }
  }
  *out = p;
  return CX_OK;
}

int cx_restrict_groups_plan_create(const cx_restrict_group_t *groups, int ngroups,
                                   int *restricted, cx_restrict_plan_t *out) {
  if (!out || ngroups < 0 || (ngroups > 0 && (!groups || !restricted)))
    return fail(CX_EINVAL, "invalid argument");
  *out = nullptr;
  std::vector<cx_restrict_box_t> sel;
  for (int g = 0; g < ngroups; ++g) {
    const cx_restrict_group_t &gr = groups[g];
    restricted[g] = 0;
    if (gr.indextype < 0 || gr.indextype > 7)
      return fail(CX_EINVAL, "group %d: indextype %d out of range 0..7", g, gr.indextype);
    if (gr.ntimelevels < 0 || gr.nfabs < 0 || gr.ncomp < 0 ||
        (gr.ntimelevels > 0 && gr.nfabs > 0 && !gr.fabs))
      return fail(CX_EINVAL, "group %d: invalid time levels, FABs or components", g);
    // schedule.cxx:2746-2750: neither the regrid error nor a group with
    // restriction disabled
    if (gr.is_regrid_error || !gr.do_restrict)
      continue;
    // schedule.cxx:2755-2756: all time levels but the oldest, all of them
    // when there is only one
    const int ntl = gr.ntimelevels > 1 ? gr.ntimelevels - 1 : gr.ntimelevels;
    for (int tl = 0; tl < ntl; ++tl)
      for (int f = 0; f < gr.nfabs; ++f) {
        const cx_restrict_box_t &b = gr.fabs[(int64_t)tl * gr.nfabs + f];
        if (b.indextype != gr.indextype || b.ncomp != gr.ncomp)
          return fail(CX_EINVAL, "group %d, time level %d, FAB %d: indextype or ncomp differs "
                                 "from the group's", g, tl, f);
        sel.push_back(b);
      }
    restricted[g] = ntl;
  }
  if (int e = cx_restrict_plan_create(sel.data(), (int)sel.size(), out)) {
    for (int g = 0; g < ngroups; ++g)
      restricted[g] = 0;
    return e;
  }
  return CX_OK;
}

int cx_restrict_plan_execute(cx_restrict_plan_t p, cx_stream_t stream) {
  if (!p)
    return fail(CX_EINVAL, "null plan");
  for (int it = 0; it < 8; ++it)
    if (p->nitems[it])
      if (int e = cuda_status(launch_restrict_level(it, p->d_items[it], p->d_first[it],
                                                    p->nitems[it], p->npts[it],
                                                    (cudaStream_t)stream),
                              "restriction launch"))
        return e;
  return CX_OK;
}

int cx_restrict_plan_stats(cx_restrict_plan_t p, int64_t *ncoarse, int64_t *bytes,
                           int *nlaunches) {
  if (!p)
    return fail(CX_EINVAL, "null plan");
  if (ncoarse)
    *ncoarse = p->ncoarse;
  if (bytes)
    *bytes = p->bytes;
  if (nlaunches)
    *nlaunches = p->nlaunch;
  return CX_OK;
}

int cx_restrict_plan_destroy(cx_restrict_plan_t p) {
  if (!p)
    return CX_OK;
  for (void *d : p->d_items)
    cudaFree(d);
  for (int *d : p->d_first)
    cudaFree(d);
  delete p;
  return CX_OK;
}

int cx_restrict_adjoint_box(int indextype, const double *crse_bar, const int crse_lo[3],
                            const int crse_hi[3], double *fine_bar, const int fine_lo[3],
                            const int fine_hi[3], const int reg_lo[3], const int reg_hi[3],
                            int ncomp, cx_stream_t stream) {
  if (indextype < 0 || indextype > 7)
    return fail(CX_EUNSUPPORTED, "indextype %d out of range 0..7", indextype);
  if (!fine_lo || !fine_hi || !crse_lo || !crse_hi || !reg_lo || !reg_hi || ncomp < 0)
    return fail(CX_EINVAL, "invalid argument");
  if (!fine_bar || !crse_bar || !box_ok(fine_lo, fine_hi) || !box_ok(crse_lo, crse_hi))
    return fail(CX_EINVAL, "invalid FAB");
  if (box_ok(reg_lo, reg_hi))
    for (int d = 0; d < 3; ++d) {
      const int cc = (indextype >> (2 - d)) & 1;
      if (reg_lo[d] < crse_lo[d] || reg_hi[d] > crse_hi[d] || 2 * reg_lo[d] < fine_lo[d] ||
          2 * reg_hi[d] + cc > fine_hi[d])
        return fail(CX_EINVAL, "region does not fit the boxes in direction %d", d);
    }
  if (int e = check_device())
    return e;
  int rlo[3], rhi[3];
  for (int d = 0; d < 3; ++d) {
    rlo[d] = reg_lo[d];
    rhi[d] = reg_hi[d];
  }
  if (!box_ok(reg_lo, reg_hi)) // nothing restricted: the transpose is zero
    rhi[0] = rlo[0] - 1;
  return cuda_status(launch_restrict_adjoint_box(indextype, crse_bar, crse_lo, crse_hi, fine_bar,
                                                 fine_lo, fine_hi, rlo, rhi, ncomp,
                                                 (cudaStream_t)stream),
                     "restriction adjoint launch");
}

int cx_prolong_adjoint_box(cx_op_t op, const double *crse, const int crse_lo[3],
                           const int crse_hi[3], const double *fine_bar, const int fine_lo[3],
                           const int fine_hi[3], const int reg_lo[3], const int reg_hi[3],
                           int ncomp, int per_group, double *crse_bar, cx_stream_t stream) {
  BoxDesc b;
  bool empty;
  if (!crse_bar)
    return fail(CX_EINVAL, "null crse_bar");
  if (int e = make_box(op, crse, crse_lo, crse_hi, const_cast<double *>(fine_bar), fine_lo, fine_hi,
                       reg_lo, reg_hi, ncomp, per_group, &b, &empty))
    return e;
  if (int e = check_device())
    return e;
  cudaStream_t s = (cudaStream_t)stream;
  if (empty) {
    if (ncomp > 0 && box_ok(crse_lo, crse_hi))
      return cuda_status(
          cudaMemsetAsync(crse_bar, 0, sizeof(double) * box_points(crse_lo, crse_hi) * ncomp, s),
          "memset");
    return CX_OK;
  }
  if (!op_separable(op, per_group) || adjoint_pair_of(b) < 0) // ENO, minmod, fallback
    return cuda_status(launch_point_adjoint_box(b, per_group, crse_bar, s), "adjoint launch");
  return cuda_status(launch_prolong_adjoint_box(b, per_group, crse_bar, s), "adjoint launch");
}

} // extern "C"

// Internal entry points for the allocation-free level transfer (noalloc.cu):
// the same validation and dispatch rules as the entry points above.
namespace cxb {
int validate_box_for_level(const cx_box_t &x, int per_group, BoxDesc *b, bool *empty) {
  return make_box(x.op, x.crse, x.crse_lo, x.crse_hi, x.fine, x.fine_lo, x.fine_hi, x.reg_lo,
                  x.reg_hi, x.ncomp, per_group, b, empty);
}
bool box_uses_stream(cx_op_t op, int per_group) { return use_stream(op, per_group); }
int record_failure(int status, const char *what) { return fail(status, "%s", what); }
} // namespace cxb
