// Region copies of CarpetX's sync on one GPU: AMReX's MultiFab::FillBoundary
// (same-level halo exchange, CarpetX/src/fillpatch.cxx:34-37, 63-64) and
// MultiFab::ParallelCopy (gather of the coarse patches, :91-93, and scatter
// of the interpolated fine patches, :122-124).
//
// The host turns the FAB lists into pieces, once per regrid: each
// destination FAB's target region is carved by the sources in order (first
// source wins), so the pieces of one FAB are disjoint boxes and one launch
// over all pieces of all FABs has no write conflicts.  A piece is a box in
// destination coordinates and a shift to its source FAB.  The kernel runs a
// flat range over the pieces' points, cut into chunks of one CTA's threads
// whose first piece the host tabulates: a thread copies one point, all
// components.
#include <algorithm>
#include <array>
#include <cstdio>
#include <vector>

#include "../../include/carpetx_b200.h"
#include "cx_internal.h"

namespace cxb {
int record_failure(int status, const char *what);
}
using namespace cxb;

namespace {

struct Piece {
  const double *src;
  double *dst;
  int64_t snp, dnp; // component strides (FAB points)
  int64_t start;    // first point of the piece in the launch's point range
  int slo[3];       // source FAB lower corner
  int snx, sny, snz; // source FAB extent
  int dlo[3];
  int dnx, dny, dnz;
  int bmin[3], ext[3]; // the piece, destination coordinates
  int shift[3];        // source index = destination index + shift
};

constexpr int kThreads = 256;

__host__ __device__ __forceinline__ int64_t offset_in(const int o[3], int nx, int ny,
                                                      const int q[3]) {
  return (int64_t)(q[0] - o[0]) + nx * ((int64_t)(q[1] - o[1]) + (int64_t)ny * (q[2] - o[2]));
}

// Chunk c of kThreads consecutive points starts in piece first[c]; a thread
// scans forward from there to the last piece starting at or before its
// point (pieces are non-empty, so starts increase strictly).  Offsets within
// a piece fit in 32 bits (checked on the host).
__global__ void __launch_bounds__(kThreads)
    copy_kernel(const Piece *__restrict__ P, const int *__restrict__ first, int npieces,
                int64_t npts, int ncomp) {
  const int64_t nchunks = (npts + kThreads - 1) / kThreads;
  for (int64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int64_t p = chunk * kThreads + threadIdx.x;
    if (p >= npts)
      continue;
    int a = first[chunk];
    while (a + 1 < npieces && P[a + 1].start <= p)
      ++a;
    const Piece &g = P[a];
    const int l = (int)(p - g.start);
    const int i = l % g.ext[0];
    const int jk = l / g.ext[0];
    const int j = jk % g.ext[1];
    const int k = jk / g.ext[1];
    const int d[3] = {g.bmin[0] + i, g.bmin[1] + j, g.bmin[2] + k};
    const int s[3] = {d[0] + g.shift[0], d[1] + g.shift[1], d[2] + g.shift[2]};
    const double *src = g.src + offset_in(g.slo, g.snx, g.sny, s);
    double *dst = g.dst + offset_in(g.dlo, g.dnx, g.dny, d);
    for (int c = 0; c < ncomp; ++c)
      dst[c * g.dnp] = src[c * g.snp];
  }
}

struct IBox {
  int lo[3], hi[3];
};

bool isect(const IBox &a, const IBox &b, IBox &r) {
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = std::max(a.lo[d], b.lo[d]);
    r.hi[d] = std::min(a.hi[d], b.hi[d]);
    if (r.lo[d] > r.hi[d])
      return false;
  }
  return true;
}

// a \ b as disjoint boxes appended to out.
void subtract(const IBox &a, const IBox &b, std::vector<IBox> &out) {
  IBox c;
  if (!isect(a, b, c)) {
    out.push_back(a);
    return;
  }
  IBox rest = a;
  for (int d = 0; d < 3; ++d) {
    if (rest.lo[d] < c.lo[d]) {
      IBox x = rest;
      x.hi[d] = c.lo[d] - 1;
      out.push_back(x);
    }
    if (rest.hi[d] > c.hi[d]) {
      IBox x = rest;
      x.lo[d] = c.hi[d] + 1;
      out.push_back(x);
    }
    rest.lo[d] = c.lo[d];
    rest.hi[d] = c.hi[d];
  }
}

IBox grown(const int lo[3], const int hi[3], const int ng[3]) {
  IBox b;
  for (int d = 0; d < 3; ++d) {
    b.lo[d] = lo[d] - ng[d];
    b.hi[d] = hi[d] + ng[d];
  }
  return b;
}

IBox fab_box(const cx_fab_t &f) {
  IBox b;
  for (int d = 0; d < 3; ++d) {
    b.lo[d] = f.lo[d];
    b.hi[d] = f.hi[d];
  }
  return b;
}

int bad(const char *fmt, int a = 0) {
  char buf[256];
  snprintf(buf, sizeof buf, fmt, a);
  return record_failure(CX_EINVAL, buf);
}

int check_fabs(const cx_fab_t *f, int n) {
  if (n < 0 || (n > 0 && !f))
    return bad("invalid FAB list");
  for (int i = 0; i < n; ++i) {
    if (!f[i].data)
      return bad("null FAB data (FAB %d)", i);
    for (int d = 0; d < 3; ++d)
      if (f[i].lo[d] > f[i].hi[d] || f[i].valid_lo[d] > f[i].valid_hi[d] ||
          f[i].valid_lo[d] < f[i].lo[d] || f[i].valid_hi[d] > f[i].hi[d])
        return bad("FAB %d: the valid box must be a non-empty box inside the FAB", i);
  }
  return CX_OK;
}

// Periodic images: shift 0 first, then -period and +period per direction, z
// outermost.
std::vector<std::array<int, 3>> images(const int period[3]) {
  std::vector<int> s[3];
  for (int d = 0; d < 3; ++d) {
    s[d].push_back(0);
    if (period && period[d] > 0) {
      s[d].push_back(-period[d]);
      s[d].push_back(period[d]);
    }
  }
  std::vector<std::array<int, 3>> out;
  for (int z : s[2])
    for (int y : s[1])
      for (int x : s[0])
        out.push_back({x, y, z});
  return out;
}

struct Builder {
  std::vector<Piece> pieces;
  int64_t npts = 0;

  // Carves the target boxes of destination dst by the sources in order and
  // emits a piece per covered part.  src_region[j]: source j's box (valid,
  // grown) clipped to its FAB.  skip_self: FillBoundary's rule.
  void carve(const cx_fab_t &dst, int di, std::vector<IBox> remaining, const cx_fab_t *src,
             const std::vector<IBox> &src_region, int nsrc,
             const std::vector<std::array<int, 3>> &imgs, bool skip_self) {
    const IBox bound = fab_box(dst);
    for (int j = 0; j < nsrc && !remaining.empty(); ++j)
      for (const auto &sh : imgs) {
        if (skip_self && j == di && sh[0] == 0 && sh[1] == 0 && sh[2] == 0)
          continue;
        IBox S = src_region[j], t;
        for (int d = 0; d < 3; ++d) {
          S.lo[d] += sh[d];
          S.hi[d] += sh[d];
        }
        if (!isect(bound, S, t))
          continue;
        std::vector<IBox> next;
        for (const IBox &r : remaining) {
          IBox c;
          if (!isect(r, S, c)) {
            next.push_back(r);
            continue;
          }
          emit(dst, src[j], c, sh);
          subtract(r, S, next);
        }
        remaining.swap(next);
        if (remaining.empty())
          break;
      }
  }

  void emit(const cx_fab_t &dst, const cx_fab_t &src, const IBox &c,
            const std::array<int, 3> &sh) {
    Piece g{};
    g.src = src.data;
    g.dst = dst.data;
    g.snx = src.hi[0] - src.lo[0] + 1;
    g.sny = src.hi[1] - src.lo[1] + 1;
    g.snz = src.hi[2] - src.lo[2] + 1;
    g.dnx = dst.hi[0] - dst.lo[0] + 1;
    g.dny = dst.hi[1] - dst.lo[1] + 1;
    g.dnz = dst.hi[2] - dst.lo[2] + 1;
    g.snp = (int64_t)g.snx * g.sny * g.snz;
    g.dnp = (int64_t)g.dnx * g.dny * g.dnz;
    for (int d = 0; d < 3; ++d) {
      g.slo[d] = src.lo[d];
      g.dlo[d] = dst.lo[d];
      g.bmin[d] = c.lo[d];
      g.ext[d] = c.hi[d] - c.lo[d] + 1;
      g.shift[d] = -sh[d];
    }
    g.start = npts;
    npts += (int64_t)g.ext[0] * g.ext[1] * g.ext[2];
    pieces.push_back(g);
  }
};

// Every piece lies in its destination FAB and, shifted, in its source FAB.
bool pieces_in_bounds(const std::vector<Piece> &ps) {
  for (const Piece &g : ps) {
    const int dn[3] = {g.dnx, g.dny, g.dnz}, sn[3] = {g.snx, g.sny, g.snz};
    for (int d = 0; d < 3; ++d) {
      const int a = g.bmin[d], b = g.bmin[d] + g.ext[d] - 1;
      if (g.ext[d] <= 0 || a < g.dlo[d] || b > g.dlo[d] + dn[d] - 1 ||
          a + g.shift[d] < g.slo[d] || b + g.shift[d] > g.slo[d] + sn[d] - 1)
        return false;
    }
    if ((int64_t)g.ext[0] * g.ext[1] * g.ext[2] > INT32_MAX)
      return false;
  }
  return true;
}

// first[c]: the piece containing point c * kThreads.
std::vector<int> chunk_firsts(const std::vector<Piece> &ps, int64_t npts) {
  const int64_t nchunks = (npts + kThreads - 1) / kThreads;
  std::vector<int> f(nchunks);
  size_t a = 0;
  for (int64_t c = 0; c < nchunks; ++c) {
    const int64_t p = c * kThreads;
    while (a + 1 < ps.size() && ps[a + 1].start <= p)
      ++a;
    f[c] = (int)a;
  }
  return f;
}

std::vector<IBox> source_regions(const cx_fab_t *src, int n, const int ng[3]) {
  std::vector<IBox> r(n);
  for (int j = 0; j < n; ++j) {
    IBox c;
    // non-empty: the valid box lies inside the FAB (checked)
    isect(grown(src[j].valid_lo, src[j].valid_hi, ng), fab_box(src[j]), c);
    r[j] = c;
  }
  return r;
}

int check_common(int ncomp, const int *a, const int *b, const int period[3], void *out) {
  if (!out)
    return bad("null plan pointer");
  if (ncomp < 1)
    return bad("ncomp %d < 1", ncomp);
  for (int d = 0; d < 3; ++d) {
    if ((a && a[d] < 0) || (b && b[d] < 0))
      return bad("negative ghost count in direction %d", d);
    if (period && period[d] < 0)
      return bad("negative period in direction %d", d);
  }
  return CX_OK;
}

} // namespace

struct cx_copy_plan {
  Piece *d_pieces = nullptr;
  int *d_first = nullptr; // chunk -> first piece
  int npieces = 0;
  int64_t npts = 0;
  int ncomp = 0;
};

namespace {

int finish(Builder &b, int ncomp, cx_copy_plan_t *out) {
  if (!pieces_in_bounds(b.pieces))
    return bad("internal error: a piece leaves its FAB");
  if (b.pieces.size() > (size_t)INT32_MAX)
    return bad("too many pieces");
  cx_copy_plan *p = new cx_copy_plan;
  p->npieces = (int)b.pieces.size();
  p->npts = b.npts;
  p->ncomp = ncomp;
  if (!b.pieces.empty()) {
    const std::vector<int> first = chunk_firsts(b.pieces, b.npts);
    cudaError_t e = cudaMalloc(&p->d_pieces, b.pieces.size() * sizeof(Piece));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_pieces, b.pieces.data(), b.pieces.size() * sizeof(Piece),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMalloc(&p->d_first, first.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_first, first.data(), first.size() * sizeof(int),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(p->d_pieces);
      cudaFree(p->d_first);
      delete p;
      char buf[256];
      snprintf(buf, sizeof buf, "copy plan upload: %s", cudaGetErrorString(e));
      return record_failure(e == cudaErrorMemoryAllocation ? CX_ENOMEM : CX_ECUDA, buf);
    }
  }
  *out = p;
  return CX_OK;
}

} // namespace

extern "C" {

int cx_copy_plan_parallel_copy(const cx_fab_t *dst, int ndst, const cx_fab_t *src, int nsrc,
                               int ncomp, const int src_nghost[3], const int dst_nghost[3],
                               const int period[3], cx_copy_plan_t *out) {
  if (out)
    *out = nullptr;
  if (!src_nghost || !dst_nghost)
    return bad("null ghost counts");
  if (int e = check_common(ncomp, src_nghost, dst_nghost, period, out))
    return e;
  if (int e = check_fabs(dst, ndst))
    return e;
  if (int e = check_fabs(src, nsrc))
    return e;
  const auto imgs = images(period);
  const auto regions = source_regions(src, nsrc, src_nghost);
  Builder b;
  for (int i = 0; i < ndst; ++i) {
    IBox t;
    if (!isect(grown(dst[i].valid_lo, dst[i].valid_hi, dst_nghost), fab_box(dst[i]), t))
      continue;
    b.carve(dst[i], i, {t}, src, regions, nsrc, imgs, false);
  }
  return finish(b, ncomp, out);
}

int cx_copy_plan_fill_boundary(const cx_fab_t *fabs, int nfabs, int ncomp, const int nghost[3],
                               const int period[3], cx_copy_plan_t *out) {
  if (out)
    *out = nullptr;
  if (!nghost)
    return bad("null ghost counts");
  if (int e = check_common(ncomp, nghost, nullptr, period, out))
    return e;
  if (int e = check_fabs(fabs, nfabs))
    return e;
  const auto imgs = images(period);
  const int zero[3] = {0, 0, 0};
  const auto regions = source_regions(fabs, nfabs, zero);
  Builder b;
  for (int i = 0; i < nfabs; ++i) {
    IBox g;
    if (!isect(grown(fabs[i].valid_lo, fabs[i].valid_hi, nghost), fab_box(fabs[i]), g))
      continue;
    std::vector<IBox> ring;
    subtract(g, grown(fabs[i].valid_lo, fabs[i].valid_hi, zero), ring); // the ghost shell
    if (!ring.empty())
      b.carve(fabs[i], i, ring, fabs, regions, nfabs, imgs, true);
  }
  return finish(b, ncomp, out);
}

int cx_copy_plan_execute(cx_copy_plan_t p, cx_stream_t stream) {
  if (!p)
    return bad("null plan");
  if (p->npts == 0)
    return CX_OK;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (p->npts + kThreads - 1) / kThreads;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)nsm * 8));
  copy_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(p->d_pieces, p->d_first, p->npieces,
                                                           p->npts, p->ncomp);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof buf, "copy launch: %s", cudaGetErrorString(e));
    return record_failure(CX_ECUDA, buf);
  }
  return CX_OK;
}

int cx_copy_plan_stats(cx_copy_plan_t p, int64_t *npoints, int64_t *npieces, int64_t *bytes) {
  if (!p)
    return bad("null plan");
  if (npoints)
    *npoints = p->npts;
  if (npieces)
    *npieces = p->npieces;
  if (bytes)
    *bytes = 16 * p->npts * p->ncomp;
  return CX_OK;
}

int cx_copy_plan_destroy(cx_copy_plan_t p) {
  if (!p)
    return CX_OK;
  cudaFree(p->d_pieces);
  cudaFree(p->d_first);
  delete p;
  return CX_OK;
}

} // extern "C"
