// Reflux of a coarse level from the next finer one, as CarpetX's Reflux()
// does it through AMReX's FluxRegister (CarpetX/src/schedule.cxx:2632-2713,
// the register built at driver.cxx:918-924):
//   for each direction d:  freg.CrseInit(coarse flux_d, d, 0, 0, n, -1);
//                          freg.FineAdd(fine flux_d, d, 0, 0, n, +1);
//   freg.Reflux(coarse state, 1.0, 0, 0, n, coarse geometry).
// AMReX (25.11) is not in the reference tree; the restatement follows the
// FluxRegister's documented semantics and its implementation's order of
// operations:
//   - a register per fine box and face orientation holds, on the coarse
//     faces of the coarsened box's boundary, mult_c * (coarse flux) (COPY
//     from the first coarse flux FAB whose valid faces hold the face), then
//     adds mult_f * (fine flux) of the 2 x 2 fine faces that cover each
//     coarse face, the higher transverse direction outer;
//   - Reflux adds to the coarse cell just outside the fine box (below a low
//     face, above a high face) -scale * reg / vol for a low face and
//     +scale * reg / vol for a high face, vol = dx * dy * dz of the coarse
//     cells, orientation by orientation (x, y, z low, then x, y, z high).
// Within one orientation no coarse cell is the outside neighbour of two
// registers (the fine boxes are disjoint), so a launch per orientation needs
// no atomics; coarse cells under other fine boxes get corrections too, as in
// AMReX, and are overwritten by the restriction that follows.  The three
// steps are fused: the register value lives in a register of the thread.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "../../include/carpetx_b200.h"
#include "cx_internal.h"

namespace cxb {
int record_failure(int status, const char *what);
}
using namespace cxb;

namespace {

struct RPiece {
  double *u;             // coarse state FAB
  const double *fc;      // coarse flux FAB (direction d)
  const double *ff;      // fine flux FAB (direction d) of the register's fine box
  int64_t unp, fcnp, ffnp; // component strides
  int64_t start;         // first point in the launch's range
  int ulo[3], unx, uny;  // state FAB lower corner and extents
  int clo[3], cnx, cny;  // coarse flux FAB
  int flo[3], fnx, fny;  // fine flux FAB
  int bmin[3], ext[3];   // the coarse cells of the piece (outside the fine box)
  int face;              // coarse face index in direction d of the register
  int fface;             // the fine face index in direction d
};

constexpr int kThreads = 256;

__device__ __forceinline__ int64_t off3(const int o[3], int nx, int ny, int x, int y, int z) {
  return (int64_t)(x - o[0]) + nx * ((int64_t)(y - o[1]) + (int64_t)ny * (z - o[2]));
}

// One orientation: direction D, sgn -1 (low face) or +1 (high face).
template <int D>
__global__ void __launch_bounds__(kThreads)
    reflux_kernel(const RPiece *__restrict__ P, const int *__restrict__ first, int npieces,
                  int64_t npts, int ncomp, double sgn_scale, double vol) {
  const int64_t nchunks = (npts + kThreads - 1) / kThreads;
  constexpr int E1 = D == 0 ? 1 : 0, E2 = D == 2 ? 1 : 2; // transverse directions, E1 < E2
  for (int64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int64_t p = chunk * kThreads + threadIdx.x;
    if (p >= npts)
      continue;
    int a = first[chunk];
    while (a + 1 < npieces && P[a + 1].start <= p)
      ++a;
    const RPiece &g = P[a];
    const int l = (int)(p - g.start);
    int c[3];
    c[0] = g.bmin[0] + l % g.ext[0];
    c[1] = g.bmin[1] + (l / g.ext[0]) % g.ext[1];
    c[2] = g.bmin[2] + l / (g.ext[0] * g.ext[1]);
    int fcq[3] = {c[0], c[1], c[2]};
    fcq[D] = g.face;
    double *u = g.u + off3(g.ulo, g.unx, g.uny, c[0], c[1], c[2]);
    const double *fc = g.fc + off3(g.clo, g.cnx, g.cny, fcq[0], fcq[1], fcq[2]);
    int fq[3];
    fq[D] = g.fface;
    for (int n = 0; n < ncomp; ++n) {
      // CrseInit with mult -1 (the product by -1 is exact), FineAdd with
      // mult +1 (exact): the register value
      double r = -fc[n * g.fcnp];
#pragma unroll
      for (int o2 = 0; o2 < 2; ++o2)
#pragma unroll
        for (int o1 = 0; o1 < 2; ++o1) {
          fq[E1] = 2 * c[E1] + o1;
          fq[E2] = 2 * c[E2] + o2;
          r = __dadd_rn(r, g.ff[n * g.ffnp + off3(g.flo, g.fnx, g.fny, fq[0], fq[1], fq[2])]);
        }
      // Reflux: s += (+-scale * reg) / vol
      u[n * g.unp] = __dadd_rn(u[n * g.unp], __ddiv_rn(__dmul_rn(sgn_scale, r), vol));
    }
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

IBox valid_of(const cx_fab_t &f) {
  IBox b;
  for (int d = 0; d < 3; ++d) {
    b.lo[d] = f.valid_lo[d];
    b.hi[d] = f.valid_hi[d];
  }
  return b;
}

int64_t npts_of(const IBox &b) {
  return (int64_t)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
}

int bad(const char *fmt, int a = 0, int b = 0) {
  char buf[256];
  snprintf(buf, sizeof buf, fmt, a, b);
  return record_failure(CX_EINVAL, buf);
}

bool inside(const IBox &in, const cx_fab_t &f) {
  for (int d = 0; d < 3; ++d)
    if (in.lo[d] < f.lo[d] || in.hi[d] > f.hi[d])
      return false;
  return true;
}

int check_list(const cx_fab_t *f, int n, const char *what) {
  if (n < 0 || (n > 0 && !f))
    return record_failure(CX_EINVAL, what);
  for (int i = 0; i < n; ++i) {
    if (!f[i].data)
      return record_failure(CX_EINVAL, what);
    for (int d = 0; d < 3; ++d)
      if (f[i].lo[d] > f[i].hi[d] || f[i].valid_lo[d] > f[i].valid_hi[d] ||
          f[i].valid_lo[d] < f[i].lo[d] || f[i].valid_hi[d] > f[i].hi[d])
        return record_failure(CX_EINVAL, what);
  }
  return CX_OK;
}

} // namespace

struct cx_reflux_plan {
  RPiece *d_pieces[6] = {};
  int *d_first[6] = {};
  int npieces[6] = {};
  int64_t npts[6] = {};
  int ncomp = 0;
  double sgn_scale[6] = {};
  double vol = 1.0;
  int64_t faces = 0, bytes = 0;
};

extern "C" {

int cx_reflux_plan_create(const cx_fab_t *crse, int ncrse, const cx_fab_t *const crse_flux[3],
                          const cx_fab_t *const fine_flux[3], int nfine, int ncomp,
                          const double dx[3], double scale, cx_reflux_plan_t *out) {
  if (!out || !crse_flux || !fine_flux || !dx || ncomp < 1)
    return bad("invalid argument");
  *out = nullptr;
  if (int e = check_list(crse, ncrse, "invalid coarse state FAB"))
    return e;
  for (int d = 0; d < 3; ++d) {
    if (int e = check_list(crse_flux[d], ncrse, "invalid coarse flux FAB"))
      return e;
    if (int e = check_list(fine_flux[d], nfine, "invalid fine flux FAB"))
      return e;
  }
  // the flux FABs' valid boxes are the state's, face centred in their
  // direction; the fine boxes, coarsenable by 2, from the x fluxes
  std::vector<IBox> fbox(nfine);
  for (int d = 0; d < 3; ++d) {
    for (int i = 0; i < ncrse; ++i)
      for (int e = 0; e < 3; ++e)
        if (crse_flux[d][i].valid_lo[e] != crse[i].valid_lo[e] ||
            crse_flux[d][i].valid_hi[e] != crse[i].valid_hi[e] + (e == d))
          return bad("coarse flux FAB %d of direction %d: valid box is not the state's, face "
                     "centred", i, d);
  }
  for (int b = 0; b < nfine; ++b) {
    fbox[b] = valid_of(fine_flux[0][b]);
    fbox[b].hi[0] -= 1;
    for (int d = 0; d < 3; ++d) {
      for (int e = 0; e < 3; ++e)
        if (fine_flux[d][b].valid_lo[e] != fbox[b].lo[e] ||
            fine_flux[d][b].valid_hi[e] != fbox[b].hi[e] + (e == d))
          return bad("fine flux FAB %d of direction %d: valid box differs from the box's "
                     "face-centred cells", b, d);
      if ((fbox[b].lo[d] & 1) || !(fbox[b].hi[d] & 1))
        return bad("fine box %d is not coarsenable by 2 in direction %d", b, d);
    }
  }
  cx_reflux_plan *p = new cx_reflux_plan;
  p->ncomp = ncomp;
  p->vol = (dx[0] * dx[1]) * dx[2];
  // orientations in AMReX's order: x, y, z low, then x, y, z high
  for (int o = 0; o < 6; ++o) {
    const int d = o % 3, hi = o / 3;
    p->sgn_scale[o] = hi ? scale : -scale;
    std::vector<RPiece> pcs;
    int64_t start = 0;
    for (int b = 0; b < nfine; ++b) {
      IBox reg; // the outside coarse cells of the register's faces
      for (int e = 0; e < 3; ++e) {
        reg.lo[e] = fbox[b].lo[e] >> 1;
        reg.hi[e] = fbox[b].hi[e] >> 1;
      }
      const int face = hi ? reg.hi[d] + 1 : reg.lo[d];
      const int fface = hi ? fbox[b].hi[d] + 1 : fbox[b].lo[d];
      reg.lo[d] = reg.hi[d] = hi ? face : face - 1;
      // the fine flux faces the register reads lie in the box's flux FAB
      IBox ffx;
      for (int e = 0; e < 3; ++e) {
        ffx.lo[e] = fbox[b].lo[e];
        ffx.hi[e] = fbox[b].hi[e];
      }
      ffx.lo[d] = ffx.hi[d] = fface;
      if (!inside(ffx, fine_flux[d][b])) {
        cx_reflux_plan_destroy(p);
        return bad("fine flux FAB %d of direction %d lacks the box's boundary faces", b, d);
      }
      for (int i = 0; i < ncrse; ++i) {
        IBox cells;
        if (!isect(reg, valid_of(crse[i]), cells))
          continue;
        // the coarse flux of these faces: the first coarse flux FAB whose
        // valid faces hold them (AMReX's copy from the valid regions)
        std::vector<IBox> rem{cells};
        for (int j = 0; j < ncrse && !rem.empty(); ++j) {
          IBox cf = valid_of(crse_flux[d][j]);
          // faces at index `face` of cells c: c's d index replaced by face
          std::vector<IBox> next;
          for (const IBox &r : rem) {
            IBox rf = r;
            rf.lo[d] = rf.hi[d] = face;
            IBox got;
            if (!isect(rf, cf, got)) {
              next.push_back(r);
              continue;
            }
            IBox gc = got;
            gc.lo[d] = gc.hi[d] = r.lo[d];
            subtract(r, gc, next);
            RPiece q{};
            q.u = crse[i].data;
            q.fc = crse_flux[d][j].data;
            q.ff = fine_flux[d][b].data;
            auto strides = [](const cx_fab_t &f, int lo[3], int &nx, int &ny) {
              for (int e = 0; e < 3; ++e)
                lo[e] = f.lo[e];
              nx = f.hi[0] - f.lo[0] + 1;
              ny = f.hi[1] - f.lo[1] + 1;
              return (int64_t)nx * ny * (f.hi[2] - f.lo[2] + 1);
            };
            q.unp = strides(crse[i], q.ulo, q.unx, q.uny);
            q.fcnp = strides(crse_flux[d][j], q.clo, q.cnx, q.cny);
            q.ffnp = strides(fine_flux[d][b], q.flo, q.fnx, q.fny);
            for (int e = 0; e < 3; ++e) {
              q.bmin[e] = gc.lo[e];
              q.ext[e] = gc.hi[e] - gc.lo[e] + 1;
            }
            q.face = face;
            q.fface = fface;
            q.start = start;
            start += npts_of(gc);
            pcs.push_back(q);
          }
          rem.swap(next);
        }
      }
    }
    p->npieces[o] = (int)pcs.size();
    p->npts[o] = start;
    p->faces += start;
    p->bytes += start * ncomp * 8 * (1 + 4 + 2);
    if (pcs.empty())
      continue;
    std::vector<int> first((start + kThreads - 1) / kThreads);
    size_t a = 0;
    for (size_t c = 0; c < first.size(); ++c) {
      while (a + 1 < pcs.size() && pcs[a + 1].start <= (int64_t)c * kThreads)
        ++a;
      first[c] = (int)a;
    }
    cudaError_t e = cudaMalloc(&p->d_pieces[o], pcs.size() * sizeof(RPiece));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_pieces[o], pcs.data(), pcs.size() * sizeof(RPiece),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMalloc(&p->d_first[o], first.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_first[o], first.data(), first.size() * sizeof(int),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaGetLastError();
      cx_reflux_plan_destroy(p);
      return record_failure(e == cudaErrorMemoryAllocation ? CX_ENOMEM : CX_ECUDA,
                            "reflux plan upload failed");
    }
  }
  *out = p;
  return CX_OK;
}

int cx_reflux_plan_execute(cx_reflux_plan_t p, cx_stream_t stream) {
  if (!p)
    return bad("null plan");
  for (int o = 0; o < 6; ++o) {
    if (!p->npieces[o])
      continue;
    const int64_t nch = (p->npts[o] + kThreads - 1) / kThreads;
    const unsigned grid = (unsigned)std::min<int64_t>(nch, 148 * 8);
    cudaStream_t s = (cudaStream_t)stream;
    switch (o % 3) {
    case 0:
      reflux_kernel<0><<<grid, kThreads, 0, s>>>(p->d_pieces[o], p->d_first[o], p->npieces[o],
                                                 p->npts[o], p->ncomp, p->sgn_scale[o], p->vol);
      break;
    case 1:
      reflux_kernel<1><<<grid, kThreads, 0, s>>>(p->d_pieces[o], p->d_first[o], p->npieces[o],
                                                 p->npts[o], p->ncomp, p->sgn_scale[o], p->vol);
      break;
    default:
      reflux_kernel<2><<<grid, kThreads, 0, s>>>(p->d_pieces[o], p->d_first[o], p->npieces[o],
                                                 p->npts[o], p->ncomp, p->sgn_scale[o], p->vol);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      return record_failure(CX_ECUDA, "reflux launch failed");
  }
  return CX_OK;
}

int cx_reflux_plan_stats(cx_reflux_plan_t p, int64_t *faces, int64_t *bytes, int *launches) {
  if (!p)
    return bad("null plan");
  if (faces)
    *faces = p->faces;
  if (bytes)
    *bytes = p->bytes;
  if (launches) {
    int n = 0;
    for (int o = 0; o < 6; ++o)
      n += p->npieces[o] > 0;
    *launches = n;
  }
  return CX_OK;
}

int cx_reflux_plan_destroy(cx_reflux_plan_t p) {
  if (!p)
    return CX_OK;
  for (int o = 0; o < 6; ++o) {
    cudaFree(p->d_pieces[o]);
    cudaFree(p->d_first[o]);
  }
  delete p;
  return CX_OK;
}

} // extern "C"
