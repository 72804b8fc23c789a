// Outer boundary conditions: CarpetX's BoundaryCondition
// (CarpetX/src/boundaries.cxx:32-118, boundaries_impl.hxx:28-444) for one
// FArrayBox, and GroupData::apply_boundary_conditions (driver.cxx:967-995)
// for every FArrayBox of a level in one launch.
//
// The host splits each FAB into the regions outside the domain interior
// (below, inside or above it per direction, at most 26) exactly as
// apply_on_face does, resolves each direction's condition and its source
// coordinate, and checks every source point: it lies inside the FAB and
// inside the interior in every direction that has a condition.  No point
// that is read is then one that is written, so the regions of all FABs are
// independent and one launch of a flat point range replaces the reference's
// launch per region and FAB.  A thread sets one point, all components.
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

enum : int { BM_NONE = 0, BM_DIRICHLET, BM_LINEXT, BM_NEUMANN, BM_ROBIN, BM_REFLECT, BM_BAD };
enum : int { F_DIRICHLET = 1, F_ROBIN = 2, F_LINEXT = 4, F_REFLECT = 8 };

// One region of one FAB and how its points are set.
struct Region {
  double *data;    // component 0 of the FAB
  int64_t np;      // component stride: points of the FAB
  int64_t start;   // first point of the region in the launch's point range
  int dmin[3];     // FAB lower corner
  int nx, ny;      // FAB extent in x and y
  int bmin[3];     // region lower corner
  int ext[3];      // region extent (all positive)
  int mode[3];     // BM_* per direction
  int srcc[3];     // source coordinate (linear extrapolation, Neumann, Robin)
                   // or reflection offset (source = offset - destination)
  int delta[3];    // second point of a linear extrapolation: -normal
  int flags;       // F_* of the conditions present
  int nrobin;      // Robin directions (the fall-off is applied once per each)
  uint32_t negpar; // bit c: the reflection parity of component c is -1
};

struct Consts {
  double dirichlet[CX_BC_MAX_COMPS], robin[CX_BC_MAX_COMPS];
  double xmin[3], dx[3];
  int ncomp;
  int nreg;
  int64_t npts;
};

constexpr int kMaxBoxRegions = 26;
struct BoxRegions {
  Region r[kMaxBoxRegions];
};
static_assert(sizeof(Consts) + sizeof(BoxRegions) + sizeof(void *) <= 4096,
              "kernel parameters within 4 KB");

constexpr int kThreads = 256;

// |x| of grid point p: sqrt(sum(pow2(xmin + p * dx))), products and sums
// rounded separately, summed from x to z as Arith's fold does.
__device__ __forceinline__ double radius(const Consts &k, const int p[3]) {
  double s = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double x = __dadd_rn(k.xmin[d], __dmul_rn((double)p[d], k.dx[d]));
    s = __dadd_rn(s, __dmul_rn(x, x));
  }
  return __dsqrt_rn(s);
}

// Source point, second point (linear extrapolation) and the three offsets
// into the FAB of destination point dst of region g.  The host checks these
// at the eight corners of every region before any launch: each offset is
// affine in dst per direction, so the corners bound every access.
struct Access {
  int src[3], sp[3];
  int64_t od, os, osp;
};
__host__ __device__ __forceinline__ int64_t fab_offset(const Region &g, const int q[3]) {
  return (int64_t)(q[0] - g.dmin[0]) +
         g.nx * ((int64_t)(q[1] - g.dmin[1]) + (int64_t)g.ny * (q[2] - g.dmin[2]));
}
__host__ __device__ __forceinline__ Access access_of(const Region &g, const int dst[3]) {
  Access a;
  for (int d = 0; d < 3; ++d) {
    const int m = g.mode[d];
    a.src[d] = m == BM_REFLECT ? g.srcc[d] - dst[d]
               : (m == BM_LINEXT || m == BM_NEUMANN || m == BM_ROBIN) ? g.srcc[d]
                                                                      : dst[d];
    a.sp[d] = a.src[d] + g.delta[d];
  }
  a.od = fab_offset(g, dst);
  a.os = fab_offset(g, a.src);
  a.osp = fab_offset(g, a.sp);
  return a;
}

// regs: the level plan's device list, with first[c] the region containing
// point c * kThreads (a thread scans forward from it); or nullptr for the
// regions passed by value (one FAB, at most 26: binary search).  Offsets
// within a region fit in 32 bits (checked on the host).
__global__ void __launch_bounds__(kThreads)
    boundary_kernel(const __grid_constant__ Consts k, const Region *__restrict__ regs,
                    const int *__restrict__ first, const __grid_constant__ BoxRegions own) {
  const Region *R = regs ? regs : own.r;
  const int64_t nchunks = (k.npts + kThreads - 1) / kThreads;
  for (int64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int64_t p = chunk * kThreads + threadIdx.x;
    if (p >= k.npts)
      continue;
    int a;
    if (regs) {
      a = first[chunk];
      while (a + 1 < k.nreg && R[a + 1].start <= p)
        ++a;
    } else {
      a = 0; // last region starting at or before p
      int b = k.nreg - 1;
      while (a < b) {
        const int m = (a + b + 1) >> 1;
        if (R[m].start <= p)
          a = m;
        else
          b = m - 1;
      }
    }
    const Region &g = R[a];
    const int l = (int)(p - g.start);
    const int i = l % g.ext[0];
    const int jk = l / g.ext[0];
    const int j = jk % g.ext[1];
    const int kz = jk / g.ext[1];
    const int dst[3] = {g.bmin[0] + i, g.bmin[1] + j, g.bmin[2] + kz};
    const Access x = access_of(g, dst);
    // Robin: the fall-off factor |x_src| / |x_dst| is the same in every
    // Robin direction.  Linear extrapolation: the distance ratio is the
    // integer quotient of the squared lengths, as in the reference.
    double q = 0, s = 0;
    if (g.flags & F_ROBIN)
      q = __ddiv_rn(radius(k, x.src), radius(k, dst));
    if (g.flags & F_LINEXT) {
      int n2 = 0, d2 = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        n2 += (dst[d] - x.src[d]) * (dst[d] - x.src[d]);
        d2 += g.delta[d] * g.delta[d];
      }
      s = __dsqrt_rn((double)(n2 / d2));
    }
    // Components in groups of four: their source values are loaded before
    // any of them is stored (no point read in a launch is written in it), so
    // four loads are in flight; each component's arithmetic is unchanged.
    const bool dir = g.flags & F_DIRICHLET, lin = g.flags & F_LINEXT;
    for (int c0 = 0; c0 < k.ncomp; c0 += 4) {
      const int n = min(4, k.ncomp - c0);
      double v[4], w[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        v[u] = w[u] = 0;
        if (u < n && !dir) {
          const double *col = g.data + (int64_t)(c0 + u) * g.np;
          v[u] = col[x.os];
          if (lin)
            w[u] = col[x.osp];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (u >= n)
          break;
        const int c = c0 + u;
        double val;
        if (dir) {
          val = k.dirichlet[c];
        } else {
          val = v[u];
          for (int r = 0; r < g.nrobin; ++r)
            val = __dadd_rn(k.robin[c], __dmul_rn(q, __dsub_rn(val, k.robin[c])));
          if (lin)
            val = __dadd_rn(val, __dmul_rn(s, __dsub_rn(val, w[u])));
          if ((g.negpar >> c) & 1u) // parity -1 (only set in reflection regions)
            val = -val;
        }
        g.data[(int64_t)c * g.np + x.od] = val;
      }
    }
  }
}

// Every offset the kernel forms for region g lies in [0, np): checked at the
// region's corners with the kernel's own index code.
bool region_in_fab(const Region &g) {
  for (int c = 0; c < 8; ++c) {
    int dst[3];
    for (int d = 0; d < 3; ++d)
      dst[d] = g.bmin[d] + (((c >> d) & 1) ? g.ext[d] - 1 : 0);
    const Access a = access_of(g, dst);
    const bool rd = !(g.flags & F_DIRICHLET);
    if (a.od < 0 || a.od >= g.np || (rd && (a.os < 0 || a.os >= g.np)) ||
        (rd && (g.flags & F_LINEXT) && (a.osp < 0 || a.osp >= g.np)))
      return false;
  }
  return true;
}

// Condition of direction d on face f, as apply_on_face chooses it
// (boundaries_impl.hxx:71-108).
int mode_of(const cx_bc_t &bc, int f, int d) {
  const int s = bc.symmetry[f][d], b = bc.boundary[f][d];
  if (((s == CX_SYM_NONE || s == CX_SYM_INTERPATCH) && b == CX_BC_NONE) || s == CX_SYM_PERIODIC)
    return BM_NONE;
  if (s == CX_SYM_REFLECTION)
    return BM_REFLECT;
  switch (b) {
  case CX_BC_DIRICHLET: return BM_DIRICHLET;
  case CX_BC_LINEAR_EXTRAPOLATION: return BM_LINEXT;
  case CX_BC_NEUMANN: return BM_NEUMANN;
  case CX_BC_ROBIN: return BM_ROBIN;
  default: return BM_BAD;
  }
}

int bad(const char *fmt, int a = 0, int b = 0) {
  char buf[256];
  snprintf(buf, sizeof buf, fmt, a, b);
  return record_failure(CX_EINVAL, buf);
}

int check_bc(const cx_bc_t *bc) {
  if (!bc)
    return bad("null boundary description");
  if (bc->ncomp < 1 || bc->ncomp > CX_BC_MAX_COMPS)
    return bad("ncomp %d outside 1..%d", bc->ncomp, CX_BC_MAX_COMPS);
  for (int d = 0; d < 3; ++d) {
    if (bc->domain_hi[d] < bc->domain_lo[d])
      return bad("empty domain in direction %d", d);
    if (bc->indextype[d] != 0 && bc->indextype[d] != 1)
      return bad("indextype %d in direction %d", bc->indextype[d], d);
    if (bc->nghost[d] < 0)
      return bad("negative ghost count in direction %d", d);
  }
  return CX_OK;
}

Consts make_consts(const cx_bc_t &bc) {
  Consts k{};
  for (int c = 0; c < bc.ncomp; ++c) {
    k.dirichlet[c] = bc.dirichlet[c];
    k.robin[c] = bc.robin[c];
  }
  for (int d = 0; d < 3; ++d) {
    // vertex coordinates shifted as in the constructor (boundaries.cxx:45-48)
    k.xmin[d] = bc.prob_lo[d] + 0.5 * bc.indextype[d] - 1;
    k.dx[d] = bc.dx[d];
  }
  k.ncomp = bc.ncomp;
  return k;
}

// Appends the regions of one FAB; npts and bytes accumulate.
int add_fab(const cx_bc_t &bc, double *data, const int lo[3], const int hi[3],
            std::vector<Region> &out, int64_t &npts, int64_t &bytes) {
  if (!data || !lo || !hi)
    return bad("null FAB");
  int imin[3], imax[3], dmin[3], dmax[3];
  for (int d = 0; d < 3; ++d) {
    if (hi[d] < lo[d])
      return bad("empty FAB in direction %d", d);
    imin[d] = bc.domain_lo[d];
    imax[d] = bc.domain_hi[d] + 1 + !bc.indextype[d];
    dmin[d] = lo[d];
    dmax[d] = hi[d] + 1;
  }
  const int64_t np = (int64_t)(dmax[0] - dmin[0]) * (dmax[1] - dmin[1]) * (dmax[2] - dmin[2]);
  for (int nk = -1; nk <= 1; ++nk)
    for (int nj = -1; nj <= 1; ++nj)
      for (int ni = -1; ni <= 1; ++ni) {
        const int nrm[3] = {ni, nj, nk};
        if (!ni && !nj && !nk)
          continue;
        Region g{};
        bool empty = false, any = false;
        for (int d = 0; d < 3; ++d) {
          int b0, b1;
          if (nrm[d] < 0) {
            b0 = dmin[d];
            b1 = std::min(dmax[d], imin[d]);
          } else if (nrm[d] > 0) {
            b0 = std::max(dmin[d], imax[d]);
            b1 = dmax[d];
          } else {
            b0 = std::max(dmin[d], imin[d]);
            b1 = std::min(dmax[d], imax[d]);
          }
          empty |= b1 <= b0;
          g.bmin[d] = b0;
          g.ext[d] = b1 - b0;
        }
        if (empty)
          continue;
        for (int d = 0; d < 3; ++d) {
          const int m = nrm[d] ? mode_of(bc, nrm[d] > 0, d) : BM_NONE;
          if (m == BM_BAD)
            return bad("direction %d, face %d: symmetry and boundary condition do not combine", d,
                       nrm[d] > 0);
          g.mode[d] = m;
          any |= m != BM_NONE;
        }
        if (!any)
          continue;
        for (int d = 0; d < 3; ++d) {
          const int m = g.mode[d];
          const int edge = nrm[d] < 0 ? imin[d] : imax[d] - 1;
          // lowest and highest source coordinate of the region
          int s0 = g.bmin[d], s1 = g.bmin[d] + g.ext[d] - 1;
          switch (m) {
          case BM_DIRICHLET: g.flags |= F_DIRICHLET; break;
          case BM_LINEXT:
            g.flags |= F_LINEXT;
            g.srcc[d] = edge;
            g.delta[d] = -nrm[d];
            s0 = std::min(edge, edge - nrm[d]);
            s1 = std::max(edge, edge - nrm[d]);
            break;
          case BM_NEUMANN: g.srcc[d] = s0 = s1 = edge; break;
          case BM_ROBIN:
            g.flags |= F_ROBIN;
            ++g.nrobin;
            g.srcc[d] = s0 = s1 = edge;
            break;
          case BM_REFLECT:
            g.flags |= F_REFLECT;
            g.srcc[d] = nrm[d] < 0 ? 2 * imin[d] - bc.indextype[d]
                                   : 2 * (imax[d] - 1) + bc.indextype[d];
            s0 = g.srcc[d] - (g.bmin[d] + g.ext[d] - 1);
            s1 = g.srcc[d] - g.bmin[d];
            break;
          default: break;
          }
          if (m != BM_NONE && m != BM_DIRICHLET &&
              (s0 < dmin[d] || s1 >= dmax[d] || s0 < imin[d] || s1 >= imax[d]))
            return bad("direction %d: a source point lies outside the FAB or the interior "
                       "(FAB narrower than the stencil, or domain narrower than the ghosts)",
                       d);
        }
        if (g.flags & F_REFLECT)
          for (int c = 0; c < bc.ncomp; ++c) {
            int par = 1;
            for (int d = 0; d < 3; ++d)
              if (g.mode[d] == BM_REFLECT) {
                const int v = bc.parity[c][d];
                if (v != 1 && v != -1)
                  return bad("parity of component %d in direction %d is not +-1", c, d);
                par *= v;
              }
            if (par < 0)
              g.negpar |= 1u << c;
          }
        if (g.flags & F_DIRICHLET)
          g.negpar = 0; // a Dirichlet value takes no parity (boundaries_impl.hxx:382-420)
        g.data = data;
        g.np = np;
        g.nx = dmax[0] - dmin[0];
        g.ny = dmax[1] - dmin[1];
        for (int d = 0; d < 3; ++d)
          g.dmin[d] = dmin[d];
        if (!region_in_fab(g))
          return bad("internal error: a region's access leaves its FAB");
        const int64_t n = (int64_t)g.ext[0] * g.ext[1] * g.ext[2];
        if (n > INT32_MAX)
          return bad("a region of more than 2^31 points");
        g.start = npts;
        npts += n;
        bytes += n * bc.ncomp * ((g.flags & F_DIRICHLET) ? 8 : 16);
        out.push_back(g);
      }
  return CX_OK;
}

int grid_for(int64_t npts) {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (npts + kThreads - 1) / kThreads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)nsm * 8));
}

int launch(const Consts &k, const Region *d_regs, const int *d_first, const BoxRegions &own,
           cudaStream_t s) {
  if (k.npts == 0)
    return CX_OK;
  boundary_kernel<<<grid_for(k.npts), kThreads, 0, s>>>(k, d_regs, d_first, own);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char buf[256];
    snprintf(buf, sizeof buf, "boundary launch: %s", cudaGetErrorString(e));
    return record_failure(CX_ECUDA, buf);
  }
  return CX_OK;
}

bool all_periodic(const cx_bc_t &bc) {
  for (int d = 0; d < 3; ++d)
    if (bc.symmetry[0][d] != CX_SYM_PERIODIC && bc.symmetry[1][d] != CX_SYM_PERIODIC)
      return false;
  return true;
}

} // namespace

struct cx_boundary_plan {
  Consts k{};
  Region *d_regs = nullptr;
  int *d_first = nullptr; // chunk of kThreads points -> its first region
  int64_t bytes = 0;
};

extern "C" {

int cx_boundary_box(const cx_bc_t *bc, double *data, const int lo[3], const int hi[3],
                    cx_stream_t stream) {
  if (int e = check_bc(bc))
    return e;
  std::vector<Region> regs;
  int64_t npts = 0, bytes = 0;
  if (int e = add_fab(*bc, data, lo, hi, regs, npts, bytes))
    return e;
  Consts k = make_consts(*bc);
  BoxRegions own{};
  std::copy(regs.begin(), regs.end(), own.r);
  k.nreg = (int)regs.size();
  k.npts = npts;
  return launch(k, nullptr, nullptr, own, (cudaStream_t)stream);
}

int cx_boundary_plan_create(const cx_bc_t *bc, const cx_bc_fab_t *fabs, int nfabs,
                            cx_boundary_plan_t *out) {
  if (!out)
    return bad("null plan pointer");
  *out = nullptr;
  if (int e = check_bc(bc))
    return e;
  if (nfabs < 0 || (nfabs > 0 && !fabs))
    return bad("invalid FAB list");
  std::vector<Region> regs;
  int64_t npts = 0, bytes = 0;
  if (!all_periodic(*bc)) {
    // the domain in the FABs' index type, grown by the ghosts in periodic
    // directions: FABs inside it have nothing to set (driver.cxx:979-994)
    int glo[3], ghi[3];
    for (int d = 0; d < 3; ++d) {
      const bool per = bc->symmetry[0][d] == CX_SYM_PERIODIC || bc->symmetry[1][d] == CX_SYM_PERIODIC;
      glo[d] = bc->domain_lo[d] - (per ? bc->nghost[d] : 0);
      ghi[d] = bc->domain_hi[d] + !bc->indextype[d] + (per ? bc->nghost[d] : 0);
    }
    for (int i = 0; i < nfabs; ++i) {
      const cx_bc_fab_t &f = fabs[i];
      bool inside = true;
      for (int d = 0; d < 3; ++d)
        inside &= f.lo[d] >= glo[d] && f.hi[d] <= ghi[d];
      if (inside)
        continue;
      if (int e = add_fab(*bc, f.data, f.lo, f.hi, regs, npts, bytes)) {
        char buf[320];
        snprintf(buf, sizeof buf, "FAB %d: %s", i, cx_last_error());
        return record_failure(e, buf);
      }
    }
  }
  if (regs.size() > (size_t)INT32_MAX)
    return bad("too many regions");
  cx_boundary_plan *p = new cx_boundary_plan;
  p->k = make_consts(*bc);
  p->k.nreg = (int)regs.size();
  p->k.npts = npts;
  p->bytes = bytes;
  if (!regs.empty()) {
    std::vector<int> first((npts + kThreads - 1) / kThreads);
    size_t a = 0;
    for (size_t c = 0; c < first.size(); ++c) {
      while (a + 1 < regs.size() && regs[a + 1].start <= (int64_t)c * kThreads)
        ++a;
      first[c] = (int)a;
    }
    cudaError_t e = cudaMalloc(&p->d_regs, regs.size() * sizeof(Region));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_regs, regs.data(), regs.size() * sizeof(Region), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMalloc(&p->d_first, first.size() * sizeof(int));
    if (e == cudaSuccess)
      e = cudaMemcpy(p->d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(p->d_regs);
      cudaFree(p->d_first);
      delete p;
      char buf[256];
      snprintf(buf, sizeof buf, "boundary plan upload: %s", cudaGetErrorString(e));
      return record_failure(e == cudaErrorMemoryAllocation ? CX_ENOMEM : CX_ECUDA, buf);
    }
  }
  *out = p;
  return CX_OK;
}

int cx_boundary_plan_execute(cx_boundary_plan_t p, cx_stream_t stream) {
  if (!p)
    return bad("null plan");
  static const BoxRegions none{};
  return launch(p->k, p->d_regs, p->d_first, none, (cudaStream_t)stream);
}

int cx_boundary_plan_stats(cx_boundary_plan_t p, int64_t *npoints, int64_t *bytes) {
  if (!p)
    return bad("null plan");
  if (npoints)
    *npoints = p->k.npts;
  if (bytes)
    *bytes = p->bytes;
  return CX_OK;
}

int cx_boundary_plan_destroy(cx_boundary_plan_t p) {
  if (!p)
    return CX_OK;
  cudaFree(p->d_regs);
  cudaFree(p->d_first);
  delete p;
  return CX_OK;
}

} // extern "C"
