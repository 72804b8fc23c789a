// Restriction kernels: AMReX's average_down family as CarpetX's Restrict calls
// it (CarpetX/src/schedule.cxx:2793-2815), and its transpose.
//
// Per coarse point c of the region: vertex-centred directions take fine point
// 2c, cell-centred directions the children 2c and 2c+1; the children are
// summed z-outer / x-inner from 0 and scaled by 1/(number of children)
// (average_down, _faces, _edges); fully vertex-centred data is injected
// (average_down_nodal).  One thread per coarse point, consecutive threads on
// consecutive coarse x, so a warp reads contiguous fine rows.
#include <algorithm>

#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

struct RBox {
  const double *src;
  double *dst;
  int64_t fnp, cnp;
  int flo[3], fnx, fny;
  int clo[3], cnx, cny;
  int rlo[3], rnx, rny;
  int64_t rnp;
};

// Coarse point (i, j, k) of component comp: the mean of its children (the
// fine point 2c itself for fully vertex-centred data).
template <int IT>
__device__ __forceinline__ void restrict_point(const RBox &r, int comp, int i, int j, int k) {
  constexpr int CX = (IT >> 2) & 1, CY = (IT >> 1) & 1, CZ = IT & 1;
  constexpr double SCALE = 1.0 / ((1 + CX) * (1 + CY) * (1 + CZ));
  const double *f = r.src + comp * r.fnp;
  const int64_t fplane = (int64_t)r.fnx * r.fny;
  const int64_t f0 =
      (2 * i - r.flo[0]) + (int64_t)r.fnx * (2 * j - r.flo[1]) + fplane * (2 * k - r.flo[2]);
  double res;
  if constexpr (IT == 0) {
    res = __ldcs(f + f0);
  } else {
    double s = 0.0;
#pragma unroll
    for (int kr = 0; kr <= CZ; ++kr)
#pragma unroll
      for (int jr = 0; jr <= CY; ++jr)
#pragma unroll
        for (int ir = 0; ir <= CX; ++ir)
          s = fadd(s, __ldcs(f + f0 + ir + (int64_t)r.fnx * jr + fplane * kr));
    res = fmul(s, SCALE);
  }
  r.dst[comp * r.cnp + (i - r.clo[0]) + (int64_t)r.cnx * ((j - r.clo[1]) + (int64_t)r.cny * (k - r.clo[2]))] =
      res;
}

template <int IT> __global__ void __launch_bounds__(256) restrict_kernel(const RBox r) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= r.rnp)
    return;
  const int i = r.rlo[0] + (int)(idx % r.rnx);
  const int j = r.rlo[1] + (int)((idx / r.rnx) % r.rny);
  const int k = r.rlo[2] + (int)(idx / ((int64_t)r.rnx * r.rny));
  restrict_point<IT>(r, blockIdx.y, i, j, k);
}

// A level's boxes of one index type: a flat range over (box, component,
// region point), boxes found by binary search on their first point.
struct RItem {
  RBox r;
  int64_t start; // first point of the box in the launch's range
  int ncomp;
};

// first[c]: the item containing point c * 256 (a thread scans forward from
// it).  An item's points x components fit in 32 bits (checked on the host).
template <int IT>
__global__ void __launch_bounds__(256)
    restrict_level_kernel(const RItem *__restrict__ items, const int *__restrict__ first,
                          int nitems, int64_t npts) {
  const int64_t nchunks = (npts + 255) / 256;
  for (int64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
    const int64_t p = chunk * 256 + threadIdx.x;
    if (p >= npts)
      continue;
    int a = first[chunk];
    while (a + 1 < nitems && items[a + 1].start <= p)
      ++a;
    const RBox &r = items[a].r;
    const int l = (int)(p - items[a].start);
    const int rnp = (int)r.rnp;
    const int comp = l / rnp;
    const int idx = l - comp * rnp;
    const int i = r.rlo[0] + idx % r.rnx;
    const int jk = idx / r.rnx;
    const int j = r.rlo[1] + jk % r.rny;
    const int k = r.rlo[2] + jk / r.rny;
    restrict_point<IT>(r, comp, i, j, k);
  }
}

// Transpose: every child receives the coarse cotangent times the scale (the
// children of distinct coarse points are distinct: no accumulation needed).
template <int IT> __global__ void __launch_bounds__(256) restrict_adjoint_kernel(const RBox r) {
  constexpr int CX = (IT >> 2) & 1, CY = (IT >> 1) & 1, CZ = IT & 1;
  constexpr double SCALE = 1.0 / ((1 + CX) * (1 + CY) * (1 + CZ));
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= r.rnp)
    return;
  const int comp = blockIdx.y;
  const int i = r.rlo[0] + (int)(idx % r.rnx);
  const int j = r.rlo[1] + (int)((idx / r.rnx) % r.rny);
  const int k = r.rlo[2] + (int)(idx / ((int64_t)r.rnx * r.rny));
  const double g = r.src[comp * r.cnp + (i - r.clo[0]) +
                         (int64_t)r.cnx * ((j - r.clo[1]) + (int64_t)r.cny * (k - r.clo[2]))];
  const double v = IT == 0 ? g : fmul(g, SCALE);
  double *f = r.dst + comp * r.fnp;
  const int64_t fplane = (int64_t)r.fnx * r.fny;
  const int64_t f0 =
      (2 * i - r.flo[0]) + (int64_t)r.fnx * (2 * j - r.flo[1]) + fplane * (2 * k - r.flo[2]);
#pragma unroll
  for (int kr = 0; kr <= CZ; ++kr)
#pragma unroll
    for (int jr = 0; jr <= CY; ++jr)
#pragma unroll
      for (int ir = 0; ir <= CX; ++ir)
        f[f0 + ir + (int64_t)r.fnx * jr + fplane * kr] = v;
}

RBox make_rbox(const double *src, double *dst, const int flo[3], const int fhi[3], const int clo[3],
               const int chi[3], const int rlo[3], const int rhi[3]) {
  RBox r;
  r.src = src;
  r.dst = dst;
  for (int d = 0; d < 3; ++d) {
    r.flo[d] = flo[d];
    r.clo[d] = clo[d];
    r.rlo[d] = rlo[d];
  }
  r.fnx = fhi[0] - flo[0] + 1;
  r.fny = fhi[1] - flo[1] + 1;
  r.fnp = (int64_t)r.fnx * r.fny * (fhi[2] - flo[2] + 1);
  r.cnx = chi[0] - clo[0] + 1;
  r.cny = chi[1] - clo[1] + 1;
  r.cnp = (int64_t)r.cnx * r.cny * (chi[2] - clo[2] + 1);
  r.rnx = rhi[0] - rlo[0] + 1;
  r.rny = rhi[1] - rlo[1] + 1;
  r.rnp = (int64_t)r.rnx * r.rny * (rhi[2] - rlo[2] + 1);
  return r;
}

template <template <int> class Launch, class... A> cudaError_t by_indextype(int it, A... a) {
  switch (it) {
  case 0: return Launch<0>::go(a...);
  case 1: return Launch<1>::go(a...);
  case 2: return Launch<2>::go(a...);
  case 3: return Launch<3>::go(a...);
  case 4: return Launch<4>::go(a...);
  case 5: return Launch<5>::go(a...);
  case 6: return Launch<6>::go(a...);
  case 7: return Launch<7>::go(a...);
  default: return cudaErrorInvalidValue;
  }
}

template <int IT> struct FwdLaunch {
  static cudaError_t go(RBox r, int ncomp, cudaStream_t s) {
    dim3 grid((unsigned)((r.rnp + 255) / 256), ncomp);
    restrict_kernel<IT><<<grid, 256, 0, s>>>(r);
    return cudaGetLastError();
  }
};
template <int IT> struct AdjLaunch {
  static cudaError_t go(RBox r, int ncomp, cudaStream_t s) {
    dim3 grid((unsigned)((r.rnp + 255) / 256), ncomp);
    restrict_adjoint_kernel<IT><<<grid, 256, 0, s>>>(r);
    return cudaGetLastError();
  }
};

template <int IT> struct LevelLaunch {
  static cudaError_t go(const void *items, const int *first, int nitems, int64_t npts,
                        cudaStream_t s) {
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (npts + 255) / 256;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)nsm * 8));
    restrict_level_kernel<IT><<<grid, 256, 0, s>>>((const RItem *)items, first, nitems, npts);
    return cudaGetLastError();
  }
};

} // namespace

// Restriction level plans: the boxes grouped by index type, one device item
// list per group, one launch per group.
int64_t restrict_item_bytes() { return (int64_t)sizeof(RItem); }

// Fills item n of a host buffer of RItem; returns the box's points x ncomp.
int64_t restrict_fill_item(void *buf, int n, const double *fine, const int flo[3],
                           const int fhi[3], double *crse, const int clo[3], const int chi[3],
                           const int rlo[3], const int rhi[3], int ncomp, int64_t start) {
  RItem &it = ((RItem *)buf)[n];
  it.r = make_rbox(fine, crse, flo, fhi, clo, chi, rlo, rhi);
  it.start = start;
  it.ncomp = ncomp;
  return it.r.rnp * ncomp;
}

cudaError_t launch_restrict_level(int indextype, const void *d_items, const int *d_first,
                                  int nitems, int64_t npts, cudaStream_t s) {
  if (nitems <= 0 || npts <= 0)
    return cudaSuccess;
  return by_indextype<LevelLaunch>(indextype, d_items, d_first, nitems, npts, s);
}

cudaError_t launch_restrict_box(int indextype, const double *fine, const int flo[3], const int fhi[3],
                                double *crse, const int clo[3], const int chi[3], const int rlo[3],
                                const int rhi[3], int ncomp, cudaStream_t s) {
  RBox r = make_rbox(fine, crse, flo, fhi, clo, chi, rlo, rhi);
  if (r.rnp <= 0 || ncomp <= 0)
    return cudaSuccess;
  return by_indextype<FwdLaunch>(indextype, r, ncomp, s);
}

cudaError_t launch_restrict_adjoint_box(int indextype, const double *crse_bar, const int clo[3],
                                        const int chi[3], double *fine_bar, const int flo[3],
                                        const int fhi[3], const int rlo[3], const int rhi[3],
                                        int ncomp, cudaStream_t s) {
  RBox r = make_rbox(crse_bar, fine_bar, flo, fhi, clo, chi, rlo, rhi);
  cudaError_t e = cudaMemsetAsync(fine_bar, 0, sizeof(double) * r.fnp * ncomp, s);
  if (e != cudaSuccess || r.rnp <= 0 || ncomp <= 0)
    return e;
  return by_indextype<AdjLaunch>(indextype, r, ncomp, s);
}

} // namespace cxb
