// Adjoint of the cell-centred minmod prolongation (CCC, minmod in all three
// directions), linearised at the coarse input, as three transposed 1-D
// passes on a tile in shared memory (no atomics, deterministic).
//
// The forward is P = Pz Py Px (x pass first, call_stencil_3d), each pass the
// 1-D minmod of impl.hxx:859-877 on the previous pass's output:
//   fine child 2 c + off = v0 + sgn * delta,  sgn = -1 (off 0) / +1 (off 1),
//   delta = (copysign(1/8, dm) + copysign(1/8, dp)) * min(|dm|, |dp|),
//   dm = v0 - v[-1], dp = v[1] - v0.
// Linearised, a line point c makes one of three choices from its own input
// values: ZERO (signs differ: delta = 0), DM (|dm| <= |dp|: delta = dm / 4)
// or DP (delta = dp / 4).  The children's weights are then
//   ZERO: v0;  DM: (1 + sgn/4) v0 - sgn/4 v[-1];  DP: (1 - sgn/4) v0 + sgn/4 v[1],
// so with h0, h1 the cotangents of c's children, S = h0 + h1, d = h1 - h0,
// the transposed pass gathers
//   g(c) = S(c) + s(c) d(c) / 4 - [c + 1 chose DM] d(c + 1) / 4
//          + [c - 1 chose DP] d(c - 1) / 4,    s = +1 (DM), -1 (DP), 0 (ZERO).
// P^T = Px^T Py^T Pz^T, each transposed pass linearised at its own forward
// input: Pz^T at the y pass's output A2, Py^T at the x pass's output A1, Px^T
// at the coarse data.  A CTA takes a tile of T^3 coarse points of the coarse
// box, one component:
//   1. the coarse window (T + 4)^3 around it -> A1 on the children of the
//      tile's coarse x +- 1 and the x choices of the tile's points +- 1 in x;
//   2. A2 (kept in registers down each column) -> the y and z choices;
//   3. fine_bar over the children of the tile +- 1 (region points only; the
//      rest count as 0) -> Pz^T into shared memory;
//   4. Py^T, 5. Px^T -> crse_bar of the tile, stored.
// A1 and A2 are evaluated with the forward's own arithmetic (CcMinmod::ap), so
// every choice is the one the forward made.  Choices at positions no region
// point reads may come from values outside the coarse box (read as 0); they
// only multiply cotangents that are exactly 0.
#include <atomic>

#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

constexpr int MT = 8;            // coarse tile edge
constexpr int MCW = MT + 4;      // coarse window (tile +- 2)
constexpr int MCH = MT + 2;      // choice centres (tile +- 1)
constexpr int MFW = 2 * MCH;     // fine window: children of the choice centres
constexpr int MNT = 256;         // threads per CTA
enum : unsigned char { MM_ZERO = 0, MM_DM = 1, MM_DP = 2 };

struct MinmodAdjShared {
  union { // the forward passes' arrays, then the transposed passes' (43 KB in
           // all, so that five CTAs fit an SM)
    struct {
      double c[MCW * MCW * MCW];  // coarse window [z][y][x]
      double a1[MCW * MCW * MFW]; // A1 [cz][cy][fx]
    } fwd;
    struct {
      double g2[MT * MFW * MFW];  // Pz^T fine_bar [cz][fy][fx]
      double g1[MT * MT * MFW];   // Py^T g2 [cz][cy][fx]
    } bwd;
  } u;
  unsigned char xc[MT * MT * MCH];   // x choices [cz][cy][cx']
  unsigned char yc[MT * MCH * MFW];  // y choices [cz][cy'][fx]
  unsigned char zc[MCH * MFW * MFW]; // z choices [cz'][fy][fx]
};

// The choice of a minmod line point with input values v[-1..1] (the branch
// the forward's delta takes; on |dm| = |dp| the dm branch, as fmin).
__device__ __forceinline__ unsigned char mm_choice(double vm, double v0, double vp) {
  const double dm = fsub(v0, vm), dp = fsub(vp, v0);
  if (copysign(0.125, dm) + copysign(0.125, dp) == 0.0)
    return MM_ZERO;
  return fabs(dm) <= fabs(dp) ? MM_DM : MM_DP;
}

// The transposed pass at centre index m of a line of choices ch (stride 1 in
// the caller's indexing) and child cotangents h (h[2 j], h[2 j + 1] of
// centre j).
__device__ __forceinline__ double mm_gather(const unsigned char *ch, int cs, const double *h,
                                            int hs, int m) {
  const double h0 = h[(2 * m) * hs], h1 = h[(2 * m + 1) * hs];
  double g = h0 + h1;
  const unsigned char c = ch[m * cs];
  if (c != MM_ZERO)
    g += (c == MM_DM ? 0.25 : -0.25) * (h1 - h0);
  if (ch[(m + 1) * cs] == MM_DM)
    g -= 0.25 * (h[(2 * m + 3) * hs] - h[(2 * m + 2) * hs]);
  if (ch[(m - 1) * cs] == MM_DP)
    g += 0.25 * (h[(2 * m - 1) * hs] - h[(2 * m - 2) * hs]);
  return g;
}

__global__ void __launch_bounds__(MNT, 5)
    minmod_adjoint_kernel(const __grid_constant__ BoxDesc b, double *__restrict__ cbar, int ntx,
                          int nty) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MinmodAdjShared &sh = *reinterpret_cast<MinmodAdjShared *>(smem_raw);
  const int tid = threadIdx.x;
  const int comp = blockIdx.y;
  const int tile = blockIdx.x;
  const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
  const int q0x = b.clo[0] + (tile % ntx) * MT, q0y = b.clo[1] + ((tile / ntx) % nty) * MT,
            q0z = b.clo[2] + (tile / (ntx * nty)) * MT;
  const double *crse = b.crse + comp * b.cnp;

  // 1. coarse window: coarse q0 - 2 + (i, j, k)
  for (int e = tid; e < MCW * MCW * MCW; e += MNT) {
    const int i = e % MCW, j = (e / MCW) % MCW, k = e / (MCW * MCW);
    const int x = q0x - 2 + i - b.clo[0], y = q0y - 2 + j - b.clo[1], z = q0z - 2 + k - b.clo[2];
    double v = 0.0;
    if (x >= 0 && x < b.cnx && y >= 0 && y < b.cny && z >= 0 && z < cnz)
      v = crse[x + (int64_t)b.cnx * (y + (int64_t)b.cny * z)];
    sh.u.fwd.c[e] = v;
  }
  __syncthreads();
  // x pass at centres cx' = q0x - 1 + a (a < MCH), every coarse (y, z) of the
  // window; the x choices of the tile's (y, z)
  for (int e = tid; e < MCH * MCW * MCW; e += MNT) {
    const int a = e % MCH, j = (e / MCH) % MCW, k = e / (MCH * MCW);
    const double *v = sh.u.fwd.c + (a + 1) + MCW * (j + MCW * k);
    double *o = sh.u.fwd.a1 + 2 * a + MFW * (j + MCW * k);
    o[0] = CcMinmod::ap<0>(v);
    o[1] = CcMinmod::ap<1>(v);
    if (j >= 2 && j < MT + 2 && k >= 2 && k < MT + 2)
      sh.xc[a + MCH * ((j - 2) + MT * (k - 2))] = mm_choice(v[-1], v[0], v[1]);
  }
  __syncthreads();
  // 2. y pass at centres cy' = q0y - 1 + bb down each fine x column over the
  // window's coarse z: the y choices (the tile's z) and A2, whose z choices
  // at cz' = q0z - 1 + m follow from three consecutive coarse z
  double zr[2][3];
  for (int e = tid; e < MFW * MCH; e += MNT) {
    const int i = e % MFW, bb = e / MFW;
    for (int k = 0; k < MCW; ++k) {
      const double *col = sh.u.fwd.a1 + i + MFW * (bb + 1 + MCW * k);
      double v[3] = {col[-MFW], col[0], col[MFW]};
      const double lo = CcMinmod::ap<0>(v + 1), hi = CcMinmod::ap<1>(v + 1);
      if (k >= 2 && k < MT + 2)
        sh.yc[i + MFW * (bb + MCH * (k - 2))] = mm_choice(v[0], v[1], v[2]);
      zr[0][0] = zr[0][1];
      zr[0][1] = zr[0][2];
      zr[0][2] = lo;
      zr[1][0] = zr[1][1];
      zr[1][1] = zr[1][2];
      zr[1][2] = hi;
      if (k >= 2) {
        const int m = k - 2; // centre cz' = q0z - 2 + (k - 1)
        sh.zc[i + MFW * (2 * bb + MFW * m)] = mm_choice(zr[0][0], zr[0][1], zr[0][2]);
        sh.zc[i + MFW * (2 * bb + 1 + MFW * m)] = mm_choice(zr[1][0], zr[1][1], zr[1][2]);
      }
    }
  }
  __syncthreads(); // the coarse window and A1 are dead: g2 takes their space
  // 3. Pz^T: per fine (x, y) column of the window, the children of the z
  // centres q0z - 1 + m (fine z 2 (q0z - 1) + kk)
  const int64_t fplane = (int64_t)b.fnx * b.fny;
  const double *fb = b.fine + comp * b.fnp;
  const int fx0 = 2 * (q0x - 1), fy0 = 2 * (q0y - 1), fz0 = 2 * (q0z - 1);
  for (int e = tid; e < MFW * MFW; e += MNT) {
    const int i = e % MFW, jj = e / MFW;
    const int fx = fx0 + i, fy = fy0 + jj;
    double h[MFW];
    const bool col = fx >= b.rlo[0] && fx <= b.rhi[0] && fy >= b.rlo[1] && fy <= b.rhi[1];
    const double *p = fb + (fx - b.flo[0]) + (int64_t)b.fnx * (fy - b.flo[1]);
#pragma unroll
    for (int kk = 0; kk < MFW; ++kk) {
      const int fz = fz0 + kk;
      h[kk] = col && fz >= b.rlo[2] && fz <= b.rhi[2] ? p[fplane * (fz - b.flo[2])] : 0.0;
    }
    const unsigned char *ch = sh.zc + i + MFW * jj;
#pragma unroll
    for (int n = 0; n < MT; ++n)
      sh.u.bwd.g2[i + MFW * (jj + MFW * n)] = mm_gather(ch, MFW * MFW, h, 1, n + 1);
  }
  __syncthreads();
  // 4. Py^T: g1 at (fx, cy = q0y + ny, cz = q0z + n)
  for (int e = tid; e < MFW * MT * MT; e += MNT) {
    const int i = e % MFW, ny = (e / MFW) % MT, n = e / (MFW * MT);
    sh.u.bwd.g1[e] = mm_gather(sh.yc + i + MFW * MCH * n, MFW, sh.u.bwd.g2 + i + MFW * MFW * n, MFW,
                         ny + 1);
  }
  __syncthreads();
  // 5. Px^T: crse_bar of the tile
  for (int e = tid; e < MT * MT * MT; e += MNT) {
    const int nx = e % MT, ny = (e / MT) % MT, n = e / (MT * MT);
    const int x = q0x + nx - b.clo[0], y = q0y + ny - b.clo[1], z = q0z + n - b.clo[2];
    if (x >= b.cnx || y >= b.cny || z >= cnz)
      continue;
    const double g = mm_gather(sh.xc + MCH * (ny + MT * n), 1, sh.u.bwd.g1 + MFW * (ny + MT * n), 1,
                               nx + 1);
    cbar[comp * b.cnp + x + (int64_t)b.cnx * (y + (int64_t)b.cny * z)] = g;
  }
}

std::atomic<bool> g_mm_attr_set[kMaxDevices];

} // namespace

bool minmod_cell_applies(const BoxDesc &b) {
  return b.kind[0] == K_CC_MINMOD1 && b.kind[1] == K_CC_MINMOD1 && b.kind[2] == K_CC_MINMOD1;
}

cudaError_t launch_minmod_adjoint_box(const BoxDesc &b, double *crse_bar, cudaStream_t s) {
  if (b.ncomp <= 0 || b.cnp <= 0)
    return cudaSuccess;
  for (int d = 0; d < 3; ++d)
    if (b.rhi[d] < b.rlo[d]) // nothing reads the coarse box: zero
      return cudaMemsetAsync(crse_bar, 0, sizeof(double) * b.cnp * b.ncomp, s);
  const int dev = cache_device();
  if (dev < 0 || !g_mm_attr_set[dev].load()) {
    const cudaError_t e = cudaFuncSetAttribute(minmod_adjoint_kernel,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)sizeof(MinmodAdjShared));
    if (e != cudaSuccess)
      return e;
    if (dev >= 0)
      g_mm_attr_set[dev].store(true);
  }
  const int cnz = (int)(b.cnp / ((int64_t)b.cnx * b.cny));
  const int ntx = (b.cnx + MT - 1) / MT, nty = (b.cny + MT - 1) / MT, ntz = (cnz + MT - 1) / MT;
  const int64_t ntiles = (int64_t)ntx * nty * ntz;
  if (ntiles > INT32_MAX || b.ncomp > 65535)
    return cudaErrorInvalidValue;
  minmod_adjoint_kernel<<<dim3((unsigned)ntiles, (unsigned)b.ncomp), MNT,
                          sizeof(MinmodAdjShared), s>>>(b, crse_bar, ntx, nty);
  return cudaGetLastError();
}

} // namespace cxb
