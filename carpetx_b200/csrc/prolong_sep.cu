// Separable prolongation kernels (all linear families and minmod).
//
// A CTA transfers a fine tile of kSepTX x kSepTY x kSepTZ points of one
// component:
//   load   the coarse window of the tile into shared memory (S0) with
//          asynchronous 8-byte copies, zero-filled outside the coarse points
//          the operator reads; the next tile's window is prefetched into the
//          second S0 buffer while the current tile computes;
//   x pass S1[cz][cy][fx] = interp_x(S0 row), 8 fine outputs per thread from
//          a register window of the coarse row;
//   y pass S2[cz][fy][fx] = interp_y(S1 column), a whole fine column per
//          thread from a register window;
//   z pass fine[fz][fy][fx] = interp_z(S2 column), written straight to global
//          memory with streaming stores (consecutive threads = consecutive x).
// This is call_stencil_3d (CarpetX/src/prolongate_3d_rf2_impl.hxx:1206-1216)
// evaluated once per distinct 1-D result instead of once per fine point; the
// arithmetic per result is the reference's, so values are bit-identical.
// Each pass dispatches on its direction's stencil kind at run time (uniform
// per CTA), so one kernel serves every centering and order of a level.
#include <cstdio>

#include "cx_internal.h"
#include "cx_stencils.cuh"

namespace cxb {
namespace {

constexpr int TX = kSepTX, TY = kSepTY, TZ = kSepTZ, NT = kSepThreads;
constexpr int P1 = TX + 1; // S1 row pitch (odd: conflict-free x-pass stores)
static_assert(TX * TY == NT, "z pass maps one thread per (fx, fy)");
static_assert(TX == 32, "y/z passes map lanes to fine x");

__device__ __forceinline__ void cp_async8(double *sdst, const double *gsrc, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait1() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

struct TileGeom {
  int o[3];  // fine origin of the tile (even)
  int c0[3]; // coarse window origin
  int W[3];  // coarse window extent
  int P0;    // S0 row pitch
  int comp;
};

__device__ __forceinline__ void make_geom(const BoxDesc &b, int tx, int ty, int tz, int comp,
                                          TileGeom &g) {
  const int t[3] = {tx, ty, tz};
  const int T[3] = {TX, TY, TZ};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int k = b.kind[d];
    g.o[d] = b.tbase[d] + t[d] * T[d];
    g.c0[d] = g.o[d] / 2 + sep_rlo(k); // o even: exact halving
    g.W[d] = T[d] / 2 + sep_rhi(k) - sep_rlo(k);
  }
  g.P0 = g.W[0] | 1;
  g.comp = comp;
}

// Stage the coarse window of tile g into S0 (asynchronous; caller commits).
__device__ __forceinline__ void load_window(const BoxDesc &b, const TileGeom &g, double *S0) {
  const double *base = b.crse + g.comp * b.cnp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nrows = g.W[1] * g.W[2];
  for (int row = warp; row < nrows; row += NT / 32) {
    const int cy = row % g.W[1], cz = row / g.W[1];
    const int gy = g.c0[1] + cy, gz = g.c0[2] + cz;
    const bool rowok = gy >= b.nlo[1] && gy <= b.nhi[1] && gz >= b.nlo[2] && gz <= b.nhi[2];
    const int64_t rowoff =
        ((int64_t)(gz - b.clo[2]) * b.cny + (gy - b.clo[1])) * b.cnx - b.clo[0];
    for (int x = lane; x < g.W[0]; x += 32) {
      const int gx = g.c0[0] + x;
      const bool ok = rowok && gx >= b.nlo[0] && gx <= b.nhi[0];
      cp_async8(S0 + row * g.P0 + x, ok ? base + rowoff + gx : base, ok ? 8 : 0);
    }
  }
}

// x pass: 8 fine outputs (4 coarse cells) per task; threads = NSEG segments
// x RPI rows, consecutive lanes on consecutive rows (odd pitches: no bank
// conflicts for the 8-byte accesses).
template <class K> __device__ __forceinline__ void xpass(const double *S0, int P0, int nrows, double *S1) {
  constexpr int XB = 8, NSEG = TX / XB, RPI = NT / NSEG;
  constexpr int WIN = XB / 2 + K::RHI - K::RLO;
  static_assert(K::RLO == sep_rlo(K::KIND) && K::RHI == sep_rhi(K::KIND), "window mismatch");
  const int seg = threadIdx.x / RPI;
  for (int row = threadIdx.x % RPI; row < nrows; row += RPI) {
    const double *src = S0 + row * P0 + seg * (XB / 2);
    double v[WIN];
#pragma unroll
    for (int i = 0; i < WIN; ++i)
      v[i] = src[i];
    double *dst = S1 + row * P1 + seg * XB;
#pragma unroll
    for (int f = 0; f < XB; ++f) {
      if (f & 1)
        dst[f] = K::template ap<1>(v + f / 2 - K::RLO);
      else
        dst[f] = K::template ap<0>(v + f / 2 - K::RLO);
    }
  }
}

// y pass: one (fx, cz) column per task, all TY fine y from a register window.
template <class K> __device__ __forceinline__ void ypass(const double *S1, int Wz, double *S2) {
  constexpr int WIN = TY / 2 + K::RHI - K::RLO; // == W[1]
  const int fx = threadIdx.x % TX;
  for (int cz = threadIdx.x / TX; cz < Wz; cz += NT / TX) {
    double v[WIN];
#pragma unroll
    for (int j = 0; j < WIN; ++j)
      v[j] = S1[(cz * WIN + j) * P1 + fx];
#pragma unroll
    for (int fy = 0; fy < TY; ++fy) {
      double r;
      if (fy & 1)
        r = K::template ap<1>(v + fy / 2 - K::RLO);
      else
        r = K::template ap<0>(v + fy / 2 - K::RLO);
      S2[(cz * TY + fy) * TX + fx] = r;
    }
  }
}

// z pass: one (fx, fy) column per thread; results go straight to the fine FAB.
template <class K>
__device__ __forceinline__ void zpass(const double *S2, const BoxDesc &b, const TileGeom &g) {
  constexpr int WIN = TZ / 2 + K::RHI - K::RLO; // == W[2]
  const int fx = threadIdx.x % TX, fy = threadIdx.x / TX;
  double v[WIN];
#pragma unroll
  for (int k = 0; k < WIN; ++k)
    v[k] = S2[(k * TY + fy) * TX + fx];
  const int gx = g.o[0] + fx, gy = g.o[1] + fy;
  if (gx < b.rlo[0] || gx > b.rhi[0] || gy < b.rlo[1] || gy > b.rhi[1])
    return;
  const int64_t plane = (int64_t)b.fnx * b.fny;
  double *out = b.fine + g.comp * b.fnp + (gx - b.flo[0]) +
                (int64_t)b.fnx * (gy - b.flo[1]) + plane * (g.o[2] - b.flo[2]);
#pragma unroll
  for (int fz = 0; fz < TZ; ++fz) {
    double r;
    if (fz & 1)
      r = K::template ap<1>(v + fz / 2 - K::RLO);
    else
      r = K::template ap<0>(v + fz / 2 - K::RLO);
    const int gz = g.o[2] + fz;
    if (gz >= b.rlo[2] && gz <= b.rhi[2])
      __stcs(out + fz * plane, r);
  }
}

__device__ __forceinline__ void sep_tile(const BoxDesc &b, const TileGeom &g, const double *S0,
                                         double *S1, double *S2) {
  CXB_DISPATCH_SEPARABLE(b.kind[0], xpass, S0, g.P0, g.W[1] * g.W[2], S1);
  __syncthreads();
  CXB_DISPATCH_SEPARABLE(b.kind[1], ypass, S1, g.W[2], S2);
  __syncthreads();
  CXB_DISPATCH_SEPARABLE(b.kind[2], zpass, S2, b, g);
}

__device__ __forceinline__ void decode_task(const BoxDesc &b, int task, TileGeom &g) {
  const int tx = task % b.ntile[0];
  int r = task / b.ntile[0];
  const int ty = r % b.ntile[1];
  r /= b.ntile[1];
  const int tz = r % b.ntile[2];
  const int comp = r / b.ntile[2];
  make_geom(b, tx, ty, tz, comp, g);
}

// One box, all its tiles and components: CTA-strided over tasks with a
// one-tile prefetch.
__global__ void __launch_bounds__(NT) sep_box_kernel(const BoxDesc b, int ntasks, int s0, int s1) {
  extern __shared__ double smem[];
  double *const S0a = smem, *const S0b = smem + s0;
  double *S1 = smem + 2 * s0, *S2 = S1 + s1;
  int task = blockIdx.x;
  if (task >= ntasks)
    return;
  TileGeom g;
  decode_task(b, task, g);
  load_window(b, g, S0a);
  cp_async_commit();
  for (int it = 0;; ++it) {
    const int next = task + gridDim.x;
    TileGeom gn;
    if (next < ntasks) {
      decode_task(b, next, gn);
      load_window(b, gn, (it & 1) ? S0a : S0b);
    }
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    sep_tile(b, g, (it & 1) ? S0b : S0a, S1, S2);
    if (next >= ntasks)
      break;
    task = next;
    g = gn;
  }
}

// A whole level: tiles of many boxes from a device work list, fetched
// dynamically (persistent CTAs), one-tile prefetch.
__global__ void __launch_bounds__(NT)
    sep_level_kernel(const BoxDesc *__restrict__ boxes, const TileRef *__restrict__ tiles,
                     int ntiles, int *counter, int s0, int s1) {
  extern __shared__ double smem[];
  __shared__ int next_s[2];
  double *const S0a = smem, *const S0b = smem + s0;
  double *S1 = smem + 2 * s0, *S2 = S1 + s1;
  if (threadIdx.x == 0)
    next_s[0] = atomicAdd(counter, 1);
  __syncthreads();
  int cur = next_s[0];
  if (cur >= ntiles)
    return;
  TileRef tr = tiles[cur];
  TileGeom g;
  make_geom(boxes[tr.box], tr.tx, tr.ty, tr.tz, tr.comp, g);
  load_window(boxes[tr.box], g, S0a);
  cp_async_commit();
  for (int it = 0;; ++it) {
    if (threadIdx.x == 0)
      next_s[(it + 1) & 1] = atomicAdd(counter, 1);
    __syncthreads();
    const int nxt = next_s[(it + 1) & 1];
    TileRef tn;
    TileGeom gn;
    if (nxt < ntiles) {
      tn = tiles[nxt];
      make_geom(boxes[tn.box], tn.tx, tn.ty, tn.tz, tn.comp, gn);
      load_window(boxes[tn.box], gn, (it & 1) ? S0a : S0b);
    }
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    sep_tile(boxes[tr.box], g, (it & 1) ? S0b : S0a, S1, S2);
    if (nxt >= ntiles)
      break;
    tr = tn;
    g = gn;
  }
}

int g_num_sms = 0;

int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(sep_box_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(sep_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  }
  return g_num_sms;
}

} // namespace

SepSmem sep_smem_for(const int kind[3]) {
  SepSmem m;
  const int T[3] = {TX, TY, TZ};
  for (int d = 0; d < 3; ++d)
    m.W[d] = T[d] / 2 + sep_rhi(kind[d]) - sep_rlo(kind[d]);
  m.P0 = m.W[0] | 1;
  m.s0 = m.P0 * m.W[1] * m.W[2];
  m.s1 = P1 * m.W[1] * m.W[2];
  m.s2 = TX * TY * m.W[2];
  return m;
}

cudaError_t launch_sep_box(const BoxDesc &b, cudaStream_t s) {
  const int nsm = num_sms();
  const SepSmem m = sep_smem_for(b.kind);
  const int64_t ntasks64 = (int64_t)b.ntile[0] * b.ntile[1] * b.ntile[2] * b.ncomp;
  if (ntasks64 <= 0)
    return cudaSuccess;
  if (ntasks64 > INT32_MAX)
    return cudaErrorInvalidValue;
  const int ntasks = (int)ntasks64;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sep_box_kernel, NT, m.bytes());
  if (per_sm < 1)
    per_sm = 1;
  const int grid = ntasks < nsm * per_sm ? ntasks : nsm * per_sm;
  sep_box_kernel<<<grid, NT, m.bytes(), s>>>(b, ntasks, m.s0, m.s1);
  return cudaGetLastError();
}

int sep_level_grid(size_t smem_bytes) {
  const int nsm = num_sms();
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sep_level_kernel, NT, smem_bytes);
  if (per_sm < 1)
    per_sm = 1;
  return nsm * per_sm;
}

cudaError_t launch_sep_level(const BoxDesc *d_boxes, const TileRef *d_tiles, int ntiles,
                             int *d_counter, int s0max, int s1max, size_t smem_bytes, int grid,
                             cudaStream_t s) {
  if (ntiles <= 0)
    return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(int), s);
  if (e != cudaSuccess)
    return e;
  sep_level_kernel<<<grid < ntiles ? grid : ntiles, NT, smem_bytes, s>>>(d_boxes, d_tiles, ntiles,
                                                                          d_counter, s0max, s1max);
  return cudaGetLastError();
}

} // namespace cxb
