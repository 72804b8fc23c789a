// Internal host/device descriptors and launcher declarations.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cx_kinds.h"

namespace cxb {

// Fine tile of the separable kernel (fine points per direction).  The tile
// origin is even in every direction, so fine offset = local index & 1.
constexpr int kSepTX = 32, kSepTY = 8, kSepTZ = 8;
constexpr int kSepThreads = 256;

// One box of a transfer as the kernels see it.  Coordinates are AMReX index
// space; strides in elements.
struct BoxDesc {
  const double *crse;
  double *fine;
  int64_t cnp, fnp;   // component strides
  int clo[3];         // coarse FAB lo
  int cnx, cny;       // coarse FAB extents in x, y
  int flo[3];         // fine FAB lo
  int fnx, fny;       // fine FAB extents in x, y
  int rlo[3], rhi[3]; // fine region (inclusive)
  int nlo[3], nhi[3]; // coarse points the operator reads (inclusive)
  int tbase[3];       // tile origin base: rlo rounded down to even
  int ntile[3];       // tiles per direction
  int kind[3];        // 1-D stencil kind per direction
  int op;             // operator handle
  int ncomp;
};

// One unit of work of the level kernel: a tile of a box, one component.
struct TileRef {
  int box;
  int16_t tx, ty, tz;
  int16_t comp;
};

// Dynamic shared memory of the separable kernel for one box's kinds.
struct SepSmem {
  int W[3];  // coarse window per direction
  int P0;    // S0 row pitch (odd)
  int s0, s1, s2; // sizes (doubles) of S0 (one buffer), S1, S2
  size_t bytes() const { return sizeof(double) * (size_t)(2 * s0 + s1 + s2); }
};

SepSmem sep_smem_for(const int kind[3]);

// Launchers (stream-ordered, no synchronisation).
cudaError_t launch_sep_box(const BoxDesc &b, cudaStream_t s);
cudaError_t launch_sep_level(const BoxDesc *d_boxes, const TileRef *d_tiles,
                             int ntiles, int *d_counter, int s0max, int s1max,
                             size_t smem_bytes, int grid, cudaStream_t s);
int sep_level_grid(size_t smem_bytes);

cudaError_t launch_point_box(const BoxDesc &b, int per_group,
                             signed char *shifts, unsigned char *fallback,
                             cudaStream_t s);
cudaError_t launch_point_level(const BoxDesc *d_boxes, const TileRef *d_tiles,
                               int ntiles, int per_group, cudaStream_t s);

cudaError_t launch_restrict_box(int indextype, const double *fine,
                                const int flo[3], const int fhi[3],
                                double *crse, const int clo[3],
                                const int chi[3], const int rlo[3],
                                const int rhi[3], int ncomp, cudaStream_t s);
cudaError_t launch_restrict_adjoint_box(int indextype, const double *crse_bar,
                                        const int clo[3], const int chi[3],
                                        double *fine_bar, const int flo[3],
                                        const int fhi[3], const int rlo[3],
                                        const int rhi[3], int ncomp,
                                        cudaStream_t s);
cudaError_t launch_prolong_adjoint_box(const BoxDesc &b, int per_group,
                                       double *crse_bar, cudaStream_t s);

} // namespace cxb
