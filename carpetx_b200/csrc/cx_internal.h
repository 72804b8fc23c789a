// Internal host/device descriptors and launcher declarations.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cx_kinds.h"

namespace cxb {

// Per-device caches of kernel attributes and persistent grid sizes:
// cudaFuncSetAttribute and the SM count apply per device, so a process
// driving several GPUs keeps one entry per device.  Devices with an index
// at or above kMaxDevices are served uncached.
constexpr int kMaxDevices = 64;
// The current device if it can be cached, else -1.
inline int cache_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return d >= 0 && d < kMaxDevices ? d : -1;
}

// Streaming kernel: threads per CTA (kStrThreadsSmall for the items of
// boxes with at most kStrSmallUnits column units per x chunk), column units
// per thread, fine y per unit (kStrFineYPerUnit / 2 coarse y centres); at
// most kStrUnitRows rows of units and kStrMaxWidth fine x per item.
constexpr int kStrThreads = 256;
constexpr int kStrThreadsSmall = 128;
constexpr int kStrUnitsPerThread = 1;
constexpr int kStrFineYPerUnit = 4;
constexpr int kStrSmallUnits = kStrThreadsSmall * kStrUnitsPerThread;
constexpr int kStrUnitRows = 32;
constexpr int kStrMaxWidth = 130;

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
  int tbase[3];       // tile origin base: rlo rounded down to even (the
                      // tile origin is even, so fine offset = local & 1)
  int ntile[3];       // streaming kernel: x chunks, unit blocks, z chunks
  int kind[3];        // 1-D stencil kind per direction
  int op;             // operator handle
  int ncomp;
  int zchunk;         // streaming kernel: fine z per item (even)
  int xcw;            // streaming kernel: fine x per x chunk
  int npr;            // streaming kernel: rows of units (kStrFineYPerUnit fine y)
  int upi;            // streaming kernel: units (columns) per item
  int scta;           // streaming kernel: 1 = the 128-thread variant
  double *cbar;       // adjoint: coarse output (P^T fine)
  int at[3];          // adjoint: coarse tile extents in x, y; coarse z per item
  int ant[3];         // adjoint: tiles per direction
};

// One unit of work of the level kernel: a tile of a box, one component.
struct TileRef {
  int box;
  int16_t tx, ty, tz;
  int16_t comp;
};

// Launchers (stream-ordered, no synchronisation).

cudaError_t launch_stream_box(const BoxDesc &b, cudaStream_t s);
// Stencil pair (stream_pairs.h) serving an operator's kinds, -1 if none.
int stream_pair_of(int kx, int ky, int kz);
// Streaming-kernel instantiation serving an operator's kinds:
// 8 x pair + (cx << 2 | cy << 1 | cz), c = 1 for a cell-centred direction;
// -1 if none.  A level's groups add kStrKinds for the 128-thread variant
// (BoxDesc::scta).
int stream_group_of(int kx, int ky, int kz);
constexpr int kStrKinds = 136;            // instantiations per CTA size (8 x kStreamPairs)
constexpr int kStrGroups = 2 * kStrKinds; // level groups: both CTA sizes
// Schedule of a level group's kernel (0 or 1; the 128-thread groups have
// 0): a setting of stream_set_schedule, else the tuned table
// (stream_tuned.h), else the default rule.  stream_maxz: the z-chunk cap of
// an instantiation (fine points, even, 16..128), chosen the same way.
int stream_sched(int group);
int stream_maxz(int kind);
// Settings for the tuner (cx_debug_set_stream_schedule): instantiation kind
// (-1: all), schedule (-1: none), z-chunk cap (0: none); -1 if invalid.
int stream_set_schedule(int kind, int sched, int maxz);
// Level launch of the items of one instantiation with a schedule; d_items
// holds only items of boxes served by that group, sorted by cost;
// d_counter: one int, zero before the launch (the CTAs take items from it).
// after_level: the launch directly follows another level launch of the same
// transfer on s (boxes disjoint), and may start while that one finishes
// (programmatic dependent launch).
cudaError_t launch_stream_level(int group, int sched, const BoxDesc *d_boxes,
                                const TileRef *d_items, int nitems, int grid,
                                int *d_counter, cudaStream_t s, bool after_level);
int stream_level_grid(int group, int sched);
// Fills the streaming-kernel tiling of a box (tbase, ntile, zchunk, xcw,
// npr, upi); min_items > 0 shortens the z chunks of a box launched alone so
// that it spreads over at least that many CTAs where it can.
void stream_tiling(BoxDesc &b, int min_items);

// after_level: as for launch_stream_level (the box's launch directly follows
// another launch of the same level transfer on s); used by the ENO kernel.
cudaError_t launch_point_box(const BoxDesc &b, int per_group,
                             signed char *shifts, unsigned char *fallback,
                             cudaStream_t s, bool after_level = false);
// The per-coarse-cell ENO kernel takes operators whose three directions are
// CC ENO 2 without an active linear fallback (launch_point_box forwards).
bool eno_cell_applies(const BoxDesc &b, int per_group);
// cshift: decisions only, one shift code per coarse cell (the adjoint's).
cudaError_t launch_eno_cell_box(const BoxDesc &b, int per_group, signed char *shifts,
                                unsigned char *fallback, cudaStream_t s,
                                bool after_level = false, unsigned char *cshift = nullptr);
// Adjoint of the ENO-per-cell operators on one box: the decision pass into
// scratch (eno_adjoint_scratch_bytes: one byte per coarse cell with
// children in the region and component block), then a tiled gather.
size_t eno_adjoint_scratch_bytes(const BoxDesc &b, int per_group);
cudaError_t launch_eno_adjoint_box(const BoxDesc &b, int per_group, void *scratch,
                                   double *crse_bar, cudaStream_t s);
// Adjoint of the CCC minmod operator (minmod in all three directions) on one
// box: the forward's choices recomputed per tile, three transposed passes in
// shared memory; no scratch.
bool minmod_cell_applies(const BoxDesc &b);
cudaError_t launch_minmod_adjoint_box(const BoxDesc &b, double *crse_bar, cudaStream_t s);
cudaError_t launch_point_level(const BoxDesc *d_boxes, const TileRef *d_tiles,
                               int ntiles, int per_group, cudaStream_t s);

// Restriction level plans (restrict.cu): size of one device item, host-side
// fill of item n (returns its points x ncomp), one launch over the items of
// one index type (first[c]: the item containing point c * 256).
int64_t restrict_item_bytes();
int64_t restrict_fill_item(void *buf, int n, const double *fine, const int flo[3],
                           const int fhi[3], double *crse, const int clo[3], const int chi[3],
                           const int rlo[3], const int rhi[3], int ncomp, int64_t start);
cudaError_t launch_restrict_level(int indextype, const void *d_items, const int *d_first,
                                  int nitems, int64_t npts, cudaStream_t s);
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
// Adjoint of the limited operators (ENO, minmod, active linear fallback):
// decision pass into stream-ordered scratch, then a gather per coarse point.
cudaError_t launch_point_adjoint_box(const BoxDesc &b, int per_group,
                                     double *crse_bar, cudaStream_t s);
// The same with the caller's scratch of at least
// point_adjoint_scratch_bytes(b, per_group) bytes (0: none needed).
size_t point_adjoint_scratch_bytes(const BoxDesc &b, int per_group);
cudaError_t launch_point_adjoint_box_scratch(const BoxDesc &b, int per_group, double *crse_bar,
                                             void *scratch, cudaStream_t s);
// Adjoint tiling of a box (cbar must be set by the caller); min_items > 0
// shortens the z chunks of a box launched alone so that it spreads over at
// least that many CTAs where it can.
void adjoint_tiling(BoxDesc &b, int min_items);
// Pair index of an operator whose adjoint has a kernel (linear separable),
// else -1.
int adjoint_pair_of(const BoxDesc &b);
// Adjoint-kernel instantiation of such an operator: 8 x pair + centring
// (cx << 2 | cy << 1 | cz); -1 if none.  Below kStrGroups.
int adjoint_group_of(const BoxDesc &b);
int adjoint_level_grid(int group);
// 1 if a bounded wait of the adjoint kernels gave up since the last call
// (and clears the flag), 0 if not, -1 if the flag could not be read.
int adjoint_take_timeout();
// The same for the streaming kernels (their compute threads' waits for a
// plane's copies).
int stream_take_timeout();
int stream_set_wait_limit(long long cycles);
// Sets the adjoint kernels' wait limit on the current device (cycles <= 0:
// the default, about a second); 0 on success, -1 on a CUDA error.
int adjoint_set_wait_limit(long long cycles);
// d_counter, after_level: as for launch_stream_level.
cudaError_t launch_adjoint_level(int group, const BoxDesc *d_boxes,
                                 const TileRef *d_items, int nitems, int grid,
                                 int *d_counter, cudaStream_t s, bool after_level);

} // namespace cxb
