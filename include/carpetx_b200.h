/* carpetx_b200 -- B200 (sm_100a) implementation of CarpetX's refinement-factor-2
 * inter-level transfer operators: the prolongation family of
 * CarpetX/src/prolongate_3d_rf2* and the restriction CarpetX performs through
 * AMReX's average_down family.
 *
 * C ABI: plain pointers, sizes and status codes; no C++ or torch types.  Every
 * entry point returns CX_OK (0) or a CX_E* status and never aborts; the C++
 * amrex::Interpolater shim (carpetx_b200/host/prolongate_3d_rf2_b200.hxx) maps
 * a non-zero status to CCTK_VERROR, which is the reference's behaviour for
 * unknown operators (CarpetX/src/driver.cxx:621-625) and failed asserts.
 *
 * Data layout, as amrex::FArrayBox: a box is the inclusive index range
 * [lo, hi] per direction; the ncomp components of a box are stored one after
 * the other, each Fortran ordered (x fastest), component stride = number of
 * points of the box.  All values are FP64.  Data pointers are DEVICE pointers
 * unless stated otherwise; work is enqueued on `stream` and returns without
 * synchronising, as the reference's GPU path does (impl.hxx:1685-1688).
 *
 * Results equal the reference operators compiled for the host as FP64 values:
 * every stencil is evaluated with the reference's association order and
 * separately rounded products and sums (no FMA contraction).  The separable
 * operators skip the reference's initial "0 +" and its products by a
 * coefficient of exactly 1, which are exact; the only bit pattern that can
 * differ is the sign of a result that is exactly zero (-0 where the
 * reference gives +0). */
#ifndef CARPETX_B200_H
#define CARPETX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *cx_stream_t; /* a cudaStream_t; NULL = default */

/* Opaque operator handle (value semantics; equal handles = same operator). */
typedef int32_t cx_op_t;

enum {
  CX_OK = 0,
  CX_EINVAL = 1,       /* bad argument: box, region, ncomp, null pointer */
  CX_EUNSUPPORTED = 2, /* unknown prolongation type / order / indextype */
  CX_ECUDA = 3,        /* a CUDA call failed (message: cx_last_error) */
  CX_ETIMEOUT = 4,     /* a bounded device wait gave up */
  CX_ENOMEM = 5,       /* scratch or plan allocation failed */
  CX_ENODEVICE = 6     /* no usable CUDA device */
};

/* Waits for all work on the current device; CX_ETIMEOUT if a kernel's
 * bounded wait (on its own asynchronous copies) gave up since the last call,
 * whose results are then not valid (the flag is cleared), CX_ECUDA on a CUDA
 * error, CX_OK otherwise.  Kernels never wait without a bound. */
int cx_check_device(void);

/* Sets, on the current device, how many SM clock cycles a kernel's bounded
 * wait on its own asynchronous copies polls before it gives up; cycles < 0
 * restores the default (2^31, about a second), cycles = 0 makes every such
 * wait give up at once.  For tests of the give-up path: the kernels then
 * return early, after letting every copy still in flight into their shared
 * memory land (bounded by the default), and cx_check_device reports
 * CX_ETIMEOUT.  Call it with the device idle.  No counterpart in the
 * reference (its kernels never wait). */
int cx_debug_set_wait_limit(long long cycles);

/* Tuning entry points (no counterpart in the reference: its kernels have
 * no schedules).  The separable operators run on one streaming-kernel
 * instantiation per stencil pair and centring; cx_debug_stream_kind
 * returns an operator's instantiation index (0..135; -1 for an operator
 * the streaming kernels do not serve, e.g. ENO).  Each instantiation has a
 * schedule (0: two CTAs per SM; 1: three CTAs per SM with a smaller loop
 * body) and a cap on the fine z points of a work item (even, 16..128),
 * taken from the tuned table the library was built with (written by
 * carpetx_b200/tune.py) unless cx_debug_set_stream_schedule sets them for
 * this process: kind -1 sets every instantiation, schedule -1 and cap 0
 * restore the table.  Plans take the setting in force when they are
 * created; results do not depend on it. */
int cx_debug_stream_kind(cx_op_t op);
int cx_debug_set_stream_schedule(int kind, int sched, int maxz);

/* Human-readable name of a status code. */
const char *cx_status_string(int status);
/* Text of the most recent failure on this thread ("" if none). */
const char *cx_last_error(void);

/* ---------------------------------------------------------------------- */
/* Operator registry                                                       */

/* Replaces get_interpolator(type, order, indextype)
 * (CarpetX/src/driver.cxx:593-628) and the nine operator tables it indexes
 * (prolongate_poly/cons/ddf/eno/minmod/hermite/natural/poly_cons3lfb/
 * poly_eno3lfb_3d_rf2, CarpetX/src/prolongate_3d_rf2.hxx:127-177).
 * type: "interpolate", "conservative", "ddf", "eno", "minmod", "hermite",
 * "natural", "poly-cons3lfb", "poly-eno3lfb"; indextype = (cx<<2)|(cy<<1)|cz
 * with c=1 for cell-centred (driver.cxx:595-596).  CX_EUNSUPPORTED if the
 * reference has no such operator. */
int cx_prolong_lookup(const char *type, int order, int indextype,
                      cx_op_t *out);

/* interp1d<...>::required_ghosts per direction (impl.hxx:398,462,518,585,
 * 636,783,847). */
int cx_prolong_required_ghosts(cx_op_t op, int ghosts[3]);

/* prolongate_3d_rf2::CoarseBox (impl.hxx:1236-1254): the fine box coarsened
 * by 2 (floor) and grown by required_ghosts. */
int cx_prolong_coarse_box(cx_op_t op, const int fine_lo[3],
                          const int fine_hi[3], int crse_lo[3],
                          int crse_hi[3]);

/* ---------------------------------------------------------------------- */
/* One box (the reference's launch granularity)                            */

/* Replaces prolongate_3d_rf2::interp (impl.hxx:2167-2188): writes the fine
 * points of reg (inclusive, must lie in the fine box) of ncomp components
 * from the coarse FAB.  per_group selects interp_per_group (impl.hxx:1691;
 * CarpetX parameter prolongate_per_group, param.ccl:449-451), which caps
 * ncomp at 16 and shares the ENO shift and the linear-fallback decision
 * between components; per_group = 0 is interp_per_var (impl.hxx:1256).  The
 * coarse FAB must contain every coarse point the stencils read (at most
 * CoarseBox(reg)); CX_EINVAL otherwise. */
int cx_prolong_box(cx_op_t op, const double *crse, const int crse_lo[3],
                   const int crse_hi[3], double *fine, const int fine_lo[3],
                   const int fine_hi[3], const int reg_lo[3],
                   const int reg_hi[3], int ncomp, int per_group,
                   cx_stream_t stream);

/* As cx_prolong_box, and additionally reports, per region point (x fastest)
 * and per component block (per-var: ncomp blocks, per-group: one), the ENO
 * shift chosen (3 signed bytes x,y,z; 0 for non-ENO directions) and whether
 * the linear fallback replaced the value (1 byte).  Either diagnostic
 * pointer may be NULL.  Diagnostic device arrays; used by the parity tests to
 * check the stencil choice bit for bit. */
int cx_prolong_box_diag(cx_op_t op, const double *crse, const int crse_lo[3],
                        const int crse_hi[3], double *fine,
                        const int fine_lo[3], const int fine_hi[3],
                        const int reg_lo[3], const int reg_hi[3], int ncomp,
                        int per_group, signed char *shifts,
                        unsigned char *fallback, cx_stream_t stream);

/* ---------------------------------------------------------------------- */
/* A whole refinement level in one launch                                  */

/* One box of a level transfer: the arguments of one interp() call. */
typedef struct {
  cx_op_t op;
  int ncomp;
  const double *crse;
  int crse_lo[3], crse_hi[3];
  double *fine;
  int fine_lo[3], fine_hi[3];
  int reg_lo[3], reg_hi[3];
} cx_box_t;

typedef struct cx_level_plan *cx_level_plan_t;

/* Builds the device-resident box/tile work list for a set of interp() calls
 * that would otherwise be one launch per box per component (the loop over
 * FillPatchInterp's boxes, CarpetX/src/fillpatch.cxx:116-119, 179-180).
 * Validates every box as cx_prolong_box does, picks the tile shape per box,
 * sorts tiles by cost and uploads the list (the only allocation).  The
 * boxes' data pointers are captured by the plan. */
int cx_level_plan_create(const cx_box_t *boxes, int nboxes, int per_group,
                         cx_level_plan_t *out);
/* Enqueues the whole level transfer on stream: one persistent launch per
 * separable kernel instantiation present (stencil pair and centring), then
 * the limited operators' launches.  Allocates nothing and does not
 * synchronise, so it can be captured into a CUDA graph. */
int cx_level_plan_execute(cx_level_plan_t plan, cx_stream_t stream);
/* Number of tiles and fine points (summed over components) in the plan. */
int cx_level_plan_stats(cx_level_plan_t plan, int64_t *ntiles,
                        int64_t *nfine_points, int64_t *algorithmic_bytes);
/* Kernel launches one execution enqueues: one per kernel instantiation
 * present, plus one per box of the limited operators (besides the memset of
 * the plan's item counters). */
int cx_level_plan_launches(cx_level_plan_t plan, int *nlaunches);
/* Frees the plan; the caller ensures no execution is still in flight. */
int cx_level_plan_destroy(cx_level_plan_t plan);
/* A level plan for the adjoint: executing it overwrites every box's crse
 * array (whole coarse box, every component) with P^T of its fine array,
 * reading the fine array only inside the region, as cx_prolong_adjoint_box
 * does box by box; one persistent launch per stencil pair and centring
 * present.  Validation is cx_prolong_box's.  Executed, destroyed and queried
 * like any level plan.  The limited operators (ENO, minmod, active linear
 * fallback) need cx_level_plan_create_adjoint_at: here they give
 * CX_EINVAL. */
int cx_level_plan_create_adjoint(const cx_box_t *boxes, int nboxes,
                                 int per_group, cx_level_plan_t *out);
/* The same with the coarse data the limited operators are linearised at:
 * crse_at[i] holds box i's coarse input (the layout of its crse array; may
 * be null for linear operators).  As cx_prolong_adjoint_box, P^T is taken
 * with each fine point's choices (ENO shift, minmod branch, linear fallback)
 * recomputed from crse_at: after the streaming launches, every box of a
 * limited operator takes its own launches (CCC minmod: one tiled kernel that
 * recomputes the choices; the others: a decision pass into scratch the plan
 * allocates once, then a gather).  Executions of one plan must not overlap
 * (the scratch is the plan's). */
int cx_level_plan_create_adjoint_at(const cx_box_t *boxes, const double *const *crse_at,
                                    int nboxes, int per_group, cx_level_plan_t *out);

/* ---------------------------------------------------------------------- */
/* A whole level without allocating device memory                          */

/* Upper limits of cx_level_execute_noalloc: boxes per call, work items per
 * call (an item is one component of up to 512 fine columns of a box over a
 * chunk of at most 128 fine z points). */
#define CX_NOALLOC_MAX_BOXES 1024
#define CX_NOALLOC_MAX_ITEMS 131072

/* The level transfer of cx_level_plan_create + cx_level_plan_execute, for
 * callers that cannot allocate device memory, such as a host framework whose
 * own allocator owns all device memory (a cudaMalloc of ours would fail, or
 * would take memory that allocator counts on): there is no plan object; the
 * work list lives in one fixed device array of the library (about 1.7 MB per
 * GPU, held until the process exits) and is rebuilt and copied onto `stream`
 * at every call.  Allocates nothing: no cudaMalloc, no cudaFree, no
 * allocating library call (an argument error records its message as every
 * entry point does).  The first call on a device looks the array's address
 * up (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the one array and a call
 * overwrites what the previous one left there, so calls whose kernels can
 * overlap on the GPU (different streams without ordering between them) race;
 * calls on one stream are ordered.  CX_EINVAL beyond CX_NOALLOC_MAX_BOXES
 * boxes or CX_NOALLOC_MAX_ITEMS work items.  No counterpart in the reference
 * (its operators never allocate device work lists). */
int cx_level_execute_noalloc(const cx_box_t *boxes, int nboxes, int per_group,
                             cx_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Restriction                                                             */

/* Replaces the average_down family called by Restrict
 * (CarpetX/src/schedule.cxx:2793-2815), picked by the number of
 * cell-centred directions of indextype: nodal (injection), edges, faces,
 * cells.  For every coarse point c of reg (inclusive, coarse index space):
 * vertex-centred directions take fine point 2c, cell-centred directions
 * average the children 2c and 2c+1; children are summed z-outer, x-inner
 * and the sum is scaled by 1/(number of children). */
int cx_restrict_box(int indextype, const double *fine, const int fine_lo[3],
                    const int fine_hi[3], double *crse, const int crse_lo[3],
                    const int crse_hi[3], const int reg_lo[3],
                    const int reg_hi[3], int ncomp, cx_stream_t stream);

/* The restriction of a whole level: average_down of every FAB pair of a
 * MultiFab (schedule.cxx:2793-2815 calls it once per level and group; AMReX
 * loops over the FABs), with the arithmetic of cx_restrict_box.  The plan
 * holds a device list of the boxes; executing it launches once per index
 * type present (one for a group).  Validation as cx_restrict_box, per box;
 * boxes with an empty region are skipped.  Coarse regions of distinct boxes
 * must not overlap. */
typedef struct {
  int indextype, ncomp;
  const double *fine;
  int fine_lo[3], fine_hi[3];
  double *crse;
  int crse_lo[3], crse_hi[3];
  int reg_lo[3], reg_hi[3];
} cx_restrict_box_t;
typedef struct cx_restrict_plan *cx_restrict_plan_t;
int cx_restrict_plan_create(const cx_restrict_box_t *boxes, int nboxes,
                            cx_restrict_plan_t *out);
int cx_restrict_plan_execute(cx_restrict_plan_t plan, cx_stream_t stream);
/* Coarse values set per execution, algorithmic bytes (8 per child read, 8
 * per coarse value written) and launches per execution. */
int cx_restrict_plan_stats(cx_restrict_plan_t plan, int64_t *ncoarse, int64_t *bytes,
                           int *nlaunches);
int cx_restrict_plan_destroy(cx_restrict_plan_t plan);

/* Restrict() of one level (CarpetX/src/schedule.cxx:2717-2837): the groups
 * to restrict from the next finer level, with the reference's selection.
 * A group is skipped when it is the regrid error (CarpetXRegrid::
 * regrid_error, :2746-2747) or has restriction disabled (do_restrict,
 * :2749-2750); of the others every time level but the oldest is restricted,
 * all of them when the group has only one (:2755-2756).  The selected time
 * levels' FAB pairs form one restriction plan (execute, stats and destroy as
 * for cx_restrict_plan_create): one launch per index type instead of one
 * average_down per group and time level.  restricted[g] receives how many
 * time levels of group g the plan restricts (0 if skipped): the caller then
 * marks the ghosts and the outer boundary of those time levels invalid on
 * the coarse level (:2821-2826).  Every FAB pair of a group must carry the
 * group's indextype and ncomp. */
typedef struct {
  int indextype;       /* the group's centring, as for cx_restrict_box */
  int ncomp;           /* the group's variables */
  int ntimelevels;     /* time levels the group stores (0 = the newest) */
  int do_restrict;     /* GroupData::do_restrict */
  int is_regrid_error; /* the group is CarpetXRegrid::regrid_error */
  int nfabs;           /* FAB pairs of one time level */
  const cx_restrict_box_t *fabs; /* ntimelevels x nfabs, time level major */
} cx_restrict_group_t;
int cx_restrict_groups_plan_create(const cx_restrict_group_t *groups, int ngroups,
                                   int *restricted, cx_restrict_plan_t *out);

/* ---------------------------------------------------------------------- */
/* Adjoints (no reference counterpart: the transposes of the above)        */

/* crse_bar = P^T fine_bar, with P the prolongation of cx_prolong_box
 * linearised at crse (ENO shift, minmod branch and linear-fallback choice
 * recomputed from crse).  crse_bar is overwritten over the whole coarse
 * box (zero where no region point reads).  Gather form, no atomics.  The
 * linear separable operators stream; the limited ones (ENO, minmod, active
 * linear fallback) take a decision pass and a gather per coarse point, with
 * stream-ordered scratch of 4 bytes per region point (cudaMallocAsync). */
int cx_prolong_adjoint_box(cx_op_t op, const double *crse,
                           const int crse_lo[3], const int crse_hi[3],
                           const double *fine_bar, const int fine_lo[3],
                           const int fine_hi[3], const int reg_lo[3],
                           const int reg_hi[3], int ncomp, int per_group,
                           double *crse_bar, cx_stream_t stream);

/* fine_bar = R^T crse_bar for cx_restrict_box; fine_bar is overwritten over
 * the whole fine box. */
int cx_restrict_adjoint_box(int indextype, const double *crse_bar,
                            const int crse_lo[3], const int crse_hi[3],
                            double *fine_bar, const int fine_lo[3],
                            const int fine_hi[3], const int reg_lo[3],
                            const int reg_hi[3], int ncomp,
                            cx_stream_t stream);

/* ---- Outer boundary conditions --------------------------------------------
 * The step after a prolongation in CarpetX's sync: points of a FAB outside
 * the domain interior are set from its symmetries and boundary conditions,
 * as BoundaryCondition(groupdata, dest).apply() does (CarpetX/src/
 * boundaries.cxx:32-118, boundaries_impl.hxx:28-444).
 *
 * The interior is the domain's cells, or its vertices in vertex-centred
 * directions: [domain_lo, domain_hi + 1 + !indextype).  A face's condition
 * is chosen as in apply_on_face (boundaries_impl.hxx:71-108): periodic
 * faces, and faces with no or an inter-patch symmetry and no boundary
 * condition, set nothing; reflection symmetry takes precedence over the
 * group's condition.  On edges and corners the conditions of all boundary
 * directions combine: Dirichlet sets the value; otherwise the value is read
 * at the source point (the interior edge point in Neumann, Robin and
 * linear-extrapolation directions, the mirror point in reflection
 * directions), then the Robin fall-off, the linear extrapolation and the
 * reflection parity are applied, in that order, with the reference's
 * rounding.  Every point written reads only points that are not written, so
 * one launch covers all regions of all FABs.
 *
 * Symmetries (PatchData::symmetries) and boundary conditions
 * (GroupData::boundaries) with CarpetX's numbering (driver.hxx:41-57). */
enum { CX_SYM_NONE = 0, CX_SYM_INTERPATCH = 1, CX_SYM_PERIODIC = 2, CX_SYM_REFLECTION = 3 };
enum {
  CX_BC_NONE = 0,
  CX_BC_SYMMETRY_BOUNDARY = 1,
  CX_BC_DIRICHLET = 2,
  CX_BC_LINEAR_EXTRAPOLATION = 3,
  CX_BC_NEUMANN = 4,
  CX_BC_ROBIN = 5
};
#define CX_BC_MAX_COMPS 16 /* maxncomps, boundaries_impl.hxx:30 */

/* A group's conditions on one level. */
typedef struct {
  int symmetry[2][3];               /* [face: 0 lower, 1 upper][direction], CX_SYM_* */
  int boundary[2][3];               /* CX_BC_*, same indexing */
  int domain_lo[3], domain_hi[3];   /* Geometry::Domain(): cell-centred, inclusive */
  double prob_lo[3], prob_hi[3];    /* Geometry::ProbLo / ProbHi */
  double dx[3];                     /* Geometry::CellSize */
  int indextype[3];                 /* 1: cell centred in direction d */
  int nghost[3];                    /* MultiFab::nGrow of the level's FABs */
  int ncomp;                        /* 1..CX_BC_MAX_COMPS */
  double dirichlet[CX_BC_MAX_COMPS]; /* GroupData::dirichlet_values */
  double robin[CX_BC_MAX_COMPS];    /* GroupData::robin_values (value at infinity) */
  int parity[CX_BC_MAX_COMPS][3];   /* GroupData::parities: +1 or -1 */
} cx_bc_t;

/* One FAB of the level: device data (ncomp components) on [lo, hi]. */
typedef struct {
  double *data;
  int lo[3], hi[3];
} cx_bc_fab_t;

/* BoundaryCondition(groupdata, dest).apply() on one FAB: one launch, no
 * allocation.  CX_EINVAL for a face whose symmetry and condition do not
 * combine (the reference's "internal error"), ncomp out of range, a
 * parity other than +-1, or a source point outside the FAB or outside the
 * interior (the reference asserts the first and does not check the second,
 * which only a domain narrower than the ghost zones can violate). */
int cx_boundary_box(const cx_bc_t *bc, double *data, const int lo[3], const int hi[3],
                    cx_stream_t stream);

/* GroupData::apply_boundary_conditions (driver.cxx:967-995) for every FAB of
 * a level in one launch.  Nothing is done when every direction is periodic;
 * FABs inside the domain grown by nghost in its periodic directions are
 * skipped.  The plan holds the device list of regions; FABs must not
 * overlap.  Create once per regrid, execute every sync (no allocation,
 * graph-capturable). */
typedef struct cx_boundary_plan *cx_boundary_plan_t;
int cx_boundary_plan_create(const cx_bc_t *bc, const cx_bc_fab_t *fabs, int nfabs,
                            cx_boundary_plan_t *out);
int cx_boundary_plan_execute(cx_boundary_plan_t plan, cx_stream_t stream);
/* Points set per execution (over all components: npoints x ncomp values)
 * and algorithmic bytes: 8 written per value, plus 8 read unless Dirichlet. */
int cx_boundary_plan_stats(cx_boundary_plan_t plan, int64_t *npoints, int64_t *bytes);
int cx_boundary_plan_destroy(cx_boundary_plan_t plan);

/* ---- Region copies: ParallelCopy and FillBoundary on one GPU ---------------
 * The copies around a prolongation in CarpetX's sync (CarpetX/src/
 * fillpatch.cxx:34-37, 63-64, 91-93, 122-124, 175, 205-207, 218-225): the
 * same-level halo exchange (AMReX MultiFab::FillBoundary), the gather of the
 * coarse patches and the scatter of the interpolated fine patches
 * (MultiFab::ParallelCopy).  A copy plan holds the pieces (destination box,
 * source FAB, periodic shift) computed once per regrid; executing it copies
 * every piece of every FAB in one launch.  AMReX's sources are not in the
 * reference tree: the rules below restate its documented behaviour.  Where
 * several sources cover a destination point (valid boxes that share a face
 * in vertex-centred directions, or grown source boxes), the first in list
 * order, then image order, sets it, so that pieces never overlap.  FABs
 * must not overlap in memory. */
typedef struct {
  double *data;                 /* device data, ncomp components on [lo, hi] */
  int lo[3], hi[3];             /* the FAB: its valid box grown by its ghosts */
  int valid_lo[3], valid_hi[3]; /* the valid box */
} cx_fab_t;

typedef struct cx_copy_plan *cx_copy_plan_t;

/* Reflux of one coarse level from the next finer (Reflux(),
 * CarpetX/src/schedule.cxx:2632-2713), replacing AMReX's FluxRegister
 * (built at driver.cxx:918-924; AMReX 25.11 is not in the reference tree):
 * per direction d CrseInit(coarse flux_d, d, 0, 0, ncomp, -1) and
 * FineAdd(fine flux_d, d, 0, 0, ncomp, +1), then Reflux(coarse state,
 * scale, 0, 0, ncomp, coarse geometry).  For every face of a fine box's
 * coarsened boundary, reg = -(coarse flux) + the fine fluxes of the 2 x 2
 * fine faces covering it (the higher transverse direction outer), and the
 * coarse cell just outside the fine box gets -scale * reg / vol across a low
 * face and +scale * reg / vol across a high face (vol = dx[0] dx[1] dx[2]),
 * orientation by orientation: x, y, z low, then x, y, z high.  The coarse
 * flux of a face comes from the first coarse flux FAB whose valid faces hold
 * it.  Coarse cells under other fine boxes are corrected too, as in AMReX;
 * the restriction that follows overwrites them.
 *   crse: the coarse state FABs (cell centred); crse_flux[d]: per direction
 *   the coarse flux FABs (ncrse each, same order, valid box = the state's
 *   face centred in d); fine_flux[d]: per direction the fine flux FABs, one
 *   per fine box (valid box = the box's cells face centred in d; the boxes
 *   must be coarsenable by 2).  The plan holds a device list of the faces;
 *   executing it launches once per orientation that has faces. */
typedef struct cx_reflux_plan *cx_reflux_plan_t;
int cx_reflux_plan_create(const cx_fab_t *crse, int ncrse, const cx_fab_t *const crse_flux[3],
                          const cx_fab_t *const fine_flux[3], int nfine, int ncomp,
                          const double dx[3], double scale, cx_reflux_plan_t *out);
int cx_reflux_plan_execute(cx_reflux_plan_t plan, cx_stream_t stream);
/* Register faces per execution (coarse faces x orientations), algorithmic
 * bytes (per face and component: the coarse flux, four fine fluxes, the
 * coarse value read and written) and launches per execution. */
int cx_reflux_plan_stats(cx_reflux_plan_t plan, int64_t *faces, int64_t *bytes, int *launches);
int cx_reflux_plan_destroy(cx_reflux_plan_t plan);

/* dst.ParallelCopy(src, 0, 0, ncomp, src_nghost, dst_nghost, period): every
 * point of each destination FAB's valid box grown by dst_nghost (clipped to
 * the FAB) is set from the first source FAB whose valid box grown by
 * src_nghost (clipped to that FAB), shifted by a periodic image (shift 0
 * first, then -period, +period per direction, z outermost), contains it;
 * points no source covers are left unchanged.  period[d] = 0: not periodic
 * in d. */
int cx_copy_plan_parallel_copy(const cx_fab_t *dst, int ndst, const cx_fab_t *src, int nsrc,
                               int ncomp, const int src_nghost[3], const int dst_nghost[3],
                               const int period[3], cx_copy_plan_t *out);

/* mf.FillBoundary(0, ncomp, nghost, period): every point of each FAB within
 * nghost of its valid box (clipped to the FAB) and outside it is set from
 * the first FAB, in list order and then image order, whose valid box
 * shifted by a periodic image contains it; a FAB is never its own source at
 * shift 0. */
int cx_copy_plan_fill_boundary(const cx_fab_t *fabs, int nfabs, int ncomp, const int nghost[3],
                               const int period[3], cx_copy_plan_t *out);

int cx_copy_plan_execute(cx_copy_plan_t plan, cx_stream_t stream);
/* Points copied per execution (each ncomp values), pieces, and algorithmic
 * bytes (16 per value: one read, one write). */
int cx_copy_plan_stats(cx_copy_plan_t plan, int64_t *npoints, int64_t *npieces, int64_t *bytes);
int cx_copy_plan_destroy(cx_copy_plan_t plan);

#ifdef __cplusplus
}
#endif
#endif
