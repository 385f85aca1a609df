/*
 * agd_b200.h - C ABI of the B200 eikonal path (Isotropic2/3, Riemann2/3).
 *
 * Plain pointers and sizes only.  Every array argument is DEVICE memory owned
 * by the caller unless stated otherwise; nothing here allocates device memory.
 * "tile layout" is the bilevel layout of the reference's kernels: a grid of
 * shape s padded to a multiple of the tile shape s_i, stored tile after tile
 * (index n_o * size_i + n_i), one plane after the other for multi-component
 * fields (agd/FiniteDifferences.py:164-222, block_expand/block_squeeze).
 * "grid layout" is plain row-major order over the true shape.
 *
 * All entry points enqueue work on `stream` and return an agd_status code
 * (0 on success); agd_last_error() describes the last failure of this thread.
 */
#ifndef AGD_B200_H
#define AGD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default) /* the library is built with hidden visibility */
#endif

typedef struct CUstream_st *agd_stream_t; /* a cudaStream_t */

enum agd_status {
    AGD_STATUS_OK = 0,
    AGD_STATUS_INVALID = 1,       /* bad argument (shape, tile, pointer, size) */
    AGD_STATUS_NOT_CONVERGED = 2, /* nitermax_o outer iterations reached */
    AGD_STATUS_CUDA = 4,          /* CUDA runtime error */
    AGD_STATUS_WATCHDOG = 8,      /* a bounded device-side wait timed out */
    AGD_STATUS_WORKSPACE = 16,    /* workspace too small */
    AGD_STATUS_UNSUPPORTED = 32   /* tile shape / model combination not built */
};

/* Diagonal: the Isotropic scheme (unit offsets) with weights per point and
 * axis, the squared dual costs (Isotropic_.h:32-36, _SetGeometry.py:134-135).
 * Rander: the Riemann scheme on the inverse of the quadratic part, with the
 * neighbour values at x -/+ e shifted by +/-<w, e> for the drift w
 * (Riemann_.h:23-29, FiniteDifferences.h:41-45; the second order neighbour
 * is not shifted). */
enum agd_model { AGD_MODEL_ISOTROPIC = 0, AGD_MODEL_RIEMANN = 1, AGD_MODEL_DIAGONAL = 2, AGD_MODEL_RANDER = 3 };

/* One eikonal problem.  Mirrors what the reference's Interface prepares for its
 * `Update` kernel: traits (shape_i, niter_i, fim_front_width), module constants
 * (shape_o/shape_tot, atol, rtol, isotropic weights, multip_step/multip_max) and
 * kernel arguments (values, valuesq, geom, seedTags, rhs), see
 * agd/Eikonal/HFM_CUDA/_Kernel.py:94-381 and cuda/Update.h:20-50. */
typedef struct agd_instance {
    int model;          /* enum agd_model */
    int ndim;           /* 2 or 3 */
    int shape[3];       /* grid shape */
    int shape_i[3];     /* tile shape: (8,8), (16,16) in 2D; (4,4,4) in 3D */
    int niter_i;        /* local iterations per tile visit */
    int fim_front_width;/* FIM front width (>= 2) */
    int nitermax_o;     /* maximum number of outer iterations */
    int flags;          /* AGD_FLAG_* */
    float atol, rtol;   /* per-point convergence: |du| <= atol + rtol |u| */
    float iso_weights[3]; /* isotropic model: gridScale^-2 per axis */
    float multip_step;  /* multiprecision: u + uq * multip_step (0: off); on output the
                           solution is values + valuesq * multip_step */
    float multip_max;
    float *values;      /* tile layout, in: initial values (+inf cold), out: solution */
    int32_t *valuesq;   /* tile layout, multiprecision integer part (or NULL) */
    float *values_next; /* multiprecision: second buffers of the double-buffered */
    int32_t *valuesq_next; /*  iterations (valuesNext, valuesqNext of _SetArgs.py:171-177) */
    const float *geom;  /* Riemann: dual metric, symdim planes; Diagonal: squared dual
                           costs 1/(c_k h_k)^2, ndim planes; Rander: the inverse of the
                           quadratic part (symdim planes) then the drift (ndim planes),
                           grid scales applied; tile layout (Isotropic: NULL) */
    const float *rhs;   /* tile layout: cost, seed values at seeds, +inf padding */
    const uint8_t *seedbits; /* tile layout bits, little endian, padding bits set;
                                4-byte aligned */
    const uint8_t *trigger;  /* per tile, nonzero = active at the first iteration
                                (NULL: tiles holding a seed) */
    /* Source factorisation (factoringRadius; _Kernel.py:47-49, 301-308,
     * cuda/FiniteDifferences.h:30-75): at the points closer than
     * sqrt(factor_radius2) (index units) to factor_origin, the neighbour values
     * are shifted so that the scheme is exact for the distance |x - origin|_m.
     * factor_radius2 = 0: off.  Not with multiprecision. */
    float factor_radius2;
    float factor_origin[3];  /* the seed, continuous index coordinates */
    float factor_metric[6];  /* metric at the seed with cost and grid scales applied (index
                                units): packed lower triangle (Riemann), squared costs per
                                axis (Isotropic) */
    /* Second order scheme (order: 2; cuda/HFM.h:91-138, 175-206): threshold on
     * |u - 2v + v2| / max(u - v) below which a neighbour is extrapolated to
     * second order (order2_threshold, default 0.3).  0: first order.  Not with
     * multiprecision or source factorisation. */
    float order2_threshold;
    /* Obstacles (walls; cuda/Walls.h:18-50, _SetGeometry.py:262-280): L1 distance
     * to the nearest wall point in tile layout, uint8, 255 beyond wallDistBound
     * and at padding (agd_prep_walls writes it).  A stencil offset whose segment
     * meets a wall has an infinite neighbour value.  The wall points themselves
     * are seeds of value +inf.  NULL: no walls.  Riemann instances with walls
     * need the stencil cache of agd_eikonal_solve / agd_plan_run (the fixed
     * scratch entry point refuses them). */
    const uint8_t *wall_dist;
    /* Release epochs (no counterpart in the reference, whose fast iterative
     * method visits a tile at the epoch after a neighbour changed,
     * _solvers.py:94-120): per tile (tile order n_o), the first epoch at which
     * the tile may be visited.  A tile the method asks for earlier waits in
     * the list of its release epoch (at most 31 epochs ahead); the iteration
     * still runs to the reference's stopping test, so the fixed point is the
     * same.  A schedule made from predicted arrival times (the learned warm
     * start) visits tiles near their upstream's convergence instead of at the
     * front's first touch.  NULL: the reference's schedule. */
    const uint16_t *release;
} agd_instance;

#define AGD_FLAG_ACTIVATE_ALL 1 /* every tile is active at the first iteration */
/* The outer iteration (the `solver` key, _Kernel.py:71-81, _solvers.py:77-193);
 * neither flag: the fast iterative method (the default). */
#define AGD_FLAG_SOLVER_AGSI 2   /* adaptive Gauss-Seidel: a tile that changed is
                                    visited again with its neighbours */
#define AGD_FLAG_SOLVER_GLOBAL 4 /* global iteration: every tile at every epoch
                                    until an epoch changes nothing */

/* Per-instance results, written by the solver into device memory. */
typedef struct agd_stats {
    int32_t niter_o;      /* outer iterations (epochs) used by this instance */
    int32_t status;       /* agd_status of this instance */
    int64_t tile_visits;  /* tile visits; grid updates = tile_visits * size_i */
} agd_stats;

/* Solver tuning (0 = automatic). */
typedef struct agd_launch {
    int ctas;             /* persistent CTAs (<= co-resident maximum) */
    int warps_per_cta;    /* 4 or 8 */
    int64_t timeout_ns;   /* bound on any device-side wait (default 2 s) */
} agd_launch;

/* ---------------------------------------------------------------- eikonal -- */

/* A plan holds, in host memory, the descriptors of n instances solved together
 * and the layout of their workspace.  It replaces the reference's per-call
 * setup of traits, module constants and kernel arguments
 * (agd/Eikonal/HFM_CUDA/_Kernel.py:23-381).  inst: host array of n. */
typedef struct agd_plan agd_plan;
int agd_plan_create(const agd_instance *inst, int n, agd_plan **plan);
void agd_plan_destroy(agd_plan *plan);

/* Bytes of device workspace needed by the plan. */
size_t agd_plan_workspace_bytes(const agd_plan *plan);

/* Copies the plan's descriptors into the workspace (once per workspace). */
int agd_plan_upload(const agd_plan *plan, void *workspace, size_t workspace_bytes, agd_stream_t stream);

/* Solves the plan's instances in one persistent launch, from the values they
 * hold (the fixed point of the reference's `Update` kernel, iterated as by
 * `_solvers.fast_iterative_method`).  Only memsets and kernel launches are
 * enqueued, so a run can be captured in a CUDA graph.
 * Replaces: _solvers.Solve / fast_iterative_method / InitStop
 * (agd/Eikonal/HFM_CUDA/_solvers.py:15-120, _StopCriterion.py:21-84) and the
 * eikonal `Update` kernel (cuda/Update.h:20-227) they launch.
 * stats: DEVICE array of n agd_stats (may be NULL).  Returns AGD_STATUS_OK
 * once enqueued; per-instance convergence is in stats[i].status. */
int agd_plan_run(const agd_plan *plan, void *workspace, size_t workspace_bytes, agd_stats *stats,
                 const agd_launch *launch, agd_stream_t stream);

/* One-shot form: plan, upload, run, destroy. */
size_t agd_eikonal_workspace_bytes(const agd_instance *inst, int n);
int agd_eikonal_solve(const agd_instance *inst, int n, void *workspace, size_t workspace_bytes,
                      agd_stats *stats, const agd_launch *launch, agd_stream_t stream);

/* Same solve as agd_eikonal_solve, for callers that cannot allocate device
 * memory: code running inside a host application that owns the device
 * allocator (plugins, sandboxed or budgeted hosts), or that must not call
 * cudaMalloc at that point.  It takes no workspace: its scratch is a
 * file-scope device array of AGD_FIXED_SCRATCH_BYTES that every device which
 * loads the library holds until the process exits.  No counterpart in the
 * reference, which allocates its work arrays per call.
 * - Instances needing more scratch than that (the scratch grows with the
 *   number of tiles: about 200 Riemann2 512^2 or Isotropic2 1024^2 problems
 *   fit), or more than AGD_FIXED_SCRATCH_MAX_INSTANCES of them, are rejected
 *   with AGD_STATUS_WORKSPACE / AGD_STATUS_INVALID before any device work.
 * - The first call on a device looks the array's device address up
 *   (cudaGetSymbolAddress); make that first call before any stream capture.
 * - Every call shares the one array, which keeps the last call's contents (the
 *   solver clears what it needs at zero itself): calls that overlap on the GPU
 *   race, so issue them on a single stream or otherwise serialise them.
 * It calls no cudaMalloc, cudaFree or allocating library routine. */
#define AGD_FIXED_SCRATCH_BYTES (32u << 20)
#define AGD_FIXED_SCRATCH_MAX_INSTANCES 256
int agd_eikonal_solve_fixed_scratch(const agd_instance *inst, int n, agd_stats *stats, const agd_launch *launch,
                                    agd_stream_t stream);

/* ------------------------------------------------------------ preparation -- */

/* Dual metric of metric.with_costs(gridScales) (or of dualMetric.with_speeds)
 * in tile layout, padded with +inf.  Replaces the host code of
 * _SetGeometry.SetGeometry (agd/Eikonal/HFM_CUDA/_SetGeometry.py:127-137,189-194).
 * metric: grid layout, (*shape, symdim) HFM order [m00, m10, m11, (m20, m21, m22)];
 * with broadcast != 0 a single (symdim,) tensor for the whole grid. */
int agd_prep_geom(int ndim, const int *shape, const int *shape_i, const float *metric, int broadcast,
                  int is_dual, const double *grid_scales, float *geom, agd_stream_t stream);

/* Diagonal model: the squared dual costs, ndim planes in tile layout padded
 * with +inf: 1/(c_k h_k)^2 of metric.with_costs(gridScales), or with is_dual
 * (d_k / h_k)^2 of dualMetric.with_speeds(gridScales) (_SetGeometry.py:134-135).
 * costs: grid layout (*shape, ndim) HFM order; with broadcast != 0 one (ndim,)
 * vector for the whole grid. */
int agd_prep_geom_diagonal(int ndim, const int *shape, const int *shape_i, const float *costs, int broadcast,
                           int is_dual, const double *grid_scales, float *geom, agd_stream_t stream);

/* Rander model: metric.with_costs(gridScales).flatten(inverse_m=True), i.e. the
 * inverse of m * outer(h, h) (symdim planes) then w * h (ndim planes), tile
 * layout padded with +inf (_SetGeometry.py:138-139, Metrics/rander.py:61-68).
 * metric: grid layout (*shape, symdim + ndim) [m lower triangle, w]; with
 * is_dual it holds the dual metric, scaled by with_speeds(gridScales) and
 * turned into the metric by Rander.dual (rander.py:35-39); broadcast != 0: one
 * (symdim + ndim,) vector for the whole grid. */
int agd_prep_geom_rander(int ndim, const int *shape, const int *shape_i, const float *metric, int broadcast,
                         int is_dual, const double *grid_scales, float *geom, agd_stream_t stream);

/* Grid layout -> tile layout for `nplanes` planes, padding with `pad`
 * (fd.block_expand).  src_broadcast != 0: src holds one value per plane. */
int agd_block_expand(int ndim, const int *shape, const int *shape_i, int nplanes, const float *src,
                     int src_broadcast, float pad, float *dst, agd_stream_t stream);

/* Tile layout -> grid layout (fd.block_squeeze). */
int agd_block_squeeze(int ndim, const int *shape, const int *shape_i, int nplanes, const float *src,
                      float *dst, agd_stream_t stream);

/* Seeds: sets rhs at the seed points to the seed values, writes the packed
 * seed bits (padding bits set) and, if trigger != NULL, the per-tile trigger.
 * seed_index: (n, ndim) int32 grid indices.  Replaces _SetArgs.SetRHS/SetArgs
 * (agd/Eikonal/HFM_CUDA/_SetArgs.py:8-177) for rounded seeds. */
int agd_prep_seeds(int ndim, const int *shape, const int *shape_i, const int32_t *seed_index,
                   const float *seed_values, int n, float *rhs, uint8_t *seedbits, uint8_t *trigger,
                   agd_stream_t stream);

/* Preparation of n instances that share one grid and tile shape, for repeated
 * batched solves: one launch writes, for every instance, the geometry (as
 * agd_prep_geom, agd_prep_geom_diagonal or agd_prep_geom_rander), the
 * right-hand side (cost, or 1, with +inf padding as agd_block_expand, +inf at
 * walls), values = +inf and the padding and wall seed bits;
 * a second launch places the seeds as agd_prep_seeds does, one thread per
 * instance, in seed order.  The reference prepares one instance per call
 * (_SetGeometry.py:16-282, _SetArgs.py:8-177); this batched form has no
 * counterpart there.  Arrays are instance-major, with the per-instance sizes
 * given beside each field. */
typedef struct agd_batch_prep {
    int model;                  /* AGD_MODEL_ISOTROPIC, _RIEMANN, _DIAGONAL or _RANDER */
    int ndim;                   /* 2 or 3 */
    int shape[3];               /* grid shape (unused trailing entries 1) */
    int shape_i[3];             /* tile shape */
    int n;                      /* number of instances */
    int is_dual;                /* `metric` holds the dual metric (speeds for Diagonal) */
    double grid_scales[3];
    /* prod(shape) x k per instance, HFM packing: Riemann k = symdim (the
     * metric), Diagonal k = ndim (the costs per axis), Rander k = symdim + ndim
     * (metric, then drift); NULL for Isotropic */
    const float *metric;
    const float *cost;          /* prod(shape), or NULL for cost 1 */
    const int32_t *seed_index;  /* nseeds x ndim grid indices */
    const float *seed_values;   /* nseeds, or NULL for 0 */
    int nseeds;                 /* seeds per instance (>= 0) */
    float *geom;                /* planes in tile layout: symdim (Riemann), ndim (Diagonal),
                                   symdim + ndim (Rander) x size_tot; NULL for Isotropic */
    float *rhs;                 /* size_tot */
    float *values;              /* size_tot */
    uint8_t *seedbits;          /* size_tot / 8 */
    int32_t *bad_seed;          /* device flag set to 1 for a seed outside the grid; may be NULL */
    /* Obstacles (optional): wall mask in grid layout, prod(shape) bytes per
     * instance, or one mask for every instance with walls_shared = 1.  Wall
     * points become seeds of value +inf, over the seeds (_SetArgs.py:124-126);
     * the wall distances of agd_instance.wall_dist come from agd_prep_walls or
     * agd_prep_walls_batch. */
    const uint8_t *walls;
    int walls_shared;
    /* size_o bytes per instance, or NULL: the tiles holding a seed (1) and the
     * others (0), the first tiles of a solve with walls (_SetArgs.py:119-126) */
    uint8_t *trigger;
} agd_batch_prep;

int agd_prep_batch(const agd_batch_prep *prep, agd_stream_t stream);

/* Obstacles: from the wall mask (grid layout uint8, nonzero = wall) writes
 * wall_dist (tile layout, size_tot bytes): the L1 distance to the nearest wall
 * point, by `bound` min-plus passes of the 3^ndim L1 kernel (inf_convolution
 * with distance_kernel(1, ndim, uint8, ord=1), saturated at 255), 255 beyond
 * `bound` and at padding (_SetGeometry.py:262-280).  If rhs / seedbits are not
 * NULL, the wall points become seeds of value +inf there (_SetArgs.py:124-126):
 * call it after agd_prep_seeds, walls override seeds.  tmp: 2 * prod(shape)
 * bytes of scratch. */
int agd_prep_walls(int ndim, const int *shape, const int *shape_i, const uint8_t *walls, int bound,
                   uint8_t *wall_dist, uint8_t *tmp, float *rhs, uint8_t *seedbits, agd_stream_t stream);

/* agd_prep_walls for n instances of one grid and tile shape at once (the
 * distance maps only; the wall points become seeds in agd_prep_batch): walls
 * n x prod(shape) bytes (grid layout), wall_dist n x size_tot bytes (tile
 * layout), tmp 2 n prod(shape) bytes of scratch.  No counterpart in the
 * reference, which prepares one instance per call. */
int agd_prep_walls_batch(int ndim, const int *shape, const int *shape_i, int n, const uint8_t *walls, int bound,
                         uint8_t *wall_dist, uint8_t *tmp, agd_stream_t stream);

/* Selling decomposition of n packed symmetric matrices (symdim floats each):
 * weights (n, symdim), integer offsets (n, symdim, ndim).  Same decomposition
 * as the kernel's decomp_m (cuda/Geometry2.h:21-48, Geometry3.h:22-58). */
int agd_selling(int ndim, const float *m, int n, float *weights, int32_t *offsets, agd_stream_t stream);

/* The same decomposition in the planar layouts of the reference's standalone
 * VoronoiDecomposition kernel (Kernel_VoronoiDecomposition.h:45-69,
 * HFM_CUDA/VoronoiDecomposition.py:15-98, dimensions 1 to 3): m (symdim, n)
 * lower triangles row major, weights (symdim, n), offsets (ndim, symdim, n) of
 * offset_bytes-byte signed integers (1, 2, 4 or 8).  Dimension 1: weight = m,
 * offset = 1. */
int agd_voronoi_decomposition(int ndim, const float *m, long long n, float *weights, void *offsets,
                              int offset_bytes, agd_stream_t stream);

/* ------------------------------------------------------------------- flow -- */

/* Upwind geodesic flow of a solved instance, one pass over all tiles (the
 * FLOW_* variant of the reference's `Update`, cuda/Update.h:171-209, run by
 * _PostProcess.PostProcess, agd/Eikonal/HFM_CUDA/_PostProcess.py:46-95).
 * Outputs, tile layout, any may be NULL: flow_vector (ndim planes),
 * flow_weightsum, flow_weights (nact planes), flow_indices (nact planes, tile
 * layout index of the upwind neighbour, INT32_MAX when the weight is zero). */
int agd_flow(const agd_instance *inst, float *flow_vector, float *flow_weightsum, float *flow_weights,
             int32_t *flow_indices, agd_stream_t stream);

/* -------------------------------------------------------------- geodesics -- */

/* Distance-to-seed map in 1/5 pixel units, saturated at 255, grid layout
 * (inf_convolution with a 3^ndim kernel, ceil(target_tolerance) passes, cut
 * beyond 5*target_tolerance: agd/Eikonal/HFM_CUDA/_GetGeodesics.py:51-75).
 * seed_mask: grid layout uint8.  tmp: scratch of the same size. */
int agd_eucl_map(int ndim, const int *shape, const uint8_t *seed_mask, int npasses, int cut,
                 uint8_t *eucl, uint8_t *tmp, agd_stream_t stream);

/* Geodesic backtracking, one warp per tip, with the reference's chunking
 * (chunks of `typical_len` points restarting the stopping-criteria history,
 * at most `max_chunks` chunks), midpoint rule, causality filtered multilinear
 * flow and stop codes (0 Continue, 1 AtSeed, 2 InWall, 3 Stationnary,
 * 4 PastSeed, 5 VanishingFlow).  The PastSeed test starts after
 * `pastseed_delay` steps in the first chunk, at once in the later ones.
 * Replaces GetGeodesics + GeodesicODE (_GetGeodesics.py:9-147,
 * cuda/Kernel_GeodesicODE.h:265-412).
 * tips: (ntips, ndim) continuous grid indices.  paths: (ntips, cap, ndim),
 * with cap >= max_chunks*(typical_len-1)+1; lengths, stops: ntips entries. */
int agd_geodesics(const agd_instance *inst, const float *flow_vector, const float *flow_weightsum,
                  const uint8_t *eucl, const float *tips, int ntips, float step, float causality,
                  int typical_len, int max_chunks, int eucl_delay, int nymin_delay, int pastseed_delay,
                  float *paths, int cap, int32_t *lengths, int8_t *stops, agd_stream_t stream);

/* ---------------------------------------------------------------- adjoint -- */

/* Workspace for agd_reverse. */
size_t agd_reverse_workspace_bytes(const agd_instance *inst);

/* Reverse-mode sensitivity: solves diag*lam - W^T lam = sens on the tiles, where
 * W holds the upwind flow weights (flow_weights/flow_indices of agd_flow) and
 * diag = flow_weightsum (1 where it vanishes).  sens, lam: tile layout.
 * Replaces SolveAD's reverse branch, graph_reverse and the linear Update kernel
 * (_PostProcess.py:97-219, graph_reverse.py:10-77, cuda/GraphReverse.h:35-82,
 * cuda/Kernel_LinearUpdate.h:99-218). */
int agd_reverse(const agd_instance *inst, const float *flow_weights, const int32_t *flow_indices,
                const float *flow_weightsum, const float *sens, float *lam, float atol, float rtol,
                void *workspace, size_t workspace_bytes, agd_stats *stats, const agd_launch *launch,
                agd_stream_t stream);

/* Forward-mode variation: solves diag*du - W du = rhs on the tiles, the system
 * itself rather than its transpose (same flow arrays and diag as agd_reverse;
 * workspace: agd_reverse_workspace_bytes).  rhs = cost * (variation of the
 * cost), or the seed value's variation at a seed; rhs, du: tile layout.
 * Replaces SolveAD's forward branch (_PostProcess.py:181-191) and its linear
 * Update kernel (cuda/Kernel_LinearUpdate.h:99-218). */
int agd_forward(const agd_instance *inst, const float *flow_weights, const int32_t *flow_indices,
                const float *flow_weightsum, const float *rhs, float *du, float atol, float rtol,
                void *workspace, size_t workspace_bytes, agd_stats *stats, const agd_launch *launch,
                agd_stream_t stream);

/* ------------------------------------------------------------------- misc -- */

const char *agd_last_error(void);
int agd_version(void); /* 4: agd_geodesics with pastseed_delay */

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* AGD_B200_H */
