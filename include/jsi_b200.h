/* jsi_b200 — B200-native NURBS minimum-distance and surface-surface
 * intersection query path, C ABI.
 *
 * This is the drop-in boundary for the query path of JSI_CAD_NEXT VERSION5.
 * Each entry point names the reference interface it replaces (paths relative
 * to JSI_CAD_NEXT_VERSION5/).  All calls return an int status (JSI_OK = 0,
 * negative = error class); nothing exits the process.  Pointers are plain
 * host pointers unless stated otherwise; no CUDA or C++ types cross the ABI.
 *
 * Threading: a context owns one CUDA stream and one device arena; calls on the
 * same context are serialised by an internal mutex.  Use one context per
 * host thread for concurrency.
 */
#ifndef JSI_B200_H
#define JSI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define JSI_B200_ABI_VERSION 3
#define JSI_MAX_ROUNDS 16
#define JSI_RECORD_SIZE 18 /* ONE_UV_SIZE, include/jsi_cad.hpp:45 */

typedef enum {
  JSI_OK = 0,
  JSI_ERR_INVALID = -1,     /* bad argument (null pointer, nuv < 2, k < 1, ...) */
  JSI_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  JSI_ERR_NOMEM = -3,       /* device arena or HBM budget exhausted */
  JSI_ERR_CAPACITY = -4,    /* a result did not fit the caller's buffer or an internal list */
  JSI_ERR_SURFACE = -5,     /* malformed surface header / data */
  JSI_ERR_TIMEOUT = -6,     /* a bounded device wait gave up */
  JSI_ERR_UNSUPPORTED = -7, /* option not available in this build */
  JSI_ERR_NO_DEVICE = -8    /* no CUDA device / extension not usable */
} jsi_status;

/* Arithmetic form of a query.
 *  V5_FP32      - VERSION5's FP32 arithmetic reproduced operation for
 *                 operation: same k-th value, same candidate sets.
 *  FP64         - the same algorithm entirely in FP64 (plain form).
 *  FP32_SCREEN  - FP32 evaluation / boxes / screening with every box widened
 *                 by a rigorous rounding-error bound, FP64 knot spans, basis
 *                 and rational division, FP64 re-check of the screened
 *                 candidates; results equal the FP64 form's.  Distance: the
 *                 first round screens in FP32.  Intersection: the first
 *                 round's samples, curvature terms, cell boxes and overlap
 *                 screen run in FP32 (the compute_K maxima are made exact by
 *                 re-evaluating in FP64 only the samples whose FP32 bound
 *                 reaches the maximum), every candidate pair is re-checked
 *                 with FP64 boxes, and later rounds run in FP64. */
typedef enum { JSI_PREC_V5_FP32 = 0, JSI_PREC_FP64 = 1, JSI_PREC_FP32_SCREEN = 2 } jsi_precision;

typedef struct jsi_context jsi_context;
typedef int jsi_surface_id;

typedef struct {
  int device;                          /* CUDA device ordinal */
  unsigned long long arena_bytes;      /* device arena of the context; 0 = 2 GiB */
  unsigned long long hbm_budget_bytes; /* cap on arena + resident surfaces; 0 = 120 GiB */
} jsi_config;

/* Replaces init_cad() / deinit_cad() (src/common/common.cu:35-61): the
 * 4 GiB host bump workspace becomes a device arena owned by the context. */
int jsi_create(const jsi_config *cfg, jsi_context **out);
int jsi_destroy(jsi_context *ctx);

const char *jsi_status_string(int status);
/* Text of the last error recorded on ctx (empty string if none). */
const char *jsi_last_error(const jsi_context *ctx);
int jsi_abi_version(void);

/* Copies one surface in EGADS layout (ivec[7] + data, include/nurbs_data.hpp:1-10,
 * decoded as in src/evaluation/evaluation.cu:239-257) to device memory and
 * keeps it resident until released.  Replaces the caller-side
 * allocate_from_workspace + cadMemcpy of ivec/data
 * (examples/intersection_example.cu:50-57).  The copy is asynchronous (the
 * data is staged in pinned memory before the call returns); queries issued
 * afterwards see the surface.  Releases return the device block to the
 * context's pool without synchronising. */
int jsi_surface_upload(jsi_context *ctx, const int ivec[7], const float *data, int ndata, jsi_surface_id *out);
int jsi_surface_release(jsi_context *ctx, jsi_surface_id id);
/* Page-locked host memory owned by the context (freed by jsi_host_free or
 * jsi_destroy).  Surface records that lie in one such block, in increasing
 * address order, 16-byte aligned and not overlapping, are uploaded by
 * jsi_surface_upload_many with one DMA per staging segment straight from it
 * instead of being copied into the pinned staging first.  Those copies are
 * asynchronous: the caller keeps the uploaded records unchanged until the
 * upload has completed on the device (any query result that uses the
 * surfaces, or jsi_host_free, which waits for it). */
int jsi_host_alloc(jsi_context *ctx, unsigned long long bytes, void **ptr);
int jsi_host_free(jsi_context *ctx, void *ptr);

/* n surfaces in one call: ivecs = n x 7 headers, datas[q] / ndatas[q] the
 * records; out[q] gets each id (0 for those not uploaded after an error). */
int jsi_surface_upload_many(jsi_context *ctx, int n, const int *ivecs, const float *const *datas, const int *ndatas,
                            jsi_surface_id *out);
/* n releases in one call (each as jsi_surface_release; stops at the first
 * failing id and returns its status). */
int jsi_surface_release_many(jsi_context *ctx, int n, const jsi_surface_id *ids);
/* Full parameter domains of n resident surfaces: rects[4q..4q+3] =
 * (ustart, vstart, ustop, vstop), the values NurbsFace::get_ubegin,
 * get_vbegin, get_uend, get_vend return (include/nurbs_data.hpp:6-9) and the
 * reference's examples put into EvalAndConstructTask
 * (examples/intersection_example.cu:62-65). */
int jsi_surface_domains(jsi_context *ctx, int n, const jsi_surface_id *ids, float *rects);
/* Resident surface bytes on the device. */
int jsi_resident_bytes(const jsi_context *ctx, unsigned long long *out);

/* --- instrumentation (no counterpart in the reference; its CAD_TIMING /
 * CAD_PROFILE hooks, src/common/profiler.hpp:11-41, time on the host) ---- */
/* The context's CUDA stream (a cudaStream_t) so callers can time it with
 * their own CUDA events. */
int jsi_context_stream(jsi_context *ctx, void **stream);
/* Cumulative host->device and device->host bytes the context has copied. */
int jsi_transfer_bytes(const jsi_context *ctx, unsigned long long *h2d, unsigned long long *d2h);
/* Cumulative number of kernels this library has launched (all contexts). */
int jsi_launch_count(unsigned long long *out);
/* Per-kernel timing: while enabled, every kernel launch of the context is
 * bracketed by CUDA events on its stream.  Enabling or disabling resets the
 * totals.  jsi_kernel_time reads the total milliseconds and launch count of
 * one kernel name; jsi_kernel_names lists the names seen (comma separated). */
int jsi_kernel_timing(jsi_context *ctx, int enable);
int jsi_kernel_time(jsi_context *ctx, const char *name, double *total_ms, long long *launches);
/* Work units the timed launches of one kernel processed: grid lines (basis),
 * samples (samples), cells (cells), tile pairs (dist_tau, dist_cull,
 * inter_cull), executed cell-pair tests (dist_leaf, inter_leaf). */
int jsi_kernel_units(jsi_context *ctx, const char *name, double *units);
const char *jsi_kernel_names(jsi_context *ctx);

/* One query side: EvalAndConstructTask (include/jsi_cad.hpp:11-23) with the
 * surface named by a resident id instead of raw device pointers. */
typedef struct {
  jsi_surface_id surface;
  float ustart, vstart, ustop, vstop;
  int nuv;  /* first-round sampling width */
  int side; /* eval_task_side: 1 or 2 */
} jsi_task;

/* --- minimum distance ---------------------------------------------------
 * Replaces float minimum_distance(const EvalAndConstructTask&,
 * const EvalAndConstructTask&) (include/jsi_cad.hpp:31,
 * src/distance_analysis/distance_analysis.cu:356-506).  Defaults equal the
 * reference statics (:33-36): k = 8, rounds = 4, refinement nuv = 16. */
typedef struct {
  int nuv_refine; /* next_nuv */
  int k;          /* k_of_topk, 1..1024 */
  int rounds;     /* max_layers, 1..JSI_MAX_ROUNDS */
  int precision;  /* jsi_precision */
  int newton;     /* 1: FP64 Levenberg-Marquardt from every final candidate pair to the closest points */
} jsi_dist_params;

typedef struct {
  float v5_value;   /* what minimum_distance returns: sqrt of the last round's k-th d2 */
  double distance;  /* FP64 forms: sqrt of the last round's k-th d2 in FP64; V5_FP32: v5_value */
  double newton_distance;     /* refined true distance (newton = 1), else -1 */
  double uv1[2], uv2[2];      /* closest parameters (newton = 1) */
  double point1[3], point2[3];
  int rounds_run;
  int npairs[JSI_MAX_ROUNDS];        /* pairs kept per round (min(k, #pairs)) */
  double kth_d2[JSI_MAX_ROUNDS];     /* k-th squared centre distance per round */
  long long pair_tests[JSI_MAX_ROUNDS];  /* cell-pair distance tests executed per round */
  long long candidates[JSI_MAX_ROUNDS];  /* pairs that passed the screen, before selection */
  /* Optional trace (caller-owned, may be null): the kept (slot, i, j)
   * triples of every round, round r at trace_pairs[(r*k + q)*3 ...]. */
  int *trace_pairs;
  long long trace_cap; /* capacity in triples; needs rounds*k */
  float device_ms;     /* device time of the query (CUDA events) */
  long long tile_pairs[JSI_MAX_ROUNDS]; /* tile pairs that passed the bound screen per round */
  long long tile_pairs_tested[JSI_MAX_ROUNDS]; /* tile pairs whose bound (or representative) was evaluated */
  long long supertile_pairs[JSI_MAX_ROUNDS];   /* supertile pairs that passed their bound (two-level rounds) */
  /* Optional trace of the first round's screen candidates (caller-owned, may
   * be null; jsi_min_distance only): the (slot, i, j) triples that passed the
   * screen, in no particular order, with each pair's FP64 squared centre
   * distance in cand_d2 (FP64 and FP32_SCREEN forms; V5_FP32: the FP32 value).
   * Every pair whose d2 is at most the round's k-th value is among them.
   * cand_written counts all candidates (also those beyond cand_cap). */
  int *cand_pairs;
  double *cand_d2;
  long long cand_cap;
  long long cand_written;
} jsi_dist_result;

void jsi_dist_params_default(jsi_dist_params *p);
int jsi_min_distance(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_dist_params *params,
                     jsi_dist_result *out);

/* --- surface-surface intersection ----------------------------------------
 * Replaces void intersection(EvalAndConstructTask, EvalAndConstructTask)
 * (include/jsi_cad.hpp:33, src/intersection/intersection.cu:338-475).  The
 * reference keeps its refinement width in a file static that the halving rule
 * mutates across calls (:36, :370); here it is a per-call parameter. */
typedef struct {
  int nuv_refine;      /* global_nuv at call start (16) */
  int use_k;           /* CAD_INTERSECT_USE_K: curvature padding on (1) / off (0) */
  int rounds;          /* 6 */
  int halve_threshold; /* 512 */
  int min_nuv;         /* 4 */
  int precision;       /* jsi_precision */
  int points;          /* 1: refine every final pair to an intersection point (FP64) */
} jsi_inter_params;

typedef struct {
  int rounds_run;
  long long counts[JSI_MAX_ROUNDS];     /* overlap pairs per round ("Round r: overlap pairs = N") */
  long long pair_tests[JSI_MAX_ROUNDS]; /* cell-pair box tests executed per round */
  long long regions1[JSI_MAX_ROUNDS];   /* unique side-1 regions evaluated per round */
  long long regions2[JSI_MAX_ROUNDS];
  double pad[2];                        /* round-1 curvature paddings of side 1 / side 2 */
  /* Optional trace (caller-owned, may be null): every round's (slot, i, j)
   * triples concatenated in round order; trace_written counts all pairs
   * (also those beyond trace_cap). */
  int *trace_pairs;
  long long trace_cap;
  long long trace_written;
  /* Optional intersection points (caller-owned, points = 1): 8 doubles per
   * final pair, in the final round's (slot, i, j) order: x, y, z of the point,
   * (u, v) on surface 1, (s, t) on surface 2, residual |S1 - S2|; a point is
   * counted as converged when residual <= 1e-9 (1 + |x| + |y| + |z|). */
  double *points;
  long long points_cap;
  long long points_written;
  long long points_converged;
  float device_ms;
  /* FP32_SCREEN only (else 0): the first round's FP32 screen.  screen_written
   * counts its candidate (slot, i, j) triples (a superset of the FP64 form's
   * round-1 pairs, which the FP64 re-check then keeps); when screen_pairs is
   * set (caller-owned) up to screen_cap of them are written there in
   * (slot, i, j) order.  kmax_rechecked counts the samples whose curvature
   * terms were re-evaluated in FP64 to get the exact compute_K maxima. */
  int *screen_pairs;
  long long screen_cap;
  long long screen_written;
  long long kmax_rechecked;
} jsi_inter_result;

void jsi_inter_params_default(jsi_inter_params *p);
int jsi_intersect(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_inter_params *params,
                  jsi_inter_result *out);

/* --- certified distance interval (bounds mode) ----------------------------
 * No counterpart in the reference, whose distance is the k-th smallest
 * distance between cell-box centres (distance_analysis.cu:202-207), not a
 * bound.  Returns lb <= (true minimum distance between the two rectangles of
 * the two surfaces) <= ub, rigorously, for non-rational surfaces, by branch
 * and bound on cell boxes of a grid covering both rectangles:
 *  - each box is its corner samples' box padded by the bilinear-interpolation
 *    error bound (du^2 max|S_uu| + dv^2 max|S_vv|) / 8, from the
 *    second-derivative control nets, and by an evaluation allowance; gaps are
 *    rounded down;
 *  - ub starts at the FP64 distance query's Newton pair and drops to the
 *    closest corner-sample pair of the kept cells each round (surface points,
 *    distances rounded up, plus the evaluation allowance);
 *  - pairs whose gap can be below (1 - rel_tol) ub are refined at nuv_refine
 *    per cell; lb is the smaller of the smallest kept gap and
 *    (1 - rel_tol) ub, which every dropped pair's gap exceeds.
 * Rounds stop when ub - lb <= rel_tol * ub or no pair is kept (certified = 1),
 * after max_rounds, or when a round keeps more than max_pairs pairs.  uv1 /
 * uv2 / point1 / point2 are the Newton pair (its distance >= ub).
 * Rational surfaces (positive weights) take the second-derivative bound of
 * the quotient A / w (jsi_surface_curvature_bounds) and an evaluation
 * allowance scaled by 1 / min w; a non-positive weight gives
 * JSI_ERR_UNSUPPORTED. */
typedef struct {
  int nuv_refine;      /* samples per direction in a refined cell (default 8) */
  int max_rounds;      /* 1..JSI_MAX_ROUNDS (default 10) */
  double rel_tol;      /* default 1e-6 */
  long long max_pairs; /* default 1 << 22 */
} jsi_bounds_params;

typedef struct {
  double lb, ub;
  int certified;
  int rounds_run;
  long long kept[JSI_MAX_ROUNDS];       /* cell pairs kept per round */
  long long pair_tests[JSI_MAX_ROUNDS]; /* cell-pair box tests per round */
  double lb_round[JSI_MAX_ROUNDS];      /* lower bound after each round */
  double uv1[2], uv2[2];                /* parameters of the Newton pair */
  double point1[3], point2[3];
  float device_ms;
} jsi_bounds_result;

void jsi_bounds_params_default(jsi_bounds_params *p);
/* Host only (no device work, no context): per coordinate c, upper bounds
 * m2u[c] >= |S_uu[c]| and m2v[c] >= |S_vv[c]| (the record as
 * jsi_surface_upload takes it), the pads of the bounds mode.  rect = NULL:
 * over the whole surface.  rect = {u0, v0, u1, v1}: over that parameter
 * rectangle, as the bounds mode pads a region, the largest of the per-knot-
 * span bounds (each from that span's own control points) over the spans it
 * touches.  Non-rational: the second-derivative control nets.  Rational: the
 * same nets of the homogeneous net (w (P - m), w), m the net's bounding-box
 * centre, combined through S_uu = (A_uu - 2 w_u S_u - w_uu (S - m)) / w with
 * |S - m| <= the net's half range and w >= min w.  Within a span the bound
 * holds everywhere; across a knot where the surface is only C0 S_uu does not
 * exist there (the bounds mode cuts its rectangles at such knots).
 * JSI_ERR_SURFACE for a bad header or length, JSI_ERR_UNSUPPORTED for a
 * non-positive weight. */
int jsi_surface_curvature_bounds(const int *ivec, const float *data, int ndata, const double *rect, double *m2u,
                                 double *m2v);
int jsi_distance_bounds(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_bounds_params *params,
                        jsi_bounds_result *out);

/* --- intersection curves ----------------------------------------------------
 * No counterpart in the reference, which stops at the per-round overlap
 * counts (intersection.cu:467-474); the step after it, and the output of
 * OpenCASCADE's GeomAPI_IntSS that its benchmark compares against
 * (benchmarks/opencascade_compare.cpp:209-219).  Runs the FP64 intersection
 * query with Newton points, sampling every refined cell to its far edge
 * (the reference's grid leaves the last strip of each cell unsampled, which
 * would leave gaps in the points), then links the converged points:
 * tangents t = N1 x N2 on the device, then from a seed point a walk to the
 * nearest unvisited point ahead along the tangent (within link_tol), in both
 * directions; a walk that returns to its seed closes the curve.  Points the
 * walk passes (nearer than the chosen next point and along the curve) join
 * that curve without becoming vertices.
 * Caller buffers: vertex (vertex_cap x 7: x, y, z, u, v, s, t, in curve
 * order), curve_start (curve_cap + 1 offsets), curve_closed (curve_cap).
 * When they are too small the call returns JSI_ERR_CAPACITY with vertices /
 * curves set to the sizes needed. */
typedef struct {
  jsi_inter_params inter; /* the intersection query (precision FP64 is used) */
  double link_tol;        /* largest step between vertices; 0: 4 x the median size of the final cells */
} jsi_curve_params;

typedef struct {
  long long points_found; /* converged intersection points */
  long long vertices;     /* polyline vertices (written, or needed) */
  long long curves;       /* polylines with >= 2 vertices (written, or needed) */
  double link_tol;        /* the tolerance used */
  double *vertex;
  long long vertex_cap;
  long long *curve_start;
  int *curve_closed;
  long long curve_cap;
  float device_ms;
} jsi_curve_result;

void jsi_curve_params_default(jsi_curve_params *p);
int jsi_intersection_curves(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_curve_params *params,
                            jsi_curve_result *out);

/* --- queued and batched queries (the serving engine) ----------------------
 * No counterpart in the reference, whose API runs one query at a time and is
 * not re-entrant (file statics, intersection.cu:36-39).  jsi_workers starts n
 * worker lanes (each: a CUDA stream, a device arena of up to lane_bytes, or
 * an equal share of the HBM budget left beside the resident surfaces when
 * lane_bytes = 0, and a host thread); queued queries run on the first free lane in arrival order
 * and their kernels overlap on the device.  n = 0 stops the pool (only when
 * nothing is queued).  A surface cannot be released while a queued query
 * uses it.  Results of a query are bit-identical whichever lane runs it and
 * whatever runs beside it. */
typedef long long jsi_ticket;
int jsi_workers(jsi_context *ctx, int n, unsigned long long lane_bytes);
/* trace_pairs (may be null) must stay valid until jsi_wait returns. */
int jsi_submit_distance(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_dist_params *params,
                        int *trace_pairs, long long trace_cap, jsi_ticket *out);
int jsi_submit_intersect(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_inter_params *params,
                         int *trace_pairs, long long trace_cap, jsi_ticket *out);
/* Waits up to timeout_ms (< 0: no limit) for a ticket; JSI_ERR_TIMEOUT if it
 * is not done yet (the ticket stays valid), else the query's own status with
 * its result copied to dist or inter. */
int jsi_wait(jsi_context *ctx, jsi_ticket ticket, int timeout_ms, jsi_dist_result *dist, jsi_inter_result *inter);
int jsi_queue_depth(jsi_context *ctx, int *queued, int *running);
/* n distance queries over the worker lanes; status[q] (may be null) gets each
 * query's status, device_ms (may be null) the device span of the batch
 * (CUDA events).  Returns the first error, else JSI_OK.
 * With k <= 8 and rounds <= 8, queries with the same first-round nuv and
 * zero flags of both sides run in lockstep batches of up to jsi_batch_chunk
 * queries per lane: one launch per stage for the whole batch, counts kept on
 * the device, one copy in and one copy out per batch.  Degrees and rational
 * flags may differ within a batch (each query's surfaces are read from its
 * slab; such a mixed batch builds its cells with the kernel that takes any
 * degree).  Results are the same
 * as the per-query path's; a query whose internal lists overflow is re-run
 * alone.  No reference counterpart (V5 runs one query per call,
 * distance_analysis.cu:356). */
int jsi_min_distance_batch(jsi_context *ctx, int n, const jsi_task *a, const jsi_task *b,
                           const jsi_dist_params *params, jsi_dist_result *out, int *status, float *device_ms);
/* jsi_min_distance_batch in two halves, so that the caller can stage and
 * upload the next batch's surfaces while this one runs: submit queues the
 * batch and returns a ticket at once; a, b, out and status must stay valid
 * until jsi_wait_distance_batch(ticket) returns.  The batch starts after the
 * uploads issued before the submit.  device_ms (may be null) is the span
 * from the submission to the end of the batch's last lane job. */
int jsi_submit_distance_batch(jsi_context *ctx, int n, const jsi_task *a, const jsi_task *b,
                              const jsi_dist_params *params, jsi_dist_result *out, int *status, jsi_ticket *ticket);
int jsi_wait_distance_batch(jsi_context *ctx, jsi_ticket ticket, float *device_ms);
/* Whether every lane job of a submitted distance batch has finished (*done =
 * 1; jsi_wait_distance_batch then returns without blocking), without waiting. */
int jsi_poll_distance_batch(jsi_context *ctx, jsi_ticket ticket, int *done);
/* Queries per lockstep batch (default 64; 0: every query runs alone). */
int jsi_batch_chunk(jsi_context *ctx, int chunk);
/* Batch items re-run alone after an internal list overflowed (all lanes). */
int jsi_batch_reruns(jsi_context *ctx, long long *out);
/* Autotuner of the lockstep batches: times jsi_min_distance_batch on the n
 * given queries (all of one shape) for chunk sizes 8, 16, 32, ... up to the
 * per-lane share of n, with the lanes as configured, and keeps the fastest for
 * queries of that shape (first-round nuv, degrees and rational flag of both
 * sides, k, rounds, precision); later batches of the shape use it.  chunk_out / ms_out
 * (may be null) get the choice and its batch device time. */
int jsi_autotune_batch(jsi_context *ctx, int n, const jsi_task *a, const jsi_task *b, const jsi_dist_params *params,
                       int *chunk_out, float *ms_out);
/* When on, lockstep batches that repeat a shape, size and lane are captured
 * once as a CUDA graph and replayed.  enable: 1 on, 0 off (default), -1
 * unchanged; replays (may be null) gets the replay count over all lanes.
 * Off by default: with three worker lanes and uploads running beside them a
 * replay crashed inside cudaGraphLaunch on driver 580. */
int jsi_batch_graphs(jsi_context *ctx, int enable, long long *replays);

/* --- mixed query batches ---------------------------------------------------
 * No counterpart in the reference, which runs one query per call.  n queries
 * of both kinds and any shapes over the worker lanes: kinds[q] = 0 distance
 * (result in dist_out[q], parameters dp), 1 intersection (inter_out[q],
 * parameters ip; its caller-owned trace, points and screen buffers are
 * honoured as by jsi_intersect).  Distance queries run as lockstep batches
 * grouped by first-round nuv (as jsi_min_distance_batch); intersection
 * queries run as lane jobs, the largest first-round grids first.  Every
 * result equals the same query run alone.  status[q] (may be null) gets each
 * query's status, device_ms (may be null) the device span from the call to
 * the end of the last job.  Returns the first error, else JSI_OK. */
int jsi_query_batch(jsi_context *ctx, int n, const int *kinds, const jsi_task *a, const jsi_task *b,
                    const jsi_dist_params *dp, const jsi_inter_params *ip, jsi_dist_result *dist_out,
                    jsi_inter_result *inter_out, int *status, float *device_ms);

/* --- grid evaluation -----------------------------------------------------
 * Replaces evalWithCuda(int*, float*, int, float, float, float, float, int,
 * float*) (include/jsi_cad.hpp:46, src/evaluation/evaluation.cu:391-405):
 * nuv x nuv records of 18 floats (P, Pu, Pv, Puu, Puv, Pvv), sample
 * (idx, idy) at (ustep*idx + ustart, vstep*idy + vstart), record at
 * (idx + idy*nuv)*18.  results is a host pointer. */
int jsi_eval_grid(jsi_context *ctx, const int ivec[7], const float *data, int ndata, float ustep, float vstep,
                  float ustart, float vstart, int nuv, float *results);
/* The same grid in FP64 (data promoted from float). */
int jsi_eval_grid_f64(jsi_context *ctx, const int ivec[7], const float *data, int ndata, double ustep,
                      double vstep, double ustart, double vstart, int nuv, double *results);

/* The FP32 grid of jsi_eval_grid without a context and without allocating
 * any device memory, for callers that cannot call cudaMalloc (a host
 * application whose memory pool owns the whole device, or a loop that cannot
 * take cudaMalloc's implicit synchronisation).  It has no counterpart in the
 * reference.  Works on the current device; every device buffer lives in one
 * fixed 32 MiB __device__ array that each GPU loading this code keeps until
 * exit.  Knots, the control net (16 bytes per point) and the nuv*nuv*18 float
 * records, each rounded up to 256 bytes, must fit in it, else
 * JSI_ERR_CAPACITY; a malformed header or a data length below what the header
 * needs gives JSI_ERR_SURFACE before any device work.  Each call uses the CUDA
 * context current on the calling thread and looks up the array's address in
 * it (cudaGetSymbolAddress, which allocates nothing).  The copies are
 * synchronous, on the legacy default stream: no call may run while any thread
 * of the process is capturing a stream in global capture mode.  All calls
 * share the array: calls whose device work overlaps race; serialise them. */
int jsi_eval_grid_noalloc(const int ivec[7], const float *data, int ndata, float ustep, float vstep, float ustart,
                          float vstart, int nuv, float *results);

#ifdef __cplusplus
}
#endif
#endif /* JSI_B200_H */
