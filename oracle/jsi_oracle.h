/* CPU oracle for the NURBS distance / intersection query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library restates the reference VERSION5
 * algorithm on the CPU (templated on float and double) so that the GPU path
 * can be checked against it.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it; the product never does.
 *
 * The float instantiation is pinned bit-for-bit against the reference itself
 * (oracle/_ref, built from the reference sources by oracle/Makefile) by
 * tests/test_oracle_vs_reference.py and the fixtures in tests/golden/.
 * The double instantiation is the plain-FP64 form of the same algorithm.
 *
 * Rect layout everywhere: {ustart, vstart, ustop, vstop}.
 * Pair triples: {slot, i, j} with i a side-1 cell, j a side-2 cell,
 * cell id = iv * (nuv-1) + iu.
 */
#ifndef JSI_ORACLE_H
#define JSI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* 18-value records (P, Pu, Pv, Puu, Puv, Pvv) for an nuv x nuv grid,
 * sample (idx, idy) at u = ustep*idx + ustart, v = vstep*idy + vstart,
 * written at (idx + idy*nuv)*18. */
void orc_eval_grid_f32(const int *ivec, const float *data, float ustep, float vstep, float ustart, float vstart,
                       int nuv, float *out);
void orc_eval_grid_f64(const int *ivec, const float *data, double ustep, double vstep, double ustart, double vstart,
                       int nuv, double *out);

float orc_compute_k_f32(const float *records, int nuv);
double orc_compute_k_f64(const double *records, int nuv);

/* Distance query.  kth_d2[r] = k-th smallest squared centre distance of round
 * r (0 when the round has no pair), npairs[r] = pairs kept in round r,
 * pairs[(r*k + q)*3 + {0,1,2}] = slot, i, j of the q-th kept pair of round r
 * (buffers sized rounds and rounds*k*3).  starts (may be null) receives the
 * Newton start (u, v, s, t) of each pair of the last round (k*4 doubles):
 * the centres of its two cells.  Returns the number of rounds run. */
int orc_dist_query_f32(const int *ivec1, const float *data1, const float *rect1, const int *ivec2,
                       const float *data2, const float *rect2, int nuv0, int nuv_refine, int k, int rounds,
                       float *kth_d2, int *npairs, int *pairs, double *starts);
int orc_dist_query_f64(const int *ivec1, const float *data1, const double *rect1, const int *ivec2,
                       const float *data2, const double *rect2, int nuv0, int nuv_refine, int k, int rounds,
                       double *kth_d2, int *npairs, int *pairs, double *starts);

/* Intersection query.  counts[r] = overlapping pairs in round r; the pair
 * triples of every round are appended to pairs (capacity pair_cap triples;
 * *pairs_written receives how many were stored).  pads receives the two
 * round-1 curvature paddings; starts (may be null, starts_cap pairs) the
 * Newton starts of the last round's pairs.  Returns the number of rounds run,
 * or -1 when a round's pair list would exceed max_pairs (the query is
 * abandoned). */
int orc_inter_query_f32(const int *ivec1, const float *data1, const float *rect1, const int *ivec2,
                        const float *data2, const float *rect2, int nuv0, int nuv_refine, int use_k, int rounds,
                        int halve_threshold, int min_nuv, long long max_pairs, long long *counts, int *pairs,
                        long long pair_cap, long long *pairs_written, float *pads, double *starts,
                        long long starts_cap);
int orc_inter_query_f64(const int *ivec1, const float *data1, const double *rect1, const int *ivec2,
                        const float *data2, const double *rect2, int nuv0, int nuv_refine, int use_k, int rounds,
                        int halve_threshold, int min_nuv, long long max_pairs, long long *counts, int *pairs,
                        long long pair_cap, long long *pairs_written, double *pads, double *starts,
                        long long starts_cap);

/* Cell boxes of one region (round-1 style): centres and radii, 3*(nuv-1)^2
 * each; padding = curvature padding added to every radius. */
void orc_region_cells_f32(const int *ivec, const float *data, const float *rect, int nuv, float padding,
                          float *centers, float *radii);
void orc_region_cells_f64(const int *ivec, const float *data, const double *rect, int nuv, double padding,
                          double *centers, double *radii);

/* FP64 Newton refinement from a start x0 = (u, v, s, t) inside
 * dom = {u0, u1, v0, v1, s0, s1, t0, t1}.
 * orc_newton_distance: Levenberg-Marquardt on |S1 - S2|^2, out = d, u, v, s, t, P1[3], P2[3].
 * orc_newton_point: minimum-norm Gauss-Newton on S1 - S2 = 0,
 *                   out = x, y, z, u, v, s, t, residual. */
void orc_newton_distance(const int *ivec1, const float *data1, const int *ivec2, const float *data2,
                         const double *dom, const double *x0, double *out);
void orc_newton_point(const int *ivec1, const float *data1, const int *ivec2, const float *data2, const double *dom,
                      const double *x0, double *out);

#ifdef __cplusplus
}
#endif
#endif
