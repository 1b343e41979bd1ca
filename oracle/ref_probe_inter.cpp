// Test-only probe around the reference VERSION5 intersection query.
//
// ORACLE code (test infrastructure, never the product).  Compiles the
// reference's own intersection.cu from the reference tree so that its file
// statics (global_nuv, initial_u_span/initial_v_span) and the static helpers
// run_evaluation_and_construction_task / intersect_collect_pairs are reachable:
//
//   refp_intersection   - the unmodified intersection()
//                         (JSI_CAD_NEXT_VERSION5/src/intersection/intersection.cu:338-475).
//                         It prints "Round r: overlap pairs = N"; the caller
//                         captures stdout.  global_nuv (:36) is reset before
//                         every call so each call sees fresh-process state.
//   refp_inter_round1   - round-1 boxes (:175-219) and the round-1 overlap
//                         list of intersect_collect_pairs (:259-309).
#include "intersection/intersection.cu"

#include <atomic>
#include <cstring>

extern std::atomic<size_t> workspace_offset;  // common.cu:19

namespace {

bool g_ready = false;

void ensure_init() {
  if (!g_ready) {
    init_cad();
    g_ready = true;
  }
  workspace_offset.store(0);
}

EvalAndConstructTask make_task(const int *ivec, const float *data, int ndata, const float rect[4], int nuv,
                               int side) {
  int *d_ivec = static_cast<int *>(allocate_from_workspace(7 * sizeof(int)));
  float *d_data = static_cast<float *>(allocate_from_workspace(static_cast<size_t>(ndata) * sizeof(float)));
  std::memcpy(d_ivec, ivec, 7 * sizeof(int));
  std::memcpy(d_data, data, static_cast<size_t>(ndata) * sizeof(float));
  EvalAndConstructTask t;
  t.d_ivec = d_ivec;
  t.d_data = d_data;
  t.d_ndata = ndata;
  t.ustart = rect[0];
  t.vstart = rect[1];
  t.ustop = rect[2];
  t.vstop = rect[3];
  t.nuv = nuv;
  t.eval_task_side = side;
  return t;
}

void set_use_k(int use_k) { setenv("CAD_INTERSECT_USE_K", use_k ? "1" : "0", 1); }

}  // namespace

extern "C" {

void refp_intersection(const int *ivec1, const float *data1, int nd1, const float *rect1, const int *ivec2,
                       const float *data2, int nd2, const float *rect2, int nuv0, int nuv_refine, int use_k) {
  ensure_init();
  set_use_k(use_k);
  global_nuv = nuv_refine;
  EvalAndConstructTask t1 = make_task(ivec1, data1, nd1, rect1, nuv0, 1);
  EvalAndConstructTask t2 = make_task(ivec2, data2, nd2, rect2, nuv0, 2);
  intersection(t1, t2);
  std::fflush(stdout);
}

// Round-1 boxes and overlap list.  centers/radii may be null; each holds
// 3 * (nuv0-1)^2 floats.  pads receives the two curvature paddings.
// Returns the number of overlapping pairs (writes at most cap of them).
int refp_inter_round1(const int *ivec1, const float *data1, int nd1, const float *rect1, const int *ivec2,
                      const float *data2, int nd2, const float *rect2, int nuv0, int use_k, int *i_out, int *j_out,
                      int cap, float *centers1, float *radii1, float *centers2, float *radii2) {
  ensure_init();
  set_use_k(use_k);
  EvalAndConstructTask t1 = make_task(ivec1, data1, nd1, rect1, nuv0, 1);
  EvalAndConstructTask t2 = make_task(ivec2, data2, nd2, rect2, nuv0, 2);
  // The span bookkeeping intersection() performs before its first evaluation
  // (intersection.cu:344-347).
  initial_k_prints = 2;  // silence the Compute_K print
  initial_u_span[1] = std::max(std::fabs(t1.ustop - t1.ustart), 1.0e-12f);
  initial_v_span[1] = std::max(std::fabs(t1.vstop - t1.vstart), 1.0e-12f);
  initial_u_span[2] = std::max(std::fabs(t2.ustop - t2.ustart), 1.0e-12f);
  initial_v_span[2] = std::max(std::fabs(t2.vstop - t2.vstart), 1.0e-12f);
  IntersectChain ch;
  ch.side1.push_back(run_evaluation_and_construction_task(t1));
  ch.side2.push_back(run_evaluation_and_construction_task(t2));
  const size_t ncell = static_cast<size_t>(nuv0 - 1) * static_cast<size_t>(nuv0 - 1);
  if (centers1) std::memcpy(centers1, ch.side1[0].d_aabb_center, 3 * ncell * sizeof(float));
  if (radii1) std::memcpy(radii1, ch.side1[0].d_aabb_radius, 3 * ncell * sizeof(float));
  if (centers2) std::memcpy(centers2, ch.side2[0].d_aabb_center, 3 * ncell * sizeof(float));
  if (radii2) std::memcpy(radii2, ch.side2[0].d_aabb_radius, 3 * ncell * sizeof(float));
  std::vector<IntersectPairRef> pairs;
  int n = intersect_collect_pairs(ch, pairs);
  for (int q = 0; q < n && q < cap; ++q) {
    i_out[q] = pairs[q].i;
    j_out[q] = pairs[q].j;
  }
  return n;
}

}  // extern "C"
