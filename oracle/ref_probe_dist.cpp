// Test-only probe around the reference VERSION5 distance query.
//
// This translation unit is part of the ORACLE (test infrastructure, never the
// product).  It compiles the reference's own distance_analysis.cu from the
// reference tree (the include path is given by oracle/Makefile) so that the
// file-static tuning knobs (k_of_topk, max_layers, next_nuv) and the static
// screening routine dist_collect_top_pairs become reachable, and exports a
// small extern "C" surface for ctypes:
//
//   refp_minimum_distance  - the unmodified minimum_distance()
//                            (JSI_CAD_NEXT_VERSION5/src/distance_analysis/distance_analysis.cu:356-506)
//                            with k / rounds / refine-nuv set through the statics at :33-36.
//   refp_dist_round1       - round-1 cell centres (:88-116) and the round-1
//                            top-k pair list of dist_collect_top_pairs (:246-338).
//   refp_eval_grid         - EG_spline2dDeriv_irrational (evaluation.cu:371-374).
//   refp_compute_k         - compute_K (common/common.cu:149-172).
//
// Nothing here changes the reference's arithmetic; it only feeds it inputs.
#include "distance_analysis/distance_analysis.cu"

#include <atomic>
#include <cstring>

extern std::atomic<size_t> workspace_offset;  // common.cu:19
extern void *workspace;                        // common.cu:17

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

}  // namespace

extern "C" {

// rect = {ustart, vstart, ustop, vstop}
float refp_minimum_distance(const int *ivec1, const float *data1, int nd1, const float *rect1, const int *ivec2,
                            const float *data2, int nd2, const float *rect2, int nuv0, int nuv_refine, int k,
                            int rounds) {
  ensure_init();
  k_of_topk = k;
  max_layers = rounds;
  next_nuv = nuv_refine;
  EvalAndConstructTask t1 = make_task(ivec1, data1, nd1, rect1, nuv0, 1);
  EvalAndConstructTask t2 = make_task(ivec2, data2, nd2, rect2, nuv0, 2);
  float r = minimum_distance(t1, t2);
  k_of_topk = 8;
  max_layers = 4;
  next_nuv = 16;
  return r;
}

// Round-1 screening of the reference.  Writes up to cap pairs (d2, i, j)
// (slot is always 0 in round 1) and the cell centres of both sides
// (3 * (nuv0-1)^2 floats each, may be null).  Returns the pair count.
int refp_dist_round1(const int *ivec1, const float *data1, int nd1, const float *rect1, const int *ivec2,
                     const float *data2, int nd2, const float *rect2, int nuv0, int k, float *d2_out, int *i_out,
                     int *j_out, int cap, float *centers1, float *centers2) {
  ensure_init();
  EvalAndConstructTask t1 = make_task(ivec1, data1, nd1, rect1, nuv0, 1);
  EvalAndConstructTask t2 = make_task(ivec2, data2, nd2, rect2, nuv0, 2);
  DistChain ch;
  ch.side1.push_back(run_evaluation_and_construction_task(t1, 0));
  ch.side2.push_back(run_evaluation_and_construction_task(t2, 0));
  const size_t ncell = static_cast<size_t>(nuv0 - 1) * static_cast<size_t>(nuv0 - 1);
  if (centers1) std::memcpy(centers1, ch.side1[0].d_aabb_center, 3 * ncell * sizeof(float));
  if (centers2) std::memcpy(centers2, ch.side2[0].d_aabb_center, 3 * ncell * sizeof(float));
  k_of_topk = k;
  std::vector<DistPairRef> pairs;
  dist_collect_top_pairs(ch, pairs);
  k_of_topk = 8;
  int n = static_cast<int>(pairs.size());
  for (int q = 0; q < n && q < cap; ++q) {
    d2_out[q] = pairs[q].d2;
    i_out[q] = pairs[q].i;
    j_out[q] = pairs[q].j;
  }
  return n;
}

void refp_eval_grid(const int *ivec, const float *data, float ustep, float vstep, float ustart, float vstart,
                    int nuv, float *results) {
  EG_spline2dDeriv_irrational(const_cast<int *>(ivec), const_cast<float *>(data), ustep, vstep, ustart, vstart, nuv,
                              results);
}

void refp_eval_with_cuda(const int *ivec, const float *data, int ndata, float ustep, float vstep, float ustart,
                         float vstart, int nuv, float *results) {
  evalWithCuda(const_cast<int *>(ivec), const_cast<float *>(data), ndata, ustep, vstep, ustart, vstart, nuv,
               results);
}

float refp_compute_k(const float *results, int nuv) {
  std::vector<float> scratch(static_cast<size_t>(nuv) * nuv * 3);
  float k = 0.0f;
  compute_K(const_cast<float *>(results), scratch.data(), &k, nuv);
  return k;
}

}  // extern "C"
