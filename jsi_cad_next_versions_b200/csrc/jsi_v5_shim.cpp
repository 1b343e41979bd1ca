// libjsi_v5_shim.so: the reference's C++ query API (JSI_CAD_NEXT VERSION5,
// include/jsi_cad.hpp:11-46 and src/common/common.cuh:17-35) implemented over
// the C ABI of libjsi_b200, so that programs written against the reference —
// its own examples/*_example.cu included — link against this library
// unchanged and run on the GPU.
//
// The struct and enum below restate the reference's interface types with the
// same names and member layout (they have to match for the C++ symbols and
// the callers' objects to agree); nothing else of the reference is used.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "jsi_b200.h"

// include/jsi_cad.hpp:11-23
struct EvalAndConstructTask {
  int *d_ivec;
  float *d_data;
  int d_ndata;
  float ustart;
  float vstart;
  float ustop;
  float vstop;
  int nuv;
  int eval_task_side;
};

// src/common/common.cuh:11
enum class CadMemcpyKind { HostToDevice, DeviceToHost, DeviceToDevice };

namespace {

jsi_context *g_ctx = nullptr;
std::mutex g_mu;
// The reference's workspace is host memory the caller fills with ivec/data
// (examples/intersection_example.cu:50-57); here it stays on the host and the
// query uploads the surfaces it is given.
unsigned char *g_ws = nullptr;
size_t g_ws_size = 4ull << 30;
size_t g_ws_off = 0;
// intersection.cu:36: the refinement width persists across calls and the
// halving rule (:370) mutates it.
int g_global_nuv = 16;

jsi_context *ctx() {
  if (!g_ctx) {
    jsi_config cfg = {0, 0, 0};
    const int st = jsi_create(&cfg, &g_ctx);
    if (st != JSI_OK) {
      std::printf("jsi_create failed: %s\n", jsi_status_string(st));
      std::exit(1);
    }
  }
  return g_ctx;
}

void check(int st, const char *what) {
  if (st != JSI_OK) {
    std::printf("%s failed: %s (%s)\n", what, jsi_status_string(st), jsi_last_error(g_ctx));
    std::exit(1);
  }
}

jsi_task upload(const EvalAndConstructTask &t, jsi_surface_id *id) {
  check(jsi_surface_upload(ctx(), t.d_ivec, t.d_data, t.d_ndata, id), "surface upload");
  jsi_task r;
  r.surface = *id;
  r.ustart = t.ustart;
  r.vstart = t.vstart;
  r.ustop = t.ustop;
  r.vstop = t.vstop;
  r.nuv = t.nuv;
  r.side = t.eval_task_side;
  return r;
}

}  // namespace

// src/common/common.cu:35-49
void init_cad() {
  std::lock_guard<std::mutex> lk(g_mu);
  ctx();
  if (!g_ws) {
    g_ws = static_cast<unsigned char *>(std::malloc(g_ws_size));
    if (!g_ws) {
      std::printf("alloc workspace failed\n");
      std::exit(1);
    }
  }
  g_ws_off = 0;
}

// src/common/common.cu:51-61
void deinit_cad() {
  std::lock_guard<std::mutex> lk(g_mu);
  std::free(g_ws);
  g_ws = nullptr;
  g_ws_off = 0;
  if (g_ctx) {
    jsi_destroy(g_ctx);
    g_ctx = nullptr;
  }
}

// src/common/common.cu:25-33 (256-byte aligned bump; nullptr when exhausted)
void *allocate_from_workspace(size_t size) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (size % 256 != 0) size += 256 - size % 256;
  if (!g_ws || g_ws_off + size > g_ws_size) {
    std::printf("Error: Out of workspace memory!\n");
    return nullptr;
  }
  void *p = g_ws + g_ws_off;
  g_ws_off += size;
  return p;
}

// src/common/common.cu:63-126: the workspace is host memory, so these are host copies.
int cadMemcpy(void *dst, const void *src, size_t size, CadMemcpyKind kind) {
  (void)kind;
  if (size) std::memcpy(dst, src, size);
  return 0;
}

int cadMemset(void *ptr, int value, size_t size) {
  if (size) std::memset(ptr, value, size);
  return 0;
}

int cadMalloc(void **ptr, size_t size) {
  if (!ptr) return -1;
  *ptr = size ? std::malloc(size) : nullptr;
  return (size && !*ptr) ? -1 : 0;
}

int cadFree(void *ptr) {
  std::free(ptr);
  return 0;
}

bool cadIsAclEnabled() { return false; }

// src/distance_analysis/distance_analysis.cu:356-506
float minimum_distance(const EvalAndConstructTask &t1, const EvalAndConstructTask &t2) {
  std::lock_guard<std::mutex> lk(g_mu);
  jsi_surface_id a, b;
  jsi_task ta = upload(t1, &a), tb = upload(t2, &b);
  jsi_dist_params p;
  jsi_dist_params_default(&p);
  jsi_dist_result r;
  std::memset(&r, 0, sizeof(r));
  const int st = jsi_min_distance(g_ctx, &ta, &tb, &p, &r);
  jsi_surface_release(g_ctx, a);
  jsi_surface_release(g_ctx, b);
  check(st, "minimum_distance");
  for (int q = 0; q < r.rounds_run; ++q) {
    std::printf("Round: %d (pair refine)\n", q + 1);
    std::printf("[current_min_dist] %lf\n", static_cast<double>(std::sqrt(static_cast<float>(r.kth_d2[q]))));
    std::printf("  pairs to refine: %d\n", r.npairs[q]);
  }
  return r.v5_value;
}

// src/intersection/intersection.cu:338-475
void intersection(EvalAndConstructTask t1, EvalAndConstructTask t2) {
  std::lock_guard<std::mutex> lk(g_mu);
  jsi_surface_id a, b;
  jsi_task ta = upload(t1, &a), tb = upload(t2, &b);
  jsi_inter_params p;
  jsi_inter_params_default(&p);
  const char *k = std::getenv("CAD_INTERSECT_USE_K");
  p.use_k = (k == nullptr || std::strcmp(k, "0") != 0) ? 1 : 0;
  p.nuv_refine = g_global_nuv;
  jsi_inter_result r;
  std::memset(&r, 0, sizeof(r));
  const int st = jsi_intersect(g_ctx, &ta, &tb, &p, &r);
  jsi_surface_release(g_ctx, a);
  jsi_surface_release(g_ctx, b);
  check(st, "intersection");
  std::printf("Compute_K AABB padding: %s\n", p.use_k ? "on" : "off");
  int nuv = g_global_nuv;
  for (int q = 0; q < r.rounds_run; ++q) {
    std::printf("Round: %d (pair refine)\n", q + 1);
    std::printf("Round %d: overlap pairs = %lld\n", q + 1, r.counts[q]);
    // replay the halving rule to carry the width into the next call
    if (q + 1 < r.rounds_run && r.counts[q] > p.halve_threshold && nuv > p.min_nuv) nuv /= 2;
  }
  g_global_nuv = nuv;
  std::fflush(stdout);
}

// src/evaluation/evaluation.cu:391-405
void evalWithCuda(int *ivec, float *data, int ndata, float ustep, float vstep, float ustart, float vstart, int nuv,
                  float *results) {
  std::lock_guard<std::mutex> lk(g_mu);
  check(jsi_eval_grid(ctx(), ivec, data, ndata, ustep, vstep, ustart, vstart, nuv, results), "evalWithCuda");
}
