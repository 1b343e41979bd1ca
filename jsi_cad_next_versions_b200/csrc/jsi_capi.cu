// Host orchestration and C ABI of libjsi_b200.
//
// One context = one CUDA stream + one device arena (a chain of cudaMalloc'd
// blocks reused across queries, rewound at the start of each query: the
// B200 counterpart of the reference's 4 GiB bump workspace,
// src/common/common.cu:17-33) + the resident surfaces.
//
// A query runs its refinement rounds on the device; the host reads one small
// stats record per round (pair count, unique-region counts) to size the next
// round, exactly where the reference's round loop decides
// (distance_analysis.cu:375-392, intersection.cu:359-370).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "jsi_b200.h"
#include "jsi_internal.h"

using namespace jsi;

namespace {

struct CudaError {
  cudaError_t err;
  const char *what;
  int line;
};

#define JSI_CUDA(call)                                 \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) throw CudaError{e_, #call, __LINE__}; \
  } while (0)

struct StatusError {
  int status;
  std::string msg;
};

[[noreturn]] void fail(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw StatusError{status, buf};
}

// Device arena: blocks are kept across queries and rewound by reset().  All
// arenas of a context draw on one shared budget (bytes held across lanes), so
// a heavy query can grow beyond an even share while the others are small;
// trim() hands blocks beyond a lane's steady size back after such a query.
class Arena {
 public:
  Arena() = default;
  Arena(const Arena &) = delete;
  Arena &operator=(const Arena &) = delete;
  ~Arena() { release_all(); }
  void configure(size_t block_bytes, size_t budget, std::atomic<size_t> *shared = nullptr, size_t shared_cap = 0) {
    block_bytes_ = block_bytes;
    budget_ = budget;
    shared_ = shared;
    shared_cap_ = shared_cap;
  }
  void reset() {
    for (auto &b : blocks_) b.used = 0;
    cur_ = 0;
  }
  void *alloc(size_t bytes) {
    bytes = (bytes + 255) & ~static_cast<size_t>(255);
    if (bytes == 0) bytes = 256;
    while (cur_ < blocks_.size()) {
      Block &b = blocks_[cur_];
      if (b.used + bytes <= b.size) {
        void *p = b.base + b.used;
        b.used += bytes;
        return p;
      }
      ++cur_;
    }
    const size_t sz = std::max(block_bytes_, bytes);
    if (total_ + sz > budget_) fail(JSI_ERR_NOMEM, "device arena budget exhausted (%zu + %zu > %zu bytes)", total_, sz, budget_);
    if (shared_) {
      const size_t before = shared_->fetch_add(sz);
      if (before + sz > shared_cap_) {
        shared_->fetch_sub(sz);
        fail(JSI_ERR_NOMEM, "HBM budget of the context exhausted (%zu + %zu > %zu bytes)", before, sz, shared_cap_);
      }
    }
    char *p = nullptr;
    if (cudaMalloc(&p, sz) != cudaSuccess) {
      cudaGetLastError();
      if (shared_) shared_->fetch_sub(sz);
      fail(JSI_ERR_NOMEM, "cudaMalloc of %zu bytes failed", sz);
    }
    blocks_.push_back({p, sz, bytes});
    total_ += sz;
    cur_ = blocks_.size() - 1;
    return p;
  }
  template <typename U>
  U *get(size_t n) {
    return static_cast<U *>(alloc(n * sizeof(U)));
  }
  size_t held() const { return total_; }
  // Frees whole blocks from the back until at most keep bytes are held (the
  // lane's stream must be idle).
  void trim(size_t keep) {
    while (!blocks_.empty() && total_ > keep) {
      Block b = blocks_.back();
      blocks_.pop_back();
      cudaFree(b.base);
      total_ -= b.size;
      if (shared_) shared_->fetch_sub(b.size);
    }
    cur_ = 0;
  }

 private:
  void release_all() {
    for (auto &b : blocks_) {
      cudaFree(b.base);
      if (shared_) shared_->fetch_sub(b.size);
    }
    blocks_.clear();
    total_ = 0;
  }
  struct Block {
    char *base;
    size_t size;
    size_t used;
  };
  std::vector<Block> blocks_;
  size_t cur_ = 0;
  size_t block_bytes_ = size_t(2) << 30;
  size_t budget_ = size_t(120) << 30;
  size_t total_ = 0;
  std::atomic<size_t> *shared_ = nullptr;
  size_t shared_cap_ = 0;
};

struct SurfaceRec {
  int ivec[7];
  int zero, rat, du, dv;
  double cmax[3] = {0, 0, 0};   // max |control point coordinate|
  double wcmax[3] = {0, 0, 0};  // max |w * control point coordinate| (rational)
  double wmin = 1, wmax = 1;    // weight range (rational)
  float dom[4] = {0, 0, 0, 0};  // parameter domain (ustart, vstart, ustop, vstop)
  float *U32 = nullptr, *V32 = nullptr;
  double *U64 = nullptr, *V64 = nullptr;
  Vec4<float> *cpw32 = nullptr;
  Vec4<double> *cpw64 = nullptr;
  size_t bytes = 0;
  char *block = nullptr;  // pooled device block of a resident surface
  size_t block_bytes = 0;
};

// Device blocks of resident surfaces: power-of-two size classes carved from
// 64 MiB slabs (blocks above a slab get a slab of their own), recycled
// through per-class free lists, so uploads and releases allocate nothing in
// steady state and never synchronise the device.
class SurfacePool {
 public:
  ~SurfacePool() {
    for (char *p : slabs_) cudaFree(p);
  }
  static size_t class_bytes(size_t bytes) {
    size_t c = 4096;
    while (c < bytes) c <<= 1;
    return c;
  }
  char *get(size_t bytes) {
    const size_t c = class_bytes(bytes);
    auto &fl = free_[c];
    if (!fl.empty()) {
      char *p = fl.back();
      fl.pop_back();
      return p;
    }
    if (c > kSlab) return new_slab(c);
    if (!cur_ || left_ < c) {
      cur_ = new_slab(kSlab);
      left_ = kSlab;
    }
    char *p = cur_;
    cur_ += c;
    left_ -= c;
    return p;
  }
  void put(char *p, size_t bytes) { free_[class_bytes(bytes)].push_back(p); }

 private:
  static constexpr size_t kSlab = size_t(64) << 20;
  char *new_slab(size_t bytes) {
    char *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      fail(JSI_ERR_NOMEM, "cudaMalloc of %zu bytes for resident surfaces failed", bytes);
    }
    slabs_.push_back(p);
    return p;
  }
  std::vector<char *> slabs_;
  std::map<size_t, std::vector<char *>> free_;
  char *cur_ = nullptr;
  size_t left_ = 0;
};

// Pinned staging of surface uploads: kRingSegs segments used in turn; an
// event recorded when a segment is left guards its reuse.
constexpr int kRingSegs = 8;
constexpr size_t kRingSeg = size_t(8) << 20;

}  // namespace

namespace {

class HostPool;

// One execution lane: a CUDA stream with its own device arena, stats record,
// transfer counters and optional kernel timing.  The context owns a main lane
// for synchronous calls and worker lanes for queued and batched queries, whose
// kernels overlap on the device.
struct Lane {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  Arena arena;
  ScreenStats *d_stats = nullptr;
  ScreenStats *h_stats = nullptr;
  // Pinned words for the few scalars read back per round (dedup tail counts,
  // curvature pads): queued behind the kernels and drained by one sync,
  // instead of one staged pageable copy each.
  unsigned long long *h_small = nullptr;
  unsigned long long h2d_bytes = 0, d2h_bytes = 0;
  // Optional per-kernel timing: CUDA events recorded on the lane's stream
  // around every launch, resolved at the next host sync.  The lane's thread
  // writes the timing state while the caller's thread turns timing on or off
  // and reads the totals, so timing, event_pool, pending, kernel_ms and
  // kernel_units are only touched under stats_mu (timing itself is atomic so
  // that the untimed launch path takes no lock).
  std::mutex stats_mu;
  std::atomic<bool> timing{false};
  std::vector<cudaEvent_t> event_pool;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::map<std::string, std::pair<double, long long>> kernel_ms;
  std::map<std::string, double> kernel_units;  // work units (samples, tile pairs, pair tests, ...)
  const std::map<int, SurfaceRec> *surfaces = nullptr;
  // Worker lanes: the context mutex that guards the surface table (uploads
  // and releases on the calling thread change it while lanes run).  Null for
  // the main lane, whose callers hold it already.
  std::mutex *surfaces_mu = nullptr;
  char *h_pin = nullptr;  // pinned staging of batch heads / records / points
  // The context's host threads (main lane only: its callers hold the context
  // mutex, as the upload path that shares them does); null on worker lanes.
  HostPool *hpool = nullptr;
  size_t h_pin_bytes = 0;
  long long batch_reruns = 0;  // batch items re-run alone after an overflow
  // Lockstep batches replayed as CUDA graphs, keyed by everything their
  // launch sequence depends on (see run_distance_batch).
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    unsigned long long nodes = 0;
    unsigned long long last_use = 0;
    int seen = 0;
  };
  std::map<std::vector<long long>, GraphEntry> graphs;
  unsigned long long graph_clock = 0;
  std::atomic<long long> graph_replays{0};
  std::atomic<bool> graphs_on{false};  // set by the caller's thread, read by the lane's
  // True while the lane's stream captures a graph: per-kernel timing then
  // stays off even if the caller turns it on meanwhile (events recorded into
  // a graph cannot be timed).
  bool capturing = false;
};

// One query of a batch: its tasks, the caller's result slot and its status
// (JSI_OK, or the error of its solo re-run).
struct BatchItem {
  const jsi_task *a = nullptr, *b = nullptr;
  jsi_dist_result *out = nullptr;
  int status = JSI_OK;
  std::string error;
};

// A queued query (or lockstep batch of distance queries) of the worker pool.
struct Job {
  int kind = 0;  // 0 distance, 1 intersection, 2 distance batch (items)
  jsi_task a{}, b{};
  jsi_dist_params dp{};
  jsi_inter_params ip{};
  jsi_dist_result dres{};
  jsi_inter_result ires{};
  std::vector<BatchItem> items;
  int status = JSI_OK;
  std::string error;
  bool done = false;
  cudaEvent_t end_ev = nullptr;  // recorded on the lane's stream after the job's work
  Job() = default;
  Job(const Job &) = delete;
  Job &operator=(const Job &) = delete;
  ~Job() {
    if (end_ev) cudaEventDestroy(end_ev);
  }
};

// A distance batch between its submission and its wait: the lane jobs (and
// tickets of queries run alone), where the results go, and the start event.
struct PendingBatch {
  std::vector<long long> tickets;
  std::vector<std::shared_ptr<Job>> batch_jobs;
  std::vector<std::shared_ptr<Job>> all_jobs;  // every job, for the device span
  std::vector<int> solo;  // query index of each ticket of a per-query job (-1: batch job)
  jsi_dist_result *out = nullptr;
  int *status = nullptr;
  int first_err = 0;
  cudaEvent_t ev0 = nullptr;
  PendingBatch() = default;
  PendingBatch(const PendingBatch &) = delete;
  PendingBatch &operator=(const PendingBatch &) = delete;
  ~PendingBatch() {
    if (ev0) cudaEventDestroy(ev0);
  }
};

}  // namespace

namespace {

// A few host threads kept for the upload path's per-surface work (header
// checks, staging copies), so a parallel loop costs a wake-up rather than
// thread creation.  run() is called with the context mutex held (one caller
// at a time); the calling thread takes part.
class HostPool {
 public:
  explicit HostPool(int n) {
    for (int i = 0; i < n; ++i) th_.emplace_back([this] { loop(); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  void run(size_t n, const std::function<void(size_t)> &fn) {
    std::unique_lock<std::mutex> lk(mu_);
    fn_ = &fn;
    n_ = n;
    next_.store(0);
    active_ = th_.size();
    ++gen_;
    lk.unlock();
    cv_.notify_all();
    work();
    lk.lock();
    done_.wait(lk, [&] { return active_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (size_t q; (q = next_.fetch_add(1)) < n_;) (*fn_)(q);
  }
  void loop() {
    unsigned long long seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
      if (stop_) return;
      seen = gen_;
      lk.unlock();
      work();
      lk.lock();
      if (--active_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(size_t)> *fn_ = nullptr;
  size_t n_ = 0;
  std::atomic<size_t> next_{0};
  size_t active_ = 0;
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

}  // namespace

struct jsi_context {
  int device = 0;
  Lane main;
  std::mutex mu;  // serialises the main lane, the upload path and the surface table
  // The part of the surface table worker lanes touch (surfaces, surface_refs,
  // upload_ev).  Writers hold it beside mu (mu first); a worker takes it
  // alone, so a bulk upload staging on host threads under mu does not hold
  // up the lanes running queries over surfaces already resident.
  std::mutex surf_mu;
  std::string last_error;
  std::map<int, SurfaceRec> surfaces;
  std::map<int, int> surface_refs;  // queued / running jobs per surface
  int next_id = 1;
  size_t budget = size_t(120) << 30;
  size_t lane_bytes = 0;  // 0: lanes draw on the shared budget
  std::atomic<size_t> lane_held{0};  // arena bytes held by all worker lanes
  size_t lane_keep = 0;              // steady arena size a lane keeps after a query
  size_t resident = 0;
  SurfacePool pool;
  char *ring = nullptr;   // pinned staging
  char *dring = nullptr;  // its device mirror (records + prep jobs)
  int ring_cur = 0;
  size_t ring_off = 0;
  cudaEvent_t ring_ev[kRingSegs] = {};
  cudaEvent_t upload_ev = nullptr;  // recorded after every upload (lanes wait on it)
  int batch_chunk = 64;  // queries per lockstep batch (0: one query per lane job)
  // Chunk sizes chosen by jsi_autotune_batch per shape: first-round nuv and
  // basis stride of both sides, k, rounds, precision.
  std::map<std::array<int, 7>, int> tuned_chunk;
  // Replay repeated lockstep batches as CUDA graphs (off by default: with
  // three worker lanes and uploads running beside them, a replay crashed
  // inside cudaGraphLaunch on this driver).
  bool batch_graphs = false;
  std::string kernel_names;
  // worker pool
  std::vector<std::unique_ptr<Lane>> lanes;
  std::vector<std::thread> threads;
  std::mutex qmu;
  std::condition_variable qcv, dcv;
  std::deque<std::shared_ptr<Job>> queue;
  std::map<long long, std::shared_ptr<Job>> jobs;
  std::map<long long, std::unique_ptr<PendingBatch>> batches;  // submitted, not yet waited for
  long long next_ticket = 1;
  int busy = 0;
  bool stopping = false;
  std::unique_ptr<HostPool> hpool;  // upload path host threads
  // Page-locked host blocks handed out by jsi_host_alloc (base -> bytes):
  // surface records inside one are uploaded by DMA straight from it.
  std::map<uintptr_t, size_t> host_blocks;
};

namespace {

int record(jsi_context *ctx, int status, const std::string &msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

template <typename Fn>
int guarded(jsi_context *ctx, Fn &&fn) {
  try {
    return fn();
  } catch (const StatusError &e) {
    return record(ctx, e.status, e.msg);
  } catch (const CudaError &e) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at line %d", static_cast<int>(e.err),
             cudaGetErrorString(e.err), e.what, e.line);
    return record(ctx, JSI_ERR_CUDA, buf);
  } catch (const std::bad_alloc &) {
    return record(ctx, JSI_ERR_NOMEM, "host allocation failed");
  }
}

// cudaMemcpyAsync that also counts the bytes crossing PCIe / C2C.
cudaError_t copy_async(Lane *ctx, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind,
                       cudaStream_t st) {
  if (kind == cudaMemcpyHostToDevice) ctx->h2d_bytes += bytes;
  if (kind == cudaMemcpyDeviceToHost) ctx->d2h_bytes += bytes;
  return cudaMemcpyAsync(dst, src, bytes, kind, st);
}

template <typename T>
SurfView<T> view(const SurfaceRec &s);
template <>
SurfView<float> view<float>(const SurfaceRec &s) {
  SurfView<float> v;
  v.degu = s.ivec[1];
  v.ncpu = s.ivec[2];
  v.nku = s.ivec[3];
  v.degv = s.ivec[4];
  v.ncpv = s.ivec[5];
  v.nkv = s.ivec[6];
  v.rat = s.rat;
  v.zero = s.zero;
  v.du = s.du;
  v.dv = s.dv;
  v.U = s.U32;
  v.V = s.V32;
  v.cpw = s.cpw32;
  return v;
}
template <>
SurfView<double> view<double>(const SurfaceRec &s) {
  SurfView<double> v;
  v.degu = s.ivec[1];
  v.ncpu = s.ivec[2];
  v.nku = s.ivec[3];
  v.degv = s.ivec[4];
  v.ncpv = s.ivec[5];
  v.nkv = s.ivec[6];
  v.rat = s.rat;
  v.zero = s.zero;
  v.du = s.du;
  v.dv = s.dv;
  v.U = s.U64;
  v.V = s.V64;
  v.cpw = s.cpw64;
  return v;
}

int p1_of(const SurfaceRec &s) { return std::max(s.ivec[1], s.ivec[4]) + 1; }

// What of a surface decides the kernels of a lockstep batch: both degrees,
// the rational flag and the zero flag (all queries of a batch share it).
int shape_of(const SurfaceRec &s) { return s.ivec[1] | (s.ivec[4] << 8) | (s.rat << 16) | (s.zero << 17); }

// Header validation.  Degrees >= 25 and non-flat surfaces with flags bits 2|3
// are accepted and evaluate to zero records, as the reference does
// (evaluation.cu:271-272).
void check_surface(const int ivec[7], const float *data, int ndata) {
  if (!ivec || !data) fail(JSI_ERR_INVALID, "null surface pointer");
  const int degu = ivec[1], ncpu = ivec[2], nku = ivec[3], degv = ivec[4], ncpv = ivec[5], nkv = ivec[6];
  if (degu < 0 || degv < 0 || ncpu < 1 || ncpv < 1) fail(JSI_ERR_SURFACE, "bad degree / control net size");
  if (ncpu < degu + 1 || ncpv < degv + 1) fail(JSI_ERR_SURFACE, "control net smaller than degree + 1");
  if (nku != ncpu + degu + 1 || nkv != ncpv + degv + 1) fail(JSI_ERR_SURFACE, "knot count != nCP + degree + 1");
  const long long ncp = static_cast<long long>(ncpu) * ncpv;
  const long long need = nku + nkv + 3 * ncp + ((ivec[0] & 2) ? ncp : 0);
  if (ndata < need) fail(JSI_ERR_SURFACE, "ndata %d < %lld required by the header", ndata, need);
}

// Header fields and the per-surface magnitudes the FP32-screen error bound
// needs (max |coordinate|, max |w coordinate|, weight range).
void surface_header(SurfaceRec &s, const int ivec[7], const float *data) {
  std::memcpy(s.ivec, ivec, sizeof(s.ivec));
  const int flags = ivec[0];
  s.rat = (flags & 2) ? 1 : 0;
  s.zero = ((!(flags & 1)) && (flags & 12)) || ivec[1] >= kMaxDeg || ivec[4] >= kMaxDeg;
  s.du = std::min(2, ivec[1]);
  s.dv = std::min(2, ivec[4]);
  s.dom[0] = data[0];
  s.dom[1] = data[ivec[3]];
  s.dom[2] = data[ivec[3] - 1];
  s.dom[3] = data[ivec[3] + ivec[6] - 1];
  const size_t ncp = static_cast<size_t>(ivec[2]) * ivec[5];
  const float *cp = data + ivec[3] + ivec[6];
  // Branch-free loops in float (|x| and max are exact, and so is the
  // conversion to double); the weighted products of two floats are exact in
  // double.
  float m[3] = {0.0f, 0.0f, 0.0f};
  for (size_t q = 0; q < ncp; ++q) {
    m[0] = std::max(m[0], std::fabs(cp[3 * q]));
    m[1] = std::max(m[1], std::fabs(cp[3 * q + 1]));
    m[2] = std::max(m[2], std::fabs(cp[3 * q + 2]));
  }
  for (int c = 0; c < 3; ++c) s.cmax[c] = s.wcmax[c] = m[c];
  s.wmin = s.wmax = 1.0;
  if (s.rat && ncp > 0) {
    const float *w = cp + 3 * ncp;
    float lo = w[0], hi = w[0];
    double wm[3] = {0.0, 0.0, 0.0};
    for (size_t q = 0; q < ncp; ++q) {
      lo = std::min(lo, w[q]);
      hi = std::max(hi, w[q]);
      for (int c = 0; c < 3; ++c)
        wm[c] = std::max(wm[c], std::fabs(static_cast<double>(w[q]) * static_cast<double>(cp[3 * q + c])));
    }
    s.wmin = lo;
    s.wmax = hi;
    for (int c = 0; c < 3; ++c) s.wcmax[c] = wm[c];
  }
}

// Runs fn(q) for q in [0, n) on the context's host threads (the upload
// path's per-surface work), or inline without them.
void parallel_for(HostPool *pool, size_t n, const std::function<void(size_t)> &fn) {
  if (pool && n > 1) {
    pool->run(n, fn);
    return;
  }
  for (size_t q = 0; q < n; ++q) fn(q);
}

SurfaceRec upload_surface(Lane *ctx, const int ivec[7], const float *data, int ndata, Arena *arena) {
  check_surface(ivec, data, ndata);
  SurfaceRec s;
  surface_header(s, ivec, data);
  const int nku = ivec[3], nkv = ivec[6];
  const size_t ncp = static_cast<size_t>(ivec[2]) * ivec[5];
  const float *cp = data + nku + nkv;
  std::vector<Vec4<float>> c32(ncp);
  std::vector<Vec4<double>> c64(ncp);
  std::vector<double> u64(data, data + nku), v64(data + nku, data + nku + nkv);
  for (size_t q = 0; q < ncp; ++q) {
    const float w = s.rat ? cp[3 * ncp + q] : 1.0f;
    c32[q] = {cp[3 * q], cp[3 * q + 1], cp[3 * q + 2], w};
    c64[q] = {cp[3 * q], cp[3 * q + 1], cp[3 * q + 2], w};
  }
  s.bytes = nku * 12 + nkv * 12 + ncp * (sizeof(Vec4<float>) + sizeof(Vec4<double>));
  auto dalloc = [&](size_t bytes) -> void * {
    if (arena) return arena->alloc(bytes);
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      fail(JSI_ERR_NOMEM, "cudaMalloc for a surface failed");
    }
    return p;
  };
  s.U32 = static_cast<float *>(dalloc(nku * sizeof(float)));
  s.V32 = static_cast<float *>(dalloc(nkv * sizeof(float)));
  s.U64 = static_cast<double *>(dalloc(nku * sizeof(double)));
  s.V64 = static_cast<double *>(dalloc(nkv * sizeof(double)));
  s.cpw32 = static_cast<Vec4<float> *>(dalloc(ncp * sizeof(Vec4<float>)));
  s.cpw64 = static_cast<Vec4<double> *>(dalloc(ncp * sizeof(Vec4<double>)));
  cudaStream_t st = ctx->stream;
  JSI_CUDA(copy_async(ctx, s.U32, data, nku * sizeof(float), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, s.V32, data + nku, nkv * sizeof(float), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, s.U64, u64.data(), nku * sizeof(double), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, s.V64, v64.data(), nkv * sizeof(double), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, s.cpw32, c32.data(), ncp * sizeof(Vec4<float>), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, s.cpw64, c64.data(), ncp * sizeof(Vec4<double>), cudaMemcpyHostToDevice, st));
  JSI_CUDA(cudaStreamSynchronize(st));
  return s;
}

// The returned record stays valid while a job holds the surface: std::map
// nodes do not move on other insertions, and a surface a queued or running
// job refers to cannot be released.
const SurfaceRec &get_surface(Lane *ctx, jsi_surface_id id) {
  std::unique_lock<std::mutex> lk;
  if (ctx->surfaces_mu) lk = std::unique_lock<std::mutex>(*ctx->surfaces_mu);
  auto it = ctx->surfaces->find(id);
  if (it == ctx->surfaces->end()) fail(JSI_ERR_INVALID, "unknown surface id %d", id);
  return it->second;
}

}  // namespace

namespace {

// Resident uploads on the main stream without a host sync.  Records (and
// the prep jobs) are packed into the current segment of the pinned ring,
// copied in one piece to the segment's device mirror, and one prep launch
// writes every surface's block (record, FP64 knots, nets).  upload_ev marks
// the point that worker lanes wait for.  A record larger than a segment goes
// through a temporary device buffer and completes before returning.
struct PendingSurface {
  const int *ivec;
  const float *data;
  int ndata;
};

SurfaceRec make_block(jsi_context *ctx, const SurfaceRec &head, const int ivec[7], int ndata, SurfacePrep *job) {
  SurfaceRec s = head;
  const int nku = ivec[3], nkv = ivec[6];
  const size_t ncp = static_cast<size_t>(ivec[2]) * ivec[5];
  auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  const size_t raw_b = al(static_cast<size_t>(ndata) * sizeof(float));
  const size_t u64_b = al(nku * sizeof(double)), v64_b = al(nkv * sizeof(double));
  const size_t c32_b = al(ncp * sizeof(Vec4<float>)), c64_b = al(ncp * sizeof(Vec4<double>));
  const size_t total = raw_b + u64_b + v64_b + c32_b + c64_b;
  if (ctx->resident + SurfacePool::class_bytes(total) > ctx->budget)
    fail(JSI_ERR_NOMEM, "HBM budget exhausted by resident surfaces");
  char *blk = ctx->pool.get(total);
  s.block = blk;
  s.block_bytes = total;
  s.bytes = SurfacePool::class_bytes(total);
  s.U32 = reinterpret_cast<float *>(blk);
  s.V32 = s.U32 + nku;
  s.U64 = reinterpret_cast<double *>(blk + raw_b);
  s.V64 = reinterpret_cast<double *>(blk + raw_b + u64_b);
  s.cpw32 = reinterpret_cast<Vec4<float> *>(blk + raw_b + u64_b + v64_b);
  s.cpw64 = reinterpret_cast<Vec4<double> *>(blk + raw_b + u64_b + v64_b + c32_b);
  job->src = nullptr;
  job->raw = s.U32;
  job->U64 = s.U64;
  job->V64 = s.V64;
  job->cpw32 = s.cpw32;
  job->cpw64 = s.cpw64;
  job->ndata = ndata;
  job->ncp = static_cast<long long>(ncp);
  job->nku = nku;
  job->nkv = nkv;
  job->rat = s.rat;
  job->pad_ = 0;
  return s;
}

// surface_header and the copy of the record into the staging ring in one
// pass over the caller's data: knots copied, then every control point (and
// weight) copied while its magnitudes are folded in.  The results equal
// surface_header's (max and |x| are exact; the weighted products of two
// floats are exact in double).
void stage_surface(SurfaceRec &s, const int ivec[7], const float *data, int ndata, float *dst) {
  std::memcpy(s.ivec, ivec, sizeof(s.ivec));
  const int flags = ivec[0];
  s.rat = (flags & 2) ? 1 : 0;
  s.zero = ((!(flags & 1)) && (flags & 12)) || ivec[1] >= kMaxDeg || ivec[4] >= kMaxDeg;
  s.du = std::min(2, ivec[1]);
  s.dv = std::min(2, ivec[4]);
  s.dom[0] = data[0];
  s.dom[1] = data[ivec[3]];
  s.dom[2] = data[ivec[3] - 1];
  s.dom[3] = data[ivec[3] + ivec[6] - 1];
  const size_t nk = static_cast<size_t>(ivec[3]) + ivec[6];
  const size_t ncp = static_cast<size_t>(ivec[2]) * ivec[5];
  std::memcpy(dst, data, nk * sizeof(float));
  const float *cp = data + nk;
  float *dcp = dst + nk;
  float m[3] = {0.0f, 0.0f, 0.0f};
  for (size_t q = 0; q < ncp; ++q) {
    const float x = cp[3 * q], y = cp[3 * q + 1], z = cp[3 * q + 2];
    dcp[3 * q] = x;
    dcp[3 * q + 1] = y;
    dcp[3 * q + 2] = z;
    m[0] = std::max(m[0], std::fabs(x));
    m[1] = std::max(m[1], std::fabs(y));
    m[2] = std::max(m[2], std::fabs(z));
  }
  for (int c = 0; c < 3; ++c) s.cmax[c] = s.wcmax[c] = m[c];
  s.wmin = s.wmax = 1.0;
  size_t done = nk + 3 * ncp;
  if (s.rat && ncp > 0) {
    const float *w = cp + 3 * ncp;
    float *dw = dcp + 3 * ncp;
    float lo = w[0], hi = w[0];
    double wm[3] = {0.0, 0.0, 0.0};
    for (size_t q = 0; q < ncp; ++q) {
      const float wq = w[q];
      dw[q] = wq;
      lo = std::min(lo, wq);
      hi = std::max(hi, wq);
      for (int c = 0; c < 3; ++c)
        wm[c] = std::max(wm[c], std::fabs(static_cast<double>(wq) * static_cast<double>(cp[3 * q + c])));
    }
    s.wmin = lo;
    s.wmax = hi;
    for (int c = 0; c < 3; ++c) s.wcmax[c] = wm[c];
    done += ncp;
  }
  // the rest of the record (nothing the header describes) as given
  if (static_cast<size_t>(ndata) > done)
    std::memcpy(dst + done, data + done, (static_cast<size_t>(ndata) - done) * sizeof(float));
}

void upload_resident_many(jsi_context *ctx, const std::vector<PendingSurface> &in, std::vector<SurfaceRec> &out) {
  Lane *L = &ctx->main;
  cudaStream_t st = L->stream;
  // Header checks (ivec and ndata only) first, so that a bad surface fails
  // the call before anything is staged.
  for (size_t q = 0; q < in.size(); ++q) check_surface(in[q].ivec, in[q].data, in[q].ndata);
  std::vector<SurfaceRec> heads(in.size());
  auto al = [](size_t b) { return (b + 255) & ~static_cast<size_t>(255); };
  auto next_segment = [&]() {
    JSI_CUDA(cudaEventRecord(ctx->ring_ev[ctx->ring_cur], st));
    ctx->ring_cur = (ctx->ring_cur + 1) % kRingSegs;
    ctx->ring_off = 0;
    JSI_CUDA(cudaEventSynchronize(ctx->ring_ev[ctx->ring_cur]));
  };
  // Records that lie, in order and without overlap, inside one block of
  // jsi_host_alloc go to the device ring by DMA straight from there: one copy
  // per ring segment of the span they cover, no staging copy on the host (the
  // header pass still reads them).  The copies are asynchronous: the caller
  // keeps those records unchanged until the upload has completed on the
  // device (jsi_host_free waits for it).
  bool direct = !in.empty() && !ctx->host_blocks.empty();
  if (direct) {
    const uintptr_t p0 = reinterpret_cast<uintptr_t>(in[0].data);
    auto it = ctx->host_blocks.upper_bound(p0);
    if (it == ctx->host_blocks.begin()) {
      direct = false;
    } else {
      --it;
      const uintptr_t lo = it->first, hi = it->first + it->second;
      uintptr_t prev = lo;
      for (size_t e = 0; e < in.size() && direct; ++e) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(in[e].data);
        const uintptr_t b = a + static_cast<size_t>(in[e].ndata) * sizeof(float);
        direct = a >= prev && b <= hi && (a & 15) == 0;
        prev = b;
      }
    }
  }
  if (direct) {
    size_t q = 0;
    while (q < in.size()) {
      // Records [q, q1) whose span and jobs fit in the rest of the segment.
      const uintptr_t base = reinterpret_cast<uintptr_t>(in[q].data);
      auto span_to = [&](size_t e) {
        return reinterpret_cast<uintptr_t>(in[e].data) + static_cast<size_t>(in[e].ndata) * sizeof(float) - base;
      };
      if (ctx->ring_off + al(span_to(q)) + al(sizeof(SurfacePrep)) > kRingSeg && ctx->ring_off > 0) next_segment();
      if (al(span_to(q)) + al(sizeof(SurfacePrep)) > kRingSeg) {
        direct = false;  // a record larger than a segment: the staged path takes the rest
        break;
      }
      size_t q1 = q + 1;
      while (q1 < in.size() &&
             ctx->ring_off + al(span_to(q1)) + al(sizeof(SurfacePrep) * (q1 - q + 1)) <= kRingSeg)
        ++q1;
      const size_t seg0 = static_cast<size_t>(ctx->ring_cur) * kRingSeg;
      const size_t off = ctx->ring_off, span = span_to(q1 - 1), joff = off + al(span);
      parallel_for(ctx->hpool.get(), q1 - q,
                   [&](size_t e) { surface_header(heads[q + e], in[q + e].ivec, in[q + e].data); });
      std::vector<SurfacePrep> jobs(q1 - q);
      long long most = 0;
      for (size_t e = q; e < q1; ++e) {
        out.push_back(make_block(ctx, heads[e], in[e].ivec, in[e].ndata, &jobs[e - q]));
        jobs[e - q].src = reinterpret_cast<const float *>(ctx->dring + seg0 + off +
                                                          (reinterpret_cast<uintptr_t>(in[e].data) - base));
        most = std::max(most, std::max(jobs[e - q].ndata, jobs[e - q].ncp));
      }
      const size_t jobs_b = sizeof(SurfacePrep) * jobs.size();
      std::memcpy(ctx->ring + seg0 + joff, jobs.data(), jobs_b);
      JSI_CUDA(copy_async(L, ctx->dring + seg0 + off, in[q].data, span, cudaMemcpyHostToDevice, st));
      JSI_CUDA(copy_async(L, ctx->dring + seg0 + joff, ctx->ring + seg0 + joff, jobs_b, cudaMemcpyHostToDevice, st));
      launch_surface_prep(reinterpret_cast<const SurfacePrep *>(ctx->dring + seg0 + joff),
                          static_cast<int>(jobs.size()), most, st);
      ctx->ring_off = joff + al(jobs_b);
      q = q1;
    }
    if (direct) {
      JSI_CUDA(cudaGetLastError());
      std::lock_guard<std::mutex> ls(ctx->surf_mu);
      JSI_CUDA(cudaEventRecord(ctx->upload_ev, st));
      return;
    }
    // fall through: the staged path uploads the records from out.size() on
  }
  size_t q = out.size();
  while (q < in.size()) {
    const size_t rec_b = al(static_cast<size_t>(in[q].ndata) * sizeof(float));
    if (rec_b + al(sizeof(SurfacePrep)) > kRingSeg) {
      // Larger than a segment: its own device staging, completed here.
      surface_header(heads[q], in[q].ivec, in[q].data);
      SurfacePrep job;
      out.push_back(make_block(ctx, heads[q], in[q].ivec, in[q].ndata, &job));
      char *tmp = nullptr;
      if (cudaMalloc(&tmp, rec_b + al(sizeof(SurfacePrep))) != cudaSuccess) {
        cudaGetLastError();
        fail(JSI_ERR_NOMEM, "cudaMalloc of %zu bytes to stage a surface failed", rec_b);
      }
      job.src = reinterpret_cast<const float *>(tmp);
      JSI_CUDA(copy_async(L, tmp, in[q].data, static_cast<size_t>(in[q].ndata) * sizeof(float),
                          cudaMemcpyHostToDevice, st));
      JSI_CUDA(copy_async(L, tmp + rec_b, &job, sizeof(job), cudaMemcpyHostToDevice, st));
      launch_surface_prep(reinterpret_cast<const SurfacePrep *>(tmp + rec_b), 1, std::max<long long>(job.ndata, job.ncp),
                          st);
      JSI_CUDA(cudaStreamSynchronize(st));
      cudaFree(tmp);
      ++q;
      continue;
    }
    // Plan the segment: as many records as fit in the rest of it, then the
    // jobs; the copies (with the header pass fused in) run on host threads.
    if (ctx->ring_off + rec_b + al(sizeof(SurfacePrep)) > kRingSeg) next_segment();
    const size_t seg0 = static_cast<size_t>(ctx->ring_cur) * kRingSeg;
    size_t off = ctx->ring_off;
    std::vector<std::pair<size_t, size_t>> copies;  // (surface, ring offset)
    while (q < in.size()) {
      const size_t rb = al(static_cast<size_t>(in[q].ndata) * sizeof(float));
      if (off + rb + al(sizeof(SurfacePrep) * (copies.size() + 1)) > kRingSeg) break;
      copies.push_back({q, off});
      off += rb;
      ++q;
    }
    parallel_for(ctx->hpool.get(), copies.size(), [&](size_t e) {
      const size_t sq = copies[e].first;
      const PendingSurface &ps = in[sq];
      stage_surface(heads[sq], ps.ivec, ps.data, ps.ndata, reinterpret_cast<float *>(ctx->ring + seg0 + copies[e].second));
    });
    std::vector<SurfacePrep> jobs(copies.size());
    long long most = 0;
    for (size_t e = 0; e < copies.size(); ++e) {
      const size_t sq = copies[e].first;
      out.push_back(make_block(ctx, heads[sq], in[sq].ivec, in[sq].ndata, &jobs[e]));
      jobs[e].src = reinterpret_cast<const float *>(ctx->dring + seg0 + copies[e].second);
      most = std::max(most, std::max(jobs[e].ndata, jobs[e].ncp));
    }
    const size_t jobs_b = sizeof(SurfacePrep) * jobs.size();
    std::memcpy(ctx->ring + seg0 + off, jobs.data(), jobs_b);
    const size_t start = ctx->ring_off;
    JSI_CUDA(copy_async(L, ctx->dring + seg0 + start, ctx->ring + seg0 + start, off + jobs_b - start,
                        cudaMemcpyHostToDevice, st));
    launch_surface_prep(reinterpret_cast<const SurfacePrep *>(ctx->dring + seg0 + off), static_cast<int>(jobs.size()),
                        most, st);
    ctx->ring_off = off + al(jobs_b);
  }
  JSI_CUDA(cudaGetLastError());
  std::lock_guard<std::mutex> ls(ctx->surf_mu);
  JSI_CUDA(cudaEventRecord(ctx->upload_ev, st));
}

SurfaceRec upload_resident(jsi_context *ctx, const int ivec[7], const float *data, int ndata) {
  std::vector<SurfaceRec> out;
  upload_resident_many(ctx, {PendingSurface{ivec, data, ndata}}, out);
  return out[0];
}


// Allocates one side's per-round arrays for nreg regions.
// tables = false (intersection sides that the fused region kernel builds):
// no spans, basis tables or sample grid.
template <typename T>
SideRound<T> make_side(Arena &ar, const Geom &g, int nreg, bool intersect, RegionRec<T> *regions,
                       bool tables = true) {
  SideRound<T> s{};
  s.g = g;
  s.nreg = nreg;
  s.regions = regions ? regions : ar.get<RegionRec<T>>(nreg);
  if (tables) {
    s.spans = ar.get<int>(static_cast<size_t>(nreg) * 2 * g.nuv);
    s.basis = ar.get<T>(static_cast<size_t>(nreg) * 2 * g.nuv * 3 * g.p1max);
  }
  s.samples = intersect && tables ? ar.get<Vec4<T>>(static_cast<size_t>(nreg) * g.nuv * g.nuv) : nullptr;
  s.kmax = ar.get<unsigned long long>(static_cast<size_t>(nreg) * 3);
  s.pad = ar.get<T>(nreg);
  s.center = ar.get<Vec4<T>>(static_cast<size_t>(nreg) * g.cpr);
  s.half = intersect ? ar.get<Vec4<T>>(static_cast<size_t>(nreg) * g.cpr) : nullptr;
  s.tlo = ar.get<Vec4<T>>(static_cast<size_t>(nreg) * g.ntiles);
  s.thi = ar.get<Vec4<T>>(static_cast<size_t>(nreg) * g.ntiles);
  s.thmax = intersect ? ar.get<Vec4<T>>(static_cast<size_t>(nreg) * g.ntiles) : nullptr;
  return s;
}

// Algorithmic flops of one sample of the intersection's sample kernel (FMA =
// 2 flops): with need_k the full record (every derivative combination within
// the degrees, evaluation.cu:259-356: rational terms N w, N w P, row sum and
// v sum, 8 flops per control point and per row; non-rational 6) plus the
// quotient rule (~60); without, the position alone.
double record_flops(int degu, int degv, int du, int dv, bool rat, bool need_k) {
  const double per_cp = rat ? 8.0 : 6.0;
  const double combo = (degv + 1.0) * (degu + 1.0) * per_cp + (degv + 1.0) * per_cp;
  if (!need_k) return combo + (rat ? 4.0 : 0.0);
  const int ku[6] = {0, 1, 0, 2, 1, 0}, kv[6] = {0, 0, 1, 0, 1, 2};
  double f = 0.0;
  for (int m = 0; m < 6; ++m)
    if (ku[m] <= du && kv[m] <= dv) f += combo;
  return f + (rat ? 60.0 : 0.0);
}

void add_units(Lane *ctx, const char *name, double units);

// Evaluation + cell + tile build of one side (run_evaluation_and_construction_task,
// distance_analysis.cu:88-116 / intersection.cu:175-219).
template <typename T>
void build_side(Lane *ctx, const SurfView<T> &v, SideRound<T> &s, bool intersect, bool use_k, T span_u0,
                T span_v0, bool cover = false) {
  cudaStream_t st = ctx->stream;
  const bool need_k = intersect && use_k;
  if (!intersect || s.samples)
    timed(ctx, "basis", [&] {
      launch_basis(v, s, st, Batch{}, static_cast<const SurfView<T> *>(nullptr), cover, !intersect && !cover);
    }, 2.0 * s.nreg * s.g.nuv);
  if (!intersect) {
    // Distance: centres straight from the basis tables, no sample grid.
    timed(ctx, "cells", [&] { launch_cells_fused(v, s, s, st); }, double(s.nreg) * s.g.W * s.g.W);
    JSI_CUDA(cudaGetLastError());
    return;
  }
  const double nsamp = double(s.nreg) * s.g.nuv * s.g.nuv;
  const double sample_flops = nsamp * record_flops(v.degu, v.degv, v.du, v.dv, v.rat != 0, need_k);
  if (!s.samples) {
    // Small regions without tables: one fused launch per side.  Its HBM
    // bytes: region records and the pads / curvature maxima per region, the
    // centre and half span of every cell and three bound vectors per tile
    // (the control net is L2-resident).
    add_units(ctx, "region_cells:flops", sample_flops);
    add_units(ctx, "region_cells:bytes",
              double(s.nreg) * (sizeof(RegionRec<T>) + sizeof(T) + 3 * sizeof(unsigned long long) +
                                double(s.g.W) * s.g.W * 2 * sizeof(Vec4<T>) + double(s.g.ntiles) * 3 * sizeof(Vec4<T>)));
    timed(ctx, "region_cells", [&] { launch_region_cells(v, s, need_k, span_u0, span_v0, cover, st); }, nsamp);
    JSI_CUDA(cudaGetLastError());
    return;
  }
  add_units(ctx, "samples:flops", sample_flops);
  if (need_k) JSI_CUDA(cudaMemsetAsync(s.kmax, 0, sizeof(unsigned long long) * 3 * s.nreg, st));
  timed(ctx, "samples", [&] { launch_samples(v, s, need_k, st); }, nsamp);
  if (intersect) timed(ctx, "pad", [&] { launch_pad(s, need_k, span_u0, span_v0, st); });
  timed(ctx, "cells", [&] { launch_cells(s, intersect, st); }, double(s.nreg) * s.g.W * s.g.W);
  JSI_CUDA(cudaGetLastError());
}

// Callers hold ctx->stats_mu.
cudaEvent_t take_event(Lane *ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  JSI_CUDA(cudaEventCreate(&e));
  return e;
}

// Resolves recorded kernel timings; call after the stream has synchronised.
void resolve_timing(Lane *ctx) {
  std::lock_guard<std::mutex> lk(ctx->stats_mu);
  for (auto &p : ctx->pending) {
    float ms = 0.0f;
    JSI_CUDA(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
    auto &acc = ctx->kernel_ms[p.first];
    acc.first += ms;
    acc.second += 1;
    ctx->event_pool.push_back(p.second.first);
    ctx->event_pool.push_back(p.second.second);
  }
  ctx->pending.clear();
}

// Work units of a kernel (for the live roofline); only kept while timing.
void add_units(Lane *ctx, const char *name, double units) {
  if (!ctx->timing || ctx->capturing) return;
  std::lock_guard<std::mutex> lk(ctx->stats_mu);
  ctx->kernel_units[name] += units;
}

// Runs one launcher, bracketed by events when timing is on.
template <typename Fn>
void timed(Lane *ctx, const char *name, Fn &&fn, double units = 0) {
  if (!ctx->timing || ctx->capturing) {
    fn();
    return;
  }
  add_units(ctx, name, units);
  cudaEvent_t a, b;
  {
    std::lock_guard<std::mutex> lk(ctx->stats_mu);
    a = take_event(ctx);
    b = take_event(ctx);
  }
  JSI_CUDA(cudaEventRecord(a, ctx->stream));
  fn();
  JSI_CUDA(cudaEventRecord(b, ctx->stream));
  std::lock_guard<std::mutex> lk(ctx->stats_mu);
  ctx->pending.push_back({name, {a, b}});
}

void reset_stats(Lane *ctx) {
  ScreenStats z{};
  z.tau_bits = 0x7f800000u;
  z.lb_bits = 0x7ff0000000000000ull;
  z.ub_bits = 0x7ff0000000000000ull;
  *ctx->h_stats = z;
  JSI_CUDA(copy_async(ctx, ctx->d_stats, ctx->h_stats, sizeof(ScreenStats), cudaMemcpyHostToDevice, ctx->stream));
}

void pull_stats(Lane *ctx) {
  JSI_CUDA(copy_async(ctx, ctx->h_stats, ctx->d_stats, sizeof(ScreenStats), cudaMemcpyDeviceToHost, ctx->stream));
  JSI_CUDA(cudaStreamSynchronize(ctx->stream));
  JSI_CUDA(cudaGetLastError());
  resolve_timing(ctx);
}

unsigned bit_cast_u32(float x) {
  unsigned u;
  std::memcpy(&u, &x, sizeof(u));
  return u;
}

int bit_width(unsigned long long x) {
  int b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

template <typename T>
void check_task(const jsi_task *t) {
  if (!t) fail(JSI_ERR_INVALID, "null task");
  if (t->nuv < 2 || t->nuv > 4096) fail(JSI_ERR_INVALID, "task nuv %d outside [2, 4096]", t->nuv);
}

constexpr unsigned long long kMaxTilePairs = 1ull << 27;
// The intersection's survivor list (8 B per tile pair): refinement rounds of
// heavily overlapping pairs reach 10^8 tile pairs (13.5 M slots x 16); the
// arena's budget bounds it further.
constexpr unsigned long long kMaxInterTilePairs = 1ull << 30;

// ---------------------------------------------------------------------------
// minimum_distance
// ---------------------------------------------------------------------------

// Per-coordinate bound of |c32 - c64| for the cell centres of one surface in
// the FP32-screen form.  The FP64 form contracts the FP64 basis N64 with the
// control net in FP64; the screen rounds the same N64 to FP32 and contracts
// with FMAs.  With gamma_n = n u / (1 - n u) and n = degu + degv + 6 roundings
// along either chain, both results lie within gamma_n * sum|Nv||Nu||CP| of the
// exact sum; the B-spline basis is non-negative and sums to 1, so that sum is
// at most max|CP| per coordinate.  Rational surfaces: the same bound for the
// homogeneous sums (w CP, w), then the FP64 division.  Centres add one FP32
// and one FP64 rounding of (lo + hi) / 2.  Margins (x1.01) cover the basis
// sums deviating from 1 by FP64 rounding.
// gamma_n(u32) + gamma_n(u64) for the n = degu + degv + 6 roundings of
// either contraction chain of a surface.
double screen_gamma(const SurfaceRec &s) {
  const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
  const double n = s.ivec[1] + s.ivec[4] + 6;
  return n * u32 / (1 - n * u32) + n * u64 / (1 - n * u64);
}

// Per-coordinate bound of |P32 - P64| for the samples themselves (before the
// centre's rounding).
void sample_error(const SurfaceRec &s, double es[3]) {
  const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
  const double g = screen_gamma(s);
  for (int c = 0; c < 3; ++c) {
    if (!s.rat) {
      es[c] = g * s.cmax[c] * 1.01;
    } else {
      const double ehx = g * s.wcmax[c] * 1.01, ehw = g * s.wmax * 1.01;
      es[c] = (ehx + s.cmax[c] * ehw) / (s.wmin - ehw) + 4 * u64 * s.cmax[c] + u32 * s.cmax[c];
    }
  }
}

void centre_error(const SurfaceRec &s, double ec[3]) {
  const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
  double ep[3];
  sample_error(s, ep);
  for (int c = 0; c < 3; ++c) ec[c] = (ep[c] + (u32 + u64) * (s.cmax[c] + ep[c])) * 1.01;
}

float screen_error(const SurfaceRec &a, const SurfaceRec &b) {
  if (a.rat && !(a.wmin > 0)) fail(JSI_ERR_UNSUPPORTED, "FP32 screen needs positive weights");
  if (b.rat && !(b.wmin > 0)) fail(JSI_ERR_UNSUPPORTED, "FP32 screen needs positive weights");
  double ea[3], eb[3];
  centre_error(a, ea);
  centre_error(b, eb);
  double ss = 0;
  for (int c = 0; c < 3; ++c) ss += (ea[c] + eb[c]) * (ea[c] + eb[c]);
  const double e = std::sqrt(ss) * (1 + 1e-6);
  return std::nextafter(static_cast<float>(e), INFINITY);
}

// One screening round of the distance query: exact k smallest cell pairs
// under (d2, slot, i, j) into top; returns how many were kept.  TC is the
// precision of the cells; TS that of the selection (TC, or double for the
// FP32 screen, whose candidates are re-checked in FP64 by `verify`).
template <typename TC, typename TS, typename Verify>
int dist_screen_round(Lane *ctx, const SideRound<TC> &A, const SideRound<TC> &B, const int *map1,
                      const int *map2, int nslots, int k, bool screen, float e, DistCand<TS> *top, Verify &&verify,
                      long long *tests, long long *cands, jsi_dist_result *trace = nullptr) {
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  const unsigned long long tile_pairs = static_cast<unsigned long long>(nslots) * A.g.ntiles * B.g.ntiles;
  unsigned long long cand_cap = 1ull << 20;
  DistCand<TC> *cand = ar.get<DistCand<TC>>(cand_cap);
  unsigned long long *surv = nullptr;
  unsigned *surv_lb = nullptr;
  reset_stats(ctx);
  if (A.g.tw > kMaxTile || B.g.tw > kMaxTile) {
    // Two levels: supertile pairs (8 x 8 tiles each) seed tau and are culled;
    // only the tile pairs inside surviving supertile pairs are examined.
    SideRound<TC> As = A, Bs = B;
    As.stlo = ar.get<Vec4<TC>>(static_cast<size_t>(A.nreg) * A.g.nst);
    As.sthi = ar.get<Vec4<TC>>(static_cast<size_t>(A.nreg) * A.g.nst);
    Bs.stlo = ar.get<Vec4<TC>>(static_cast<size_t>(B.nreg) * B.g.nst);
    Bs.sthi = ar.get<Vec4<TC>>(static_cast<size_t>(B.nreg) * B.g.nst);
    timed(ctx, "supertiles", [&] {
      launch_supertiles(As, st);
      launch_supertiles(Bs, st);
    }, double(A.nreg) * A.g.nst + double(B.nreg) * B.g.nst);
    const unsigned long long st_pairs = static_cast<unsigned long long>(nslots) * A.g.nst * B.g.nst;
    if (st_pairs > kMaxTilePairs) fail(JSI_ERR_CAPACITY, "%llu supertile pairs exceed the screen's list", st_pairs);
    unsigned long long *st_surv = ar.get<unsigned long long>(st_pairs);
    timed(ctx, "dist_tau", [&] { launch_dist_tau_st(As, Bs, map1, map2, nslots, k, ctx->d_stats, screen, e, st); },
          double(st_pairs));
    timed(ctx, "dist_cull", [&] {
      launch_dist_cull_st(As, Bs, map1, map2, nslots, st_surv, st_pairs, ctx->d_stats, screen, e, st);
    }, double(st_pairs));
    pull_stats(ctx);
    const unsigned long long n_st = ctx->h_stats->st_survivors;
    const unsigned long long cap = n_st * kMaxTile * kMaxTile * kMaxTile * kMaxTile;
    if (cap > kMaxTilePairs) fail(JSI_ERR_CAPACITY, "%llu tile pairs exceed the screen's list", cap);
    surv = ar.get<unsigned long long>(std::max<unsigned long long>(cap, 1));
    surv_lb = ar.get<unsigned>(std::max<unsigned long long>(cap, 1));
    timed(ctx, "dist_expand", [&] {
      launch_dist_expand(As, Bs, map1, map2, st_surv, n_st, n_st, k, 0, surv, surv_lb, cap, ctx->d_stats, screen, e,
                         st);
      launch_dist_expand(As, Bs, map1, map2, st_surv, n_st, n_st, k, 1, surv, surv_lb, cap, ctx->d_stats, screen, e,
                         st);
    }, 2.0 * double(cap));
  } else {
    if (tile_pairs > kMaxTilePairs) fail(JSI_ERR_CAPACITY, "%llu tile pairs exceed the screen's list", tile_pairs);
    surv = ar.get<unsigned long long>(tile_pairs);
    surv_lb = ar.get<unsigned>(tile_pairs);
    if (dist_tau_folds(B.g, k))
      timed(ctx, "dist_tau", [&] { launch_dist_tau(A, B, map1, map2, nslots, k, ctx->d_stats, screen, e, st); },
            double(tile_pairs));
    timed(ctx, "dist_cull", [&] {
      launch_dist_cull(A, B, map1, map2, nslots, surv, surv_lb, tile_pairs, ctx->d_stats, screen, e, st);
    }, double(tile_pairs));
  }
  pull_stats(ctx);
  const unsigned long long nsurv = ctx->h_stats->survivors;
  // Leaf order: ascending lower bound, so that the first tile pairs tighten
  // tau and the rest stop early (exactness does not depend on the order).
  const unsigned long long *leaf_surv = surv;
  const unsigned *leaf_lb = nullptr;
  if (nsurv > 2048) {
    unsigned long long *surv_alt = ar.get<unsigned long long>(nsurv);
    unsigned *lb_alt = ar.get<unsigned>(nsurv);
    cub::DoubleBuffer<unsigned> kb(surv_lb, lb_alt);
    cub::DoubleBuffer<unsigned long long> vb(surv, surv_alt);
    size_t tmp_bytes = 0;
    JSI_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, kb, vb, static_cast<int>(nsurv), 0, 32, st));
    void *tmp = ar.alloc(tmp_bytes);
    timed(ctx, "sort_tiles", [&] {
      JSI_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, kb, vb, static_cast<int>(nsurv), 0, 32, st));
    });
    leaf_surv = vb.Current();
    leaf_lb = kb.Current();
  }
  {
    // Tighten tau before any candidate is collected, so that the collecting
    // pass appends few pairs: exact per-tile-pair k-th (k <= 8) over the tile
    // pairs with the smallest bounds (all of them when few survive).
    const unsigned long long head = leaf_lb ? std::min<unsigned long long>(nsurv, 148ull * 4) : nsurv;
    if (k <= 8) {
      timed(ctx, "dist_head", [&] {
        launch_dist_head(A, B, map1, map2, leaf_surv, head, head, k, ctx->d_stats, screen, e, st);
      });
    } else {
      timed(ctx, "dist_head", [&] {
        launch_dist_leaf(A, B, map1, map2, leaf_surv, leaf_lb, head, head, leaf_lb != nullptr, k, 0, cand, cand_cap,
                         ctx->d_stats, screen, e,
                         st);
      });
      JSI_CUDA(cudaMemsetAsync(&ctx->d_stats->work, 0, sizeof(unsigned long long), st));
    }
  }
  const DistCand<TS> *checked_out = nullptr;  // the screen's candidates with their FP64 d2
  for (int attempt = 0;; ++attempt) {
    timed(ctx, "dist_leaf", [&] {
      launch_dist_leaf(A, B, map1, map2, leaf_surv, leaf_lb, nsurv, nsurv, leaf_lb != nullptr, k, 1, cand, cand_cap,
                       ctx->d_stats, screen, e,
                       st);
    });
    bool fits = true;
    if constexpr (std::is_same<TC, TS>::value) {
      timed(ctx, "dist_select", [&] { launch_dist_select(cand, cand_cap, k, top, ctx->d_stats, st); });
    } else {
      pull_stats(ctx);
      const unsigned long long m = ctx->h_stats->candidates;
      fits = m <= cand_cap;
      if (fits) {
        DistCand<TS> *checked = ar.get<DistCand<TS>>(std::max<unsigned long long>(m, 1));
        timed(ctx, "dist_verify", [&] { verify(cand, static_cast<long long>(m), checked); });
        timed(ctx, "dist_select", [&] { launch_dist_select(checked, m, k, top, ctx->d_stats, st); });
        checked_out = checked;
      }
    }
    pull_stats(ctx);
    ScreenStats &hs = *ctx->h_stats;
    if (fits && hs.candidates <= cand_cap && hs.status == 0) break;
    if (attempt >= 4) fail(JSI_ERR_CAPACITY, "distance candidates did not fit after %d passes", attempt + 1);
    // The leaf pass tightened tau: rerun it with the tighter bound.
    if (hs.candidates > cand_cap) {
      cand_cap = std::min<unsigned long long>(hs.candidates, 1ull << 26);
      cand = ar.get<DistCand<TC>>(cand_cap);
    }
    hs.candidates = 0;
    hs.pair_tests = 0;
    hs.status = 0;
    hs.work = 0;
    JSI_CUDA(copy_async(ctx, ctx->d_stats, &hs, sizeof(ScreenStats), cudaMemcpyHostToDevice, st));
  }
  *tests = static_cast<long long>(ctx->h_stats->pair_tests);
  *cands = static_cast<long long>(ctx->h_stats->candidates);
  add_units(ctx, "dist_leaf", static_cast<double>(*tests));
  const int nsel = ctx->h_stats->nsel;
  if (trace && trace->cand_pairs) {
    // The screen's candidate set: with the FP64 d2 of each (re-checked for
    // the FP32 screen), so that a caller can check it holds every pair whose
    // d2 is at most the k-th value.
    const long long m = *cands;
    const long long keep = std::min<long long>(m, trace->cand_cap);
    if (keep > 0) {
      std::vector<unsigned char> h;
      if constexpr (std::is_same<TC, TS>::value) {
        h.resize(static_cast<size_t>(keep) * sizeof(DistCand<TC>));
        JSI_CUDA(copy_async(ctx, h.data(), cand, h.size(), cudaMemcpyDeviceToHost, st));
      } else {
        h.resize(static_cast<size_t>(keep) * sizeof(DistCand<TS>));
        JSI_CUDA(copy_async(ctx, h.data(), checked_out, h.size(), cudaMemcpyDeviceToHost, st));
      }
      JSI_CUDA(cudaStreamSynchronize(st));
      for (long long q = 0; q < keep; ++q) {
        int *tp = trace->cand_pairs + q * 3;
        double d2;
        if constexpr (std::is_same<TC, TS>::value) {
          const DistCand<TC> &c = reinterpret_cast<const DistCand<TC> *>(h.data())[q];
          tp[0] = c.slot, tp[1] = c.i, tp[2] = c.j, d2 = static_cast<double>(c.d2);
        } else {
          const DistCand<TS> &c = reinterpret_cast<const DistCand<TS> *>(h.data())[q];
          tp[0] = c.slot, tp[1] = c.i, tp[2] = c.j, d2 = static_cast<double>(c.d2);
        }
        if (trace->cand_d2) trace->cand_d2[q] = d2;
      }
    }
    trace->cand_written = m;
  }
  return nsel;
}

// Query rectangles as Newton bounds {u0, u1, v0, v1, s0, s1, t0, t1}.
void newton_domain(const jsi_task *ta, const jsi_task *tb, double dom[8]) {
  const float r[2][4] = {{ta->ustart, ta->ustop, ta->vstart, ta->vstop}, {tb->ustart, tb->ustop, tb->vstart, tb->vstop}};
  for (int side = 0; side < 2; ++side)
    for (int d = 0; d < 2; ++d) {
      const double a = r[side][2 * d], b = r[side][2 * d + 1];
      dom[side * 4 + 2 * d] = std::min(a, b);
      dom[side * 4 + 2 * d + 1] = std::max(a, b);
    }
}

// FP64 Levenberg-Marquardt from every final candidate pair; the smallest
// distance wins (earliest candidate on ties).
template <typename TP>
void newton_refine(Lane *ctx, const SurfaceRec &sa, const SurfaceRec &sb, const jsi_task *ta, const jsi_task *tb,
                   const SideRound<TP> &A, const SideRound<TP> &B, const int *map1, const int *map2,
                   const DistCand<TP> *top, int n, jsi_dist_result *out) {
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  double dom[8];
  newton_domain(ta, tb, dom);
  double *ddom = ar.get<double>(8);
  double *dres = ar.get<double>(static_cast<size_t>(n) * 11);
  JSI_CUDA(copy_async(ctx, ddom, dom, sizeof(dom), cudaMemcpyHostToDevice, st));
  timed(ctx, "newton", [&] {
    launch_newton_dist(view<double>(sa), view<double>(sb), A.regions, B.regions, map1, map2, A.g.nuv, B.g.nuv, top,
                       n, ddom, dres, st);
  }, double(n));
  std::vector<double> h(static_cast<size_t>(n) * 11);
  JSI_CUDA(copy_async(ctx, h.data(), dres, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  JSI_CUDA(cudaStreamSynchronize(st));
  int best = 0;
  for (int q = 1; q < n; ++q)
    if (h[q * 11] < h[best * 11]) best = q;
  const double *b = h.data() + static_cast<size_t>(best) * 11;
  out->newton_distance = b[0];
  out->uv1[0] = b[1];
  out->uv1[1] = b[2];
  out->uv2[0] = b[3];
  out->uv2[1] = b[4];
  for (int c = 0; c < 3; ++c) {
    out->point1[c] = b[5 + c];
    out->point2[c] = b[8 + c];
  }
}

struct NoVerify {
  template <typename A, typename B>
  void operator()(const A *, long long, B *) const {}
};

// The round loop (distance_analysis.cu:375-492).  TP = precision of the
// parameter rectangles, basis tables and selection; TC = precision of the
// samples and cells.  Exact forms: TP = TC.  FP32 screen: TP = double,
// TC = float, candidates re-checked in FP64.
template <typename TP, typename TC>
void run_distance(Lane *ctx, const jsi_task *ta, const jsi_task *tb, const jsi_dist_params *p,
                  jsi_dist_result *out) {
  constexpr bool kScreen = !std::is_same<TP, TC>::value;
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  const SurfaceRec &sa = get_surface(ctx, ta->surface);
  const SurfaceRec &sb = get_surface(ctx, tb->surface);
  const SurfView<TP> pa = view<TP>(sa), pb = view<TP>(sb);
  const SurfView<TC> ca = view<TC>(sa), cb = view<TC>(sb);
  const float e = kScreen ? screen_error(sa, sb) : 0.0f;
  const int k = p->k;
  RegionRec<TP> roots[2] = {{TP(ta->ustart), TP(ta->vstart), TP(ta->ustop), TP(ta->vstop)},
                            {TP(tb->ustart), TP(tb->vstart), TP(tb->ustop), TP(tb->vstop)}};
  RegionRec<TP> *dreg = ar.get<RegionRec<TP>>(2);
  int *dmap = ar.get<int>(2);
  const int zeros[2] = {0, 0};
  JSI_CUDA(copy_async(ctx, dreg, roots, sizeof(roots), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, dmap, zeros, sizeof(zeros), cudaMemcpyHostToDevice, st));
  SideRound<TP> A = make_side<TP>(ar, make_geom(ta->nuv, p1_of(sa)), 1, false, dreg);
  SideRound<TP> B = make_side<TP>(ar, make_geom(tb->nuv, p1_of(sb)), 1, false, dreg + 1);
  const int *map1 = dmap, *map2 = dmap + 1;
  int nslots = 1;
  DistCand<TP> *top = ar.get<DistCand<TP>>(kMaxK);
  std::vector<DistCand<TP>> htop(kMaxK);
  for (int round = 1; round <= p->rounds; ++round) {
    long long tests = 0, cands = 0;
    int n = 0;
    // The FP32 screen pays where the screen is large: the first round's
    // (nuv0-1)^4 pairs over cells much wider than the FP32 error bound.
    // Refinement rounds shrink cells to ~1e-6 of the coordinates, below FP32
    // resolution, so they run in FP64 (same results either way).
    if (!kScreen || round > 1) {
      build_side(ctx, pa, A, false, false, TP(1), TP(1));
      build_side(ctx, pb, B, false, false, TP(1), TP(1));
      n = dist_screen_round<TP, TP>(ctx, A, B, map1, map2, nslots, k, false, 0.0f, top, NoVerify{}, &tests, &cands,
                                    round == 1 ? out : nullptr);
    } else if constexpr (kScreen) {
      // FP64 rectangles and basis tables, FP32 samples / cells / tiles.
      SideRound<TC> A32{}, B32{};
      for (int side = 0; side < 2; ++side) {
        SideRound<TP> &P = side ? B : A;
        SideRound<TC> &C = side ? B32 : A32;
        C.g = P.g;
        C.nreg = P.nreg;
        C.center = ar.get<Vec4<TC>>(static_cast<size_t>(P.nreg) * P.g.cpr);
        C.tlo = ar.get<Vec4<TC>>(static_cast<size_t>(P.nreg) * P.g.ntiles);
        C.thi = ar.get<Vec4<TC>>(static_cast<size_t>(P.nreg) * P.g.ntiles);
        timed(ctx, "basis", [&] {
          launch_basis(side ? pb : pa, P, st, Batch{}, static_cast<const SurfView<TP> *>(nullptr), false, true);
        }, 2.0 * P.nreg * P.g.nuv);
        timed(ctx, "cells", [&] { launch_cells_fused(side ? cb : ca, P, C, st); }, double(C.nreg) * C.g.W * C.g.W);
      }
      auto verify = [&](const DistCand<TC> *c, long long m, DistCand<TP> *o) {
        launch_dist_verify(pa, pb, A, B, map1, map2, c, m, o, st);
      };
      n = dist_screen_round<TC, TP>(ctx, A32, B32, map1, map2, nslots, k, true, e, top, verify, &tests, &cands, out);
    }
    out->npairs[round - 1] = n;
    out->pair_tests[round - 1] = tests;
    out->candidates[round - 1] = cands;
    out->tile_pairs[round - 1] = static_cast<long long>(ctx->h_stats->survivors);
    out->tile_pairs_tested[round - 1] = static_cast<long long>(ctx->h_stats->tile_pairs);
    out->supertile_pairs[round - 1] = static_cast<long long>(ctx->h_stats->st_survivors);
    if (n > 0) {
      JSI_CUDA(copy_async(ctx, htop.data(), top, sizeof(DistCand<TP>) * n, cudaMemcpyDeviceToHost, st));
      JSI_CUDA(cudaStreamSynchronize(st));
      out->kth_d2[round - 1] = static_cast<double>(htop[n - 1].d2);
      if (out->trace_pairs && static_cast<long long>(round) * k <= out->trace_cap) {
        for (int q = 0; q < n; ++q) {
          int *tp = out->trace_pairs + (static_cast<long long>(round - 1) * k + q) * 3;
          tp[0] = htop[q].slot;
          tp[1] = htop[q].i;
          tp[2] = htop[q].j;
        }
      }
    } else {
      out->kth_d2[round - 1] = 0.0;
    }
    out->rounds_run = round;
    if (n == 0 || round == p->rounds) {
      const TP kth = n > 0 ? htop[n - 1].d2 : TP(0);
      const TP root = std::sqrt(kth);
      out->v5_value = static_cast<float>(root);
      out->distance = static_cast<double>(root);
      if (p->newton && n > 0) newton_refine(ctx, sa, sb, ta, tb, A, B, map1, map2, top, n, out);
      break;
    }
    // Next round (nuv = next_nuv after round 1, distance_analysis.cu:389).
    RegionRec<TP> *next1 = ar.get<RegionRec<TP>>(n), *next2 = ar.get<RegionRec<TP>>(n);
    int *nmap1 = ar.get<int>(n), *nmap2 = ar.get<int>(n);
    timed(ctx, "dist_next", [&] {
      launch_dist_next(top, ctx->d_stats, A, B, map1, map2, p->nuv_refine, next1, next2, nmap1, nmap2, st);
    });
    pull_stats(ctx);
    const int r1 = ctx->h_stats->nreg1, r2 = ctx->h_stats->nreg2;
    A = make_side<TP>(ar, make_geom(p->nuv_refine, p1_of(sa)), r1, false, next1);
    B = make_side<TP>(ar, make_geom(p->nuv_refine, p1_of(sb)), r2, false, next2);
    map1 = nmap1;
    map2 = nmap2;
    nslots = n;
  }
}

// ---------------------------------------------------------------------------
// minimum_distance, lockstep batch
// ---------------------------------------------------------------------------
//
// Queries with one shape (first-round nuv and basis stride of both sides, k,
// rounds, refinement nuv, precision) run together: every stage is one launch
// over the batch (query = blockIdx.y), every count stays on the device, and
// the host touches the batch twice (one strided copy of the query heads in,
// one of the records out).  Each query owns a slab of identical layout; the
// kernels reach query q's arrays at the query-0 addresses + q * slab bytes.
// Lists have fixed capacities; a query that overflows one is flagged in its
// record and re-run alone by run_distance.

// Bump planner over one slab (base = nullptr: sizing pass).
class SlabPlan {
 public:
  explicit SlabPlan(char *base) : base_(base) {}
  template <typename U>
  U *get(size_t n) {
    const size_t bytes = (std::max<size_t>(n * sizeof(U), 1) + 255) & ~static_cast<size_t>(255);
    U *p = reinterpret_cast<U *>(base_ + off_);
    off_ += bytes;
    return p;
  }
  size_t size() const { return off_; }

 private:
  char *base_;
  size_t off_ = 0;
};

// What the host writes into each slab before the batch runs.
template <typename TP>
struct DistHead {
  SurfView<double> a64, b64;
  SurfView<float> a32, b32;
  double dom[8];
  RegionRec<TP> roots[2];
  int maps[2];
  int pad_[2];
  ScreenStats stats;
};

template <typename TP>
const SurfView<TP> *head_view(const DistHead<TP> *h, int side);
template <>
const SurfView<double> *head_view<double>(const DistHead<double> *h, int side) {
  return side ? &h->b64 : &h->a64;
}
template <>
const SurfView<float> *head_view<float>(const DistHead<float> *h, int side) {
  return side ? &h->b32 : &h->a32;
}

template <typename T>
SideRound<T> slab_side(SlabPlan &sp, const Geom &g, int nreg, RegionRec<T> *regions, const int *dnreg, bool basis,
                       bool cells, bool super) {
  SideRound<T> s{};
  s.g = g;
  s.nreg = nreg;
  s.regions = regions;
  s.dnreg = dnreg;
  if (basis) {
    s.spans = sp.get<int>(static_cast<size_t>(nreg) * 2 * g.nuv);
    s.basis = sp.get<T>(static_cast<size_t>(nreg) * 2 * g.nuv * 3 * g.p1max);
  }
  if (cells) {
    s.center = sp.get<Vec4<T>>(static_cast<size_t>(nreg) * g.cpr);
    s.tlo = sp.get<Vec4<T>>(static_cast<size_t>(nreg) * g.ntiles);
    s.thi = sp.get<Vec4<T>>(static_cast<size_t>(nreg) * g.ntiles);
  }
  if (super) {
    // Folded by the cell kernels (initialised before them: minima all ones,
    // maxima zero, see batch_fold_init).
    s.stmin = sp.get<typename OrdBits<T>::type>(static_cast<size_t>(nreg) * g.nst * 4);
    s.stmax = sp.get<typename OrdBits<T>::type>(static_cast<size_t>(nreg) * g.nst * 4);
  }
  return s;
}

// List capacities per query and round: tile pairs after the supertile
// expansion and screen candidates.  JSI_BATCH_SURV_CAP / JSI_BATCH_CAND_CAP
// override them (the small values exercise the re-run of overflowed queries).
struct BatchCaps {
  unsigned long long surv = 1ull << 16;
  unsigned long long cand = 1ull << 14;
};

BatchCaps batch_caps() {
  BatchCaps c;
  auto env = [](const char *name, unsigned long long dflt) {
    const char *v = std::getenv(name);
    if (!v || !*v) return dflt;
    const unsigned long long x = std::strtoull(v, nullptr, 10);
    return std::min<unsigned long long>(std::max<unsigned long long>(x, 1), 1ull << 24);
  };
  c.surv = env("JSI_BATCH_SURV_CAP", c.surv);
  c.cand = env("JSI_BATCH_CAND_CAP", c.cand);
  return c;
}
constexpr unsigned long long kBatchHeadCap = 2048;        // threshold-pass list
// Threshold-pass list sizes: round 1 (large grids) and refinement rounds.
constexpr unsigned kBatchHeadWant = 64;
constexpr unsigned kBatchHeadWantRefine = 16;

// One round's arrays in the slab.  TP sides hold the regions and basis tables
// (and, in exact rounds, the cells); the FP32 screen's first round keeps its
// cells in the TC sides.
template <typename TP, typename TC>
struct BatchRound {
  SideRound<TP> A, B;
  SideRound<TC> A32, B32;
  const int *map1 = nullptr, *map2 = nullptr;
  int max_slots = 1;
  bool super = false;
  unsigned long long st_cap = 0, surv_cap = 0, cand_cap = 0;
  unsigned long long *st_surv = nullptr, *surv = nullptr, *head = nullptr;
  unsigned *surv_lb = nullptr;
  void *cand = nullptr;  // DistCand of the round's screening precision
  DistCand<TP> *checked = nullptr;
  DistCand<TP> *top = nullptr;
  RegionRec<TP> *next1 = nullptr, *next2 = nullptr;
  int *nmap1 = nullptr, *nmap2 = nullptr;
};

template <typename TP, typename TC>
struct BatchLayout {
  DistHead<TP> *head = nullptr;
  DistRecord<TP> *rec = nullptr;
  std::vector<BatchRound<TP, TC>> rounds;
  size_t bytes = 0;
};

template <typename TP, typename TC>
BatchLayout<TP, TC> plan_batch(char *base, int nuv1, int nuv2, int p1a, int p1b, const jsi_dist_params &p,
                               const BatchCaps &caps) {
  constexpr bool kScreen = !std::is_same<TP, TC>::value;
  SlabPlan sp(base);
  BatchLayout<TP, TC> L;
  L.head = sp.get<DistHead<TP>>(1);
  L.rec = sp.get<DistRecord<TP>>(1);
  RegionRec<TP> *reg1 = L.head->roots, *reg2 = L.head->roots + 1;
  const int *map1 = L.head->maps, *map2 = L.head->maps + 1;
  const int *dn1 = nullptr, *dn2 = nullptr;
  int nreg = 1;
  for (int r = 1; r <= p.rounds; ++r) {
    BatchRound<TP, TC> R;
    const Geom g1 = make_geom(r == 1 ? nuv1 : p.nuv_refine, p1a);
    const Geom g2 = make_geom(r == 1 ? nuv2 : p.nuv_refine, p1b);
    R.super = g1.tw > kMaxTile || g2.tw > kMaxTile;
    R.max_slots = r == 1 ? 1 : p.k;
    const bool scr = kScreen && r == 1;
    R.A = slab_side<TP>(sp, g1, nreg, reg1, dn1, true, !scr, !scr && R.super);
    R.B = slab_side<TP>(sp, g2, nreg, reg2, dn2, true, !scr, !scr && R.super);
    if (scr) {
      R.A32 = slab_side<TC>(sp, g1, nreg, nullptr, dn1, false, true, R.super);
      R.B32 = slab_side<TC>(sp, g2, nreg, nullptr, dn2, false, true, R.super);
    }
    R.map1 = map1;
    R.map2 = map2;
    if (R.super) {
      R.st_cap = static_cast<unsigned long long>(R.max_slots) * g1.nst * g2.nst;
      R.st_surv = sp.get<unsigned long long>(R.st_cap);
      R.surv_cap = caps.surv;
    } else {
      R.surv_cap = static_cast<unsigned long long>(R.max_slots) * g1.ntiles * g2.ntiles;
    }
    R.surv = sp.get<unsigned long long>(R.surv_cap);
    R.surv_lb = sp.get<unsigned>(R.surv_cap);
    R.head = sp.get<unsigned long long>(kBatchHeadCap);
    R.cand_cap = caps.cand;
    R.cand = sp.get<DistCand<TP>>(R.cand_cap);  // TP is the wider type
    if (scr) R.checked = sp.get<DistCand<TP>>(R.cand_cap);
    R.top = sp.get<DistCand<TP>>(p.k);
    if (r < p.rounds) {
      R.next1 = sp.get<RegionRec<TP>>(p.k);
      R.next2 = sp.get<RegionRec<TP>>(p.k);
      R.nmap1 = sp.get<int>(p.k);
      R.nmap2 = sp.get<int>(p.k);
      reg1 = R.next1;
      reg2 = R.next2;
      map1 = R.nmap1;
      map2 = R.nmap2;
      dn1 = &L.head->stats.nreg1;
      dn2 = &L.head->stats.nreg2;
      nreg = p.k;
    }
    L.rounds.push_back(R);
  }
  L.bytes = sp.size();
  return L;
}

// Supertile accumulators of the batch's sides set to their identities before
// the cell kernels fold into them (one strided memset per array).
template <typename T>
void batch_fold_init(const SideRound<T> &S, cudaStream_t st, const Batch &bt) {
  if (!S.stmin) return;
  const size_t bytes = static_cast<size_t>(S.nreg) * S.g.nst * 4 * sizeof(typename OrdBits<T>::type);
  JSI_CUDA(cudaMemset2DAsync(S.stmin, static_cast<size_t>(bt.qs), 0xff, bytes, bt.n, st));
  JSI_CUDA(cudaMemset2DAsync(S.stmax, static_cast<size_t>(bt.qs), 0x00, bytes, bt.n, st));
}

// Screening stages of one batched round over sides of precision T.
template <typename T, typename TP, typename TC>
void batch_screen(Lane *L, const BatchRound<TP, TC> &R, const SideRound<T> &X, const SideRound<T> &Y,
                  ScreenStats *stats, int k, bool screen, float e, const Batch &bt) {
  cudaStream_t st = L->stream;
  const int ns = R.max_slots == 1 ? 1 : -R.max_slots;
  if (R.super) {
    timed(L, "dist_tau", [&] { launch_dist_tau_st(X, Y, R.map1, R.map2, ns, k, stats, screen, e, st, bt); });
    timed(L, "dist_cull", [&] {
      launch_dist_cull_st(X, Y, R.map1, R.map2, ns, R.st_surv, R.st_cap, stats, screen, e, st, bt);
    });
    // The seed of dist_tau (2 x 2 representative tiles per supertile) is
    // tight enough that the expansion goes straight to its bound pass: a
    // threshold-tightening pass over the representatives first cost more than
    // the extra surviving tile pairs it saves.
    timed(L, "dist_expand", [&] {
      launch_dist_expand(X, Y, R.map1, R.map2, R.st_surv, kFromDevice, R.st_cap, k, 1, R.surv, R.surv_lb, R.surv_cap,
                         stats, screen, e, st, bt);
    });
  } else {
    if (dist_tau_folds(Y.g, k))
      timed(L, "dist_tau", [&] { launch_dist_tau(X, Y, R.map1, R.map2, ns, k, stats, screen, e, st, bt); });
    timed(L, "dist_cull", [&] {
      launch_dist_cull(X, Y, R.map1, R.map2, ns, R.surv, R.surv_lb, R.surv_cap, stats, screen, e, st, bt);
    });
  }
  const unsigned want = R.max_slots == 1 ? kBatchHeadWant : kBatchHeadWantRefine;
  timed(L, "dist_pick", [&] { launch_dist_pick(R.surv, R.surv_lb, R.surv_cap, R.head, kBatchHeadCap, want, stats, st, bt); });
  timed(L, "dist_head", [&] {
    launch_dist_head(X, Y, R.map1, R.map2, R.head, kFromDevice, kBatchHeadCap, k, stats, screen, e, st, bt);
  });
  timed(L, "dist_leaf", [&] {
    launch_dist_leaf(X, Y, R.map1, R.map2, R.surv, R.surv_lb, kFromDevice, R.surv_cap, false, k, 1,
                     static_cast<DistCand<T> *>(R.cand), R.cand_cap, stats, screen, e, st, bt);
  });
}

char *lane_pinned(Lane *L, size_t bytes) {
  if (L->h_pin_bytes < bytes) {
    // At least double: every regrowth frees page-locked memory, which waits
    // for the whole device (the other lanes' work included), so a lane whose
    // jobs grow step by step regrows a logarithmic number of times.
    const size_t want = std::max(bytes, std::max<size_t>(2 * L->h_pin_bytes, size_t(1) << 20));
    JSI_CUDA(cudaStreamSynchronize(L->stream));
    if (L->h_pin) JSI_CUDA(cudaFreeHost(L->h_pin));
    L->h_pin = nullptr;
    L->h_pin_bytes = 0;
    JSI_CUDA(cudaMallocHost(reinterpret_cast<void **>(&L->h_pin), want));
    L->h_pin_bytes = want;
  }
  return L->h_pin;
}

// The lockstep batch (all items share the shape of items[0]); items whose
// record reports an overflow are re-run alone.  Returns the number re-run.
template <typename TP, typename TC>
int run_distance_batch(Lane *L, std::vector<BatchItem> &items, const jsi_dist_params &p) {
  constexpr bool kScreen = !std::is_same<TP, TC>::value;
  const int n = static_cast<int>(items.size());
  if (n == 0) return 0;
  cudaStream_t st = L->stream;
  const SurfaceRec &s0a = get_surface(L, items[0].a->surface);
  const SurfaceRec &s0b = get_surface(L, items[0].b->surface);
  const int nuv1 = items[0].a->nuv, nuv2 = items[0].b->nuv;
  // A batch shares the first-round nuv of each side and the zero flags;
  // degrees and rational flags may differ (a mixed batch): the slabs are laid
  // out for the largest degrees, the kernels read each query's surface from
  // its head, and the cell build takes the kernel that handles any degree.
  int dua = 0, dva = 0, dub = 0, dvb = 0;
  bool mixed = false;
  for (int q = 0; q < n; ++q) {
    const SurfaceRec &sa = get_surface(L, items[q].a->surface);
    const SurfaceRec &sb = get_surface(L, items[q].b->surface);
    if (sa.zero != s0a.zero || sb.zero != s0b.zero || items[q].a->nuv != nuv1 || items[q].b->nuv != nuv2)
      fail(JSI_ERR_INVALID, "batch items differ in first-round nuv or zero flag");
    mixed = mixed || shape_of(sa) != shape_of(s0a) || shape_of(sb) != shape_of(s0b);
    dua = std::max(dua, sa.ivec[1]);
    dva = std::max(dva, sa.ivec[4]);
    dub = std::max(dub, sb.ivec[1]);
    dvb = std::max(dvb, sb.ivec[4]);
  }
  const int p1a = std::max(dua, dva) + 1, p1b = std::max(dub, dvb) + 1;
  // Host views: only the kernel variant choice reads them (largest degrees).
  auto host_view = [&](auto v, int du, int dv) {
    v.degu = du;
    v.degv = dv;
    return v;
  };
  const BatchCaps caps = batch_caps();
  const BatchLayout<TP, TC> probe = plan_batch<TP, TC>(nullptr, nuv1, nuv2, p1a, p1b, p, caps);
  const size_t slab = (probe.bytes + 255) & ~static_cast<size_t>(255);
  char *base = static_cast<char *>(L->arena.alloc(slab * n));
  const BatchLayout<TP, TC> lay = plan_batch<TP, TC>(base, nuv1, nuv2, p1a, p1b, p, caps);
  const Batch bt{n, static_cast<long long>(slab)};

  // Heads: surface views, Newton domains, root rectangles, fresh counters.
  const size_t hsz = sizeof(DistHead<TP>), rsz = sizeof(DistRecord<TP>);
  char *pin = lane_pinned(L, std::max(hsz, rsz) * n);
  float e = 0.0f;
  for (int q = 0; q < n; ++q) {
    const SurfaceRec &sa = get_surface(L, items[q].a->surface);
    const SurfaceRec &sb = get_surface(L, items[q].b->surface);
    DistHead<TP> h{};
    h.a64 = view<double>(sa);
    h.b64 = view<double>(sb);
    h.a32 = view<float>(sa);
    h.b32 = view<float>(sb);
    newton_domain(items[q].a, items[q].b, h.dom);
    const jsi_task *ta = items[q].a, *tb = items[q].b;
    h.roots[0] = RegionRec<TP>{TP(ta->ustart), TP(ta->vstart), TP(ta->ustop), TP(ta->vstop)};
    h.roots[1] = RegionRec<TP>{TP(tb->ustart), TP(tb->vstart), TP(tb->ustop), TP(tb->vstop)};
    h.stats.tau_bits = 0x7f800000u;
    h.stats.nslots = 1;
    std::memcpy(pin + q * hsz, &h, hsz);
    if (kScreen) e = std::max(e, screen_error(sa, sb));
  }
  // The bound enters the kernels as an argument: rounded up to a power of
  // two (still a valid bound, a negligible widening) so that batches of
  // similar surfaces share one captured graph.
  if (kScreen && e > 0.0f) {
    int ex = 0;
    std::frexp(e, &ex);
    e = std::ldexp(1.0f, ex);
  }
  ScreenStats *stats = &lay.head->stats;
  const SurfView<TP> va = host_view(view<TP>(s0a), dua, dva), vb = host_view(view<TP>(s0b), dub, dvb);
  const SurfView<float> va32 = host_view(view<float>(s0a), dua, dva), vb32 = host_view(view<float>(s0b), dub, dvb);
  const int R = p.rounds;
  auto enqueue = [&]() {
    JSI_CUDA(cudaMemcpy2DAsync(lay.head, slab, pin, hsz, hsz, n, cudaMemcpyHostToDevice, st));
    L->h2d_bytes += hsz * n;

    // Refinement rounds at nuv <= kRefineNuv run as one fused launch
    // (k_dist_refine: every round of a query in one block).
    const bool fused = R >= 2 && p.nuv_refine <= kRefineNuv && p.k <= kBatchK;
    for (int r = 1; r <= (fused ? 1 : R); ++r) {
      const BatchRound<TP, TC> &Rd = lay.rounds[r - 1];
      const bool scr = kScreen && r == 1;
      timed(L, "basis", [&] {
        launch_basis(va, Rd.A, st, bt, head_view<TP>(lay.head, 0), false, true);
        launch_basis(vb, Rd.B, st, bt, head_view<TP>(lay.head, 1), false, true);
      });
      // Work units of the cell build: cells of both sides (exact in round 1,
      // where every query has one region per side; the refinement rounds'
      // region counts live on the device).
      const double cells_units = r == 1 ? double(n) * (double(Rd.A.g.W) * Rd.A.g.W + double(Rd.B.g.W) * Rd.B.g.W) : 0.0;
      const char *cells_name = r == 1 ? "cells_r1" : "cells";
      if (!scr) {
        batch_fold_init(Rd.A, st, bt);
        batch_fold_init(Rd.B, st, bt);
        timed(L, cells_name, [&] {
          launch_cells_fused(va, Rd.A, Rd.A, st, bt, head_view<TP>(lay.head, 0), mixed);
          launch_cells_fused(vb, Rd.B, Rd.B, st, bt, head_view<TP>(lay.head, 1), mixed);
        }, cells_units);
        batch_screen<TP>(L, Rd, Rd.A, Rd.B, stats, p.k, false, 0.0f, bt);
        timed(L, "dist_select", [&] {
          launch_dist_select(static_cast<const DistCand<TP> *>(Rd.cand), Rd.cand_cap, p.k, Rd.top, stats, st, bt);
        });
      } else if constexpr (kScreen) {
        batch_fold_init(Rd.A32, st, bt);
        batch_fold_init(Rd.B32, st, bt);
        timed(L, cells_name, [&] {
          launch_cells_fused(va32, Rd.A, Rd.A32, st, bt, &lay.head->a32, mixed);
          launch_cells_fused(vb32, Rd.B, Rd.B32, st, bt, &lay.head->b32, mixed);
        }, cells_units);
        batch_screen<TC>(L, Rd, Rd.A32, Rd.B32, stats, p.k, true, e, bt);
        timed(L, "dist_verify", [&] {
          launch_dist_verify(view<double>(s0a), view<double>(s0b), Rd.A, Rd.B, Rd.map1, Rd.map2,
                             static_cast<const DistCand<float> *>(Rd.cand), 0, Rd.checked,
                             st, bt, &lay.head->a64, &lay.head->b64, stats, Rd.cand_cap);
        });
        timed(L, "dist_select", [&] { launch_dist_select(Rd.checked, Rd.cand_cap, p.k, Rd.top, stats, st, bt); });
      }
      if (r < R) {
        timed(L, "dist_next", [&] {
          launch_dist_next(Rd.top, stats, Rd.A, Rd.B, Rd.map1, Rd.map2, p.nuv_refine, Rd.next1, Rd.next2, Rd.nmap1,
                           Rd.nmap2, st, bt);
        });
      }
      timed(L, "dist_close", [&] {
        launch_dist_close(stats, Rd.top, lay.rec, r - 1, Rd.surv_cap, Rd.cand_cap, r == R, st, bt);
      });
    }
    if (fused) {
      RefineArgs<TP> ra{};
      for (int r = 2; r <= R; ++r) {
        const BatchRound<TP, TC> &Rd = lay.rounds[r - 1];
        // the round's centre arrays hold k x cpr >= k x (nuv - 1)^2 entries
        ra.r[r - 1] = RefineRound<TP>{Rd.A.regions, Rd.B.regions, Rd.map1,  Rd.map2,  Rd.top,
                                      Rd.next1,     Rd.next2,     Rd.nmap1, Rd.nmap2, Rd.A.center, Rd.B.center};
      }
      ra.first = 2;
      ra.last = R;
      ra.nuv = p.nuv_refine;
      ra.k = p.k;
      timed(L, "refine", [&] {
        launch_dist_refine<TP>(va, vb, head_view<TP>(lay.head, 0), head_view<TP>(lay.head, 1), stats, lay.rec, ra,
                               st, bt);
      });
    }
    if (p.newton) {
      const BatchRound<TP, TC> &Rd = lay.rounds[R - 1];
      timed(L, "newton", [&] {
        launch_newton_dist(host_view(view<double>(s0a), dua, dva), host_view(view<double>(s0b), dub, dvb),
                           Rd.A.regions, Rd.B.regions, Rd.map1, Rd.map2,
                           Rd.A.g.nuv, Rd.B.g.nuv, Rd.top, p.k, lay.head->dom, lay.rec->newton, st, bt,
                           &lay.head->a64, &lay.head->b64, stats);
      });
    }
    JSI_CUDA(cudaGetLastError());
    JSI_CUDA(cudaMemcpy2DAsync(pin, rsz, lay.rec, slab, rsz, n, cudaMemcpyDeviceToHost, st));
    L->d2h_bytes += rsz * n;
  };

  // CUDA graphs: a key's first batch runs eagerly, its second is captured
  // and later ones replay it.  The key holds what the launch sequence
  // depends on: form, shape and parameters, batch size, the slab and staging
  // addresses (the arena rewinds to the same addresses while its blocks stay)
  // and the rounded bound.  Per-kernel timing always runs eagerly.
  const std::vector<long long> key = {
      static_cast<long long>(sizeof(TP)), static_cast<long long>(sizeof(TC)), nuv1, nuv2, p1a, p1b, p.k, p.rounds,
      p.nuv_refine, p.newton, n, static_cast<long long>(slab), reinterpret_cast<long long>(base),
      reinterpret_cast<long long>(pin), static_cast<long long>(caps.surv), static_cast<long long>(caps.cand),
      static_cast<long long>(bit_cast_u32(e)), shape_of(s0a), shape_of(s0b), dua | (dva << 8) | (dub << 16) | (dvb << 24),
      mixed ? 1 : 0};
  const bool graphs = !L->timing && L->graphs_on;
  auto it = graphs ? L->graphs.find(key) : L->graphs.end();
  if (it != L->graphs.end() && it->second.exec) {
    JSI_CUDA(cudaGraphLaunch(it->second.exec, st));
    add_launches(it->second.nodes);
    L->h2d_bytes += hsz * n;
    L->d2h_bytes += rsz * n;
    it->second.last_use = ++L->graph_clock;
    ++L->graph_replays;
  } else if (it != L->graphs.end()) {
    const unsigned long long before = launch_count();
    cudaGraph_t graph = nullptr;
    JSI_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    L->capturing = true;
    try {
      enqueue();
    } catch (...) {
      L->capturing = false;
      cudaStreamEndCapture(st, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    L->capturing = false;
    JSI_CUDA(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    JSI_CUDA(ie);
    it->second.exec = exec;
    it->second.nodes = launch_count() - before;
    it->second.last_use = ++L->graph_clock;
    JSI_CUDA(cudaGraphLaunch(exec, st));
  } else {
    enqueue();
    if (graphs) {
      if (L->graphs.size() >= 8) {  // keep the 8 most recently used
        auto lru = L->graphs.begin();
        for (auto g = L->graphs.begin(); g != L->graphs.end(); ++g)
          if (g->second.last_use < lru->second.last_use) lru = g;
        if (lru->second.exec) cudaGraphExecDestroy(lru->second.exec);
        L->graphs.erase(lru);
      }
      auto &ent = L->graphs[key];
      ent.seen = 1;
      ent.last_use = ++L->graph_clock;
    }
  }
  JSI_CUDA(cudaStreamSynchronize(st));
  resolve_timing(L);

  // Results, in the order and with the meaning run_distance gives them.
  int rerun = 0;
  for (int q = 0; q < n; ++q) {
    const DistRecord<TP> &rec = *reinterpret_cast<const DistRecord<TP> *>(pin + q * rsz);
    jsi_dist_result *out = items[q].out;
    bool bad = false;
    for (int r = 0; r < R && !bad; ++r) {
      bad = rec.status[r] != 0;
      if (rec.npairs[r] == 0) break;
    }
    if (bad) {
      items[q].status = -1;  // re-run below
      ++rerun;
      continue;
    }
    for (int round = 1; round <= R; ++round) {
      const int np = rec.npairs[round - 1];
      out->npairs[round - 1] = np;
      out->pair_tests[round - 1] = rec.tests[round - 1];
      out->candidates[round - 1] = rec.cands[round - 1];
      out->tile_pairs[round - 1] = static_cast<long long>(rec.survivors[round - 1]);
      out->tile_pairs_tested[round - 1] = static_cast<long long>(rec.examined[round - 1]);
      out->supertile_pairs[round - 1] = static_cast<long long>(rec.st_kept[round - 1]);
      out->kth_d2[round - 1] = np > 0 ? static_cast<double>(rec.top[round - 1][np - 1].d2) : 0.0;
      if (np > 0 && out->trace_pairs && static_cast<long long>(round) * p.k <= out->trace_cap) {
        for (int e2 = 0; e2 < np; ++e2) {
          int *tp = out->trace_pairs + (static_cast<long long>(round - 1) * p.k + e2) * 3;
          tp[0] = rec.top[round - 1][e2].slot;
          tp[1] = rec.top[round - 1][e2].i;
          tp[2] = rec.top[round - 1][e2].j;
        }
      }
      out->rounds_run = round;
      if (np == 0 || round == R) {
        const TP kth = np > 0 ? rec.top[round - 1][np - 1].d2 : TP(0);
        const TP root = std::sqrt(kth);
        out->v5_value = static_cast<float>(root);
        out->distance = static_cast<double>(root);
        if (p.newton && np > 0 && round == R) {
          int best = 0;
          for (int e2 = 1; e2 < np; ++e2)
            if (rec.newton[e2 * 11] < rec.newton[best * 11]) best = e2;
          const double *b = rec.newton + best * 11;
          out->newton_distance = b[0];
          out->uv1[0] = b[1];
          out->uv1[1] = b[2];
          out->uv2[0] = b[3];
          out->uv2[1] = b[4];
          for (int c = 0; c < 3; ++c) {
            out->point1[c] = b[5 + c];
            out->point2[c] = b[8 + c];
          }
        }
        break;
      }
    }
  }
  return rerun;
}

// ---------------------------------------------------------------------------
// intersection
// ---------------------------------------------------------------------------
// Next round's regions from the round's kept pairs, sorted by (slot, i, j):
// pair-preserving jobs with (slot, cell) dedup per side on the device
// (intersection.cu:380-447); cover selects the bounds mode's child grid.
template <typename T>
void next_regions(Lane *ctx, const unsigned long long *sorted, long long n, int ij_bits, int slot_bits,
                  const SideRound<T> &A, const SideRound<T> &B, const int *map1, const int *map2, bool cover,
                  RegionRec<T> **next1_out, RegionRec<T> **next2_out, int **nmap1_out, int **nmap2_out, int *r1_out,
                  int *r2_out) {
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  unsigned long long *key2 = ar.get<unsigned long long>(n), *key2s = ar.get<unsigned long long>(n);
  int *idx = ar.get<int>(n), *idxs = ar.get<int>(n);
  unsigned *flag1 = ar.get<unsigned>(n), *ex1 = ar.get<unsigned>(n), *flag2 = ar.get<unsigned>(n),
           *ex2 = ar.get<unsigned>(n);
  timed(ctx, "inter_prep", [&] { launch_inter_prep(sorted, n, ij_bits, key2, idx, flag1, st); });
  size_t tb1 = 0, tb2 = 0, tb3 = 0;
  JSI_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb1, flag1, ex1, static_cast<int>(n), st));
  JSI_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb2, key2, key2s, idx, idxs, static_cast<int>(n), 0,
                                           ij_bits + slot_bits, st));
  JSI_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb3, flag2, ex2, static_cast<int>(n), st));
  const size_t tmax = std::max(tb1, std::max(tb2, tb3));
  void *tmp = ar.alloc(tmax);
  size_t tbs = tmax;
  JSI_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tbs, flag1, ex1, static_cast<int>(n), st));
  tbs = tmax;
  JSI_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tbs, key2, key2s, idx, idxs, static_cast<int>(n), 0,
                                           ij_bits + slot_bits, st));
  timed(ctx, "flag_runs", [&] { launch_flag_runs(key2s, n, flag2, st); });
  tbs = tmax;
  JSI_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tbs, flag2, ex2, static_cast<int>(n), st));
  RegionRec<T> *next1 = ar.get<RegionRec<T>>(n), *next2 = ar.get<RegionRec<T>>(n);
  int *nmap1 = ar.get<int>(n), *nmap2 = ar.get<int>(n);
  timed(ctx, "inter_side1", [&] {
    launch_inter_side1(sorted, n, ij_bits, flag1, ex1, A, map1, next1, nmap1, st, cover);
  });
  timed(ctx, "inter_side2", [&] {
    launch_inter_side2(key2s, idxs, n, ij_bits, flag2, ex2, B, map2, next2, nmap2, st, cover);
  });
  unsigned *tail = reinterpret_cast<unsigned *>(ctx->h_small);
  JSI_CUDA(copy_async(ctx, &tail[0], ex1 + n - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  JSI_CUDA(copy_async(ctx, &tail[1], flag1 + n - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  JSI_CUDA(copy_async(ctx, &tail[2], ex2 + n - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  JSI_CUDA(copy_async(ctx, &tail[3], flag2 + n - 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  JSI_CUDA(cudaStreamSynchronize(st));
  JSI_CUDA(cudaGetLastError());
  *r1_out = static_cast<int>(tail[0] + tail[1]);
  *r2_out = static_cast<int>(tail[2] + tail[3]);
  *next1_out = next1;
  *next2_out = next2;
  *nmap1_out = nmap1;
  *nmap2_out = nmap2;
}

// Per-axis widening w of the intersection's FP32 overlap screen for a pair
// of surfaces.  The FP64 form keeps (i, j) when, on every axis,
// fl(|c1 - c2|) < fl((h1 + p1) + (h2 + p2)) over its FP64 centres and half
// spans; with the exact centres and half spans of the FP64 samples that
// implies |c1 - c2| < h1 + h2 + p1 + p2 + R64, R64 <= 9 u64 (C1 + C2) +
// 4 u64 (p1 + p2), C = max |coordinate| (the samples lie in the control
// net's convex hull: non-negative basis, positive weights).  FP32 samples
// within e of the FP64 ones move each centre and each half span by at most
// e, and the FP32 centres / half spans round once more (u32 C').  The FP32
// screen keeps (i, j) when fl(|c1 - c2|) < fl(fl(h1 + h2) + Q): with
// Q >= p1 + p2 + 2 (e1 + e2) + 8.2 u32 (C1' + C2') + R64, all times
// (1 + 4 u32) for the screen's own three roundings, every pair the FP64
// form keeps passes.  Here Q = ru((p1 + p2)(1 + 2^-20) + w) on the device
// (iscreen_q) with w = 1.01 (2 (e1 + e2) + 10 u32 (C + e) + 10 u64 C).
void inter_screen_widen(const SurfaceRec &a, const SurfaceRec &b, float w[3]) {
  const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
  double ea[3], eb[3];
  sample_error(a, ea);
  sample_error(b, eb);
  for (int c = 0; c < 3; ++c) {
    const double C = (a.cmax[c] + b.cmax[c]) * 1.01, e = ea[c] + eb[c];
    const double W = (2 * e + 10 * u32 * (C + e) + 10 * u64 * C) * 1.01;
    w[c] = std::nextafter(static_cast<float>(W), INFINITY);
  }
}

// The first round of the FP32-screen intersection (intersection.cu:175-219,
// 259-309 with every box and test in FP32, widened): FP64 spans and basis
// tables; FP32 samples and curvature bounds; the exact FP64 compute_K maxima
// and paddings; FP32 cells, tile cull and cell-pair screen; FP64 re-check of
// every candidate.  Returns the FP64 form's overlap keys, unordered.
void inter_screen_round(Lane *ctx, const SurfaceRec &sa, const SurfaceRec &sb, SideRound<double> &A,
                        SideRound<double> &B, bool use_k, const double span0[2][2], const int *map1,
                        const int *map2, int ij_bits, int slot_bits, jsi_inter_result *out,
                        unsigned long long **keys_out, long long *n_out, long long *tests_out) {
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  if ((sa.rat && !(sa.wmin > 0)) || (sb.rat && !(sb.wmin > 0)))
    fail(JSI_ERR_UNSUPPORTED, "FP32 screen needs positive weights");
  float w[3];
  inter_screen_widen(sa, sb, w);
  reset_stats(ctx);
  SideRound<float> S32[2];
  for (int side = 0; side < 2; ++side) {
    SideRound<double> &P = side ? B : A;
    const SurfaceRec &s = side ? sb : sa;
    SideRound<float> &C = S32[side];
    C = SideRound<float>{};
    C.g = P.g;
    C.nreg = P.nreg;
    const size_t nsamp = static_cast<size_t>(P.nreg) * P.g.nuv * P.g.nuv;
    C.samples = ar.get<Vec4<float>>(nsamp);
    C.center = ar.get<Vec4<float>>(static_cast<size_t>(P.nreg) * P.g.cpr);
    C.half = ar.get<Vec4<float>>(static_cast<size_t>(P.nreg) * P.g.cpr);
    C.tlo = ar.get<Vec4<float>>(static_cast<size_t>(P.nreg) * P.g.ntiles);
    C.thi = ar.get<Vec4<float>>(static_cast<size_t>(P.nreg) * P.g.ntiles);
    C.thmax = ar.get<Vec4<float>>(static_cast<size_t>(P.nreg) * P.g.ntiles);
    const SurfView<double> v64 = view<double>(s);
    timed(ctx, "basis", [&] { launch_basis(v64, P, st, Batch{}, static_cast<const SurfView<double> *>(nullptr)); },
          2.0 * P.nreg * P.g.nuv);
    Vec4<float> *khi = use_k ? ar.get<Vec4<float>>(nsamp) : nullptr;
    unsigned *klo = use_k ? ar.get<unsigned>(static_cast<size_t>(P.nreg) * 3) : nullptr;
    if (use_k) {
      JSI_CUDA(cudaMemsetAsync(klo, 0, sizeof(unsigned) * 3 * P.nreg, st));
      JSI_CUDA(cudaMemsetAsync(P.kmax, 0, sizeof(unsigned long long) * 3 * P.nreg, st));
    }
    add_units(ctx, "samples:flops",
              double(nsamp) * record_flops(s.ivec[1], s.ivec[4], s.du, s.dv, s.rat != 0, use_k));
    timed(ctx, "samples", [&] {
      launch_iscreen_samples(view<float>(s), P, C, use_k, khi, klo, screen_gamma(s) * 1.01, s.cmax, s.wcmax, s.wmax,
                             st);
    }, double(nsamp));
    if (use_k)
      timed(ctx, "kmax_recheck", [&] { launch_kmax_recheck(v64, P, khi, klo, &ctx->d_stats->rechecked, st); });
    timed(ctx, "pad", [&] { launch_pad<double>(P, use_k, span0[side][0], span0[side][1], st); });
    timed(ctx, "cells", [&] { launch_cells<float>(C, true, st); }, double(C.nreg) * C.g.W * C.g.W);
    // FP64 positions (one contraction per sample, no curvature terms) and
    // the FP64 form's cells from them, for the re-check of the candidates.
    timed(ctx, "samples64", [&] { launch_samples<double>(v64, P, false, st); }, double(nsamp));
    timed(ctx, "cells64", [&] { launch_cells<double>(P, true, st); }, double(P.nreg) * P.g.W * P.g.W);
  }
  JSI_CUDA(cudaGetLastError());
  const unsigned long long tile_pairs = static_cast<unsigned long long>(A.g.ntiles) * B.g.ntiles;
  if (tile_pairs > kMaxInterTilePairs) fail(JSI_ERR_CAPACITY, "%llu tile pairs exceed the screen's list", tile_pairs);
  unsigned long long *surv = ar.get<unsigned long long>(tile_pairs);
  timed(ctx, "inter_cull", [&] {
    launch_inter_cull_screen(S32[0], S32[1], map1, map2, 1, surv, tile_pairs, ctx->d_stats, w, A.pad, B.pad, st);
  }, double(tile_pairs));
  pull_stats(ctx);
  const unsigned long long nsurv = ctx->h_stats->survivors;
  unsigned long long key_cap =
      std::max<unsigned long long>(1ull << 16, std::min<unsigned long long>(nsurv * 64, 1ull << 24));
  unsigned long long *keys = ar.get<unsigned long long>(key_cap);
  for (int attempt = 0;; ++attempt) {
    timed(ctx, "inter_leaf", [&] {
      launch_inter_leaf_screen(S32[0], S32[1], map1, map2, surv, nsurv, ij_bits, keys, key_cap, ctx->d_stats, w, A.pad,
                               B.pad, st);
    });
    pull_stats(ctx);
    ScreenStats &hs = *ctx->h_stats;
    if (hs.candidates <= key_cap) break;
    if (attempt >= 1) fail(JSI_ERR_CAPACITY, "overlap list overflow");
    key_cap = hs.candidates;
    keys = ar.get<unsigned long long>(key_cap);
    hs.candidates = 0;
    hs.pair_tests = 0;
    hs.work = 0;
    JSI_CUDA(copy_async(ctx, ctx->d_stats, &hs, sizeof(ScreenStats), cudaMemcpyHostToDevice, st));
  }
  const unsigned long long m = ctx->h_stats->candidates;
  *tests_out = static_cast<long long>(ctx->h_stats->pair_tests);
  add_units(ctx, "inter_leaf", static_cast<double>(ctx->h_stats->pair_tests));
  add_units(ctx, "inter_cull", static_cast<double>(tile_pairs));
  unsigned long long *kept = ar.get<unsigned long long>(std::max<unsigned long long>(m, 1));
  timed(ctx, "inter_verify", [&] {
    launch_inter_verify_cells(A, B, map1, map2, keys, m, ij_bits, kept, m, ctx->d_stats, st);
  }, double(m));
  pull_stats(ctx);
  out->screen_written = static_cast<long long>(m);
  out->kmax_rechecked = static_cast<long long>(ctx->h_stats->rechecked);
  if (out->screen_pairs && m > 0) {
    // The screen's candidates in (slot, i, j) order, for a superset check.
    const int end_bit = 2 * ij_bits + slot_bits;
    unsigned long long *alt = ar.get<unsigned long long>(m);
    size_t tmp_bytes = 0;
    cub::DoubleBuffer<unsigned long long> db(keys, alt);
    JSI_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, static_cast<int>(m), 0, end_bit, st));
    void *tmp = ar.alloc(tmp_bytes);
    JSI_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, static_cast<int>(m), 0, end_bit, st));
    const long long keep = std::min<long long>(static_cast<long long>(m), out->screen_cap);
    std::vector<unsigned long long> h(static_cast<size_t>(std::max<long long>(keep, 0)));
    if (keep > 0)
      JSI_CUDA(copy_async(ctx, h.data(), db.Current(), keep * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    JSI_CUDA(cudaStreamSynchronize(st));
    const unsigned long long mij = (1ull << ij_bits) - 1ull;
    for (long long q = 0; q < keep; ++q) {
      int *tp = out->screen_pairs + q * 3;
      tp[0] = static_cast<int>(h[q] >> (2 * ij_bits));
      tp[1] = static_cast<int>((h[q] >> ij_bits) & mij);
      tp[2] = static_cast<int>(h[q] & mij);
    }
  }
  *keys_out = kept;
  *n_out = static_cast<long long>(ctx->h_stats->checked);
}

// The final round of an intersection query, for the curve linking.
template <typename T>
struct FinalRound {
  const double *points = nullptr;  // 8 doubles per pair, key order
  long long n = 0;
  const RegionRec<T> *reg1 = nullptr, *reg2 = nullptr;
  const int *map1 = nullptr, *map2 = nullptr;
  int nuv1 = 0, nuv2 = 0;
  const unsigned long long *keys = nullptr;
  int ij_bits = 0;
};

// cover: sample the covering grid (every refined cell sampled to its far edge)
// instead of the reference's grid; used by the curve linking, whose points
// would otherwise skip the last strip of every refined cell.
// screen (T = double only): the first round runs the FP32 screen
// (inter_screen_round); its result, and so every later round, equals the
// FP64 form's.
// Intersection points to the caller: one DMA into the lane's pinned staging,
// then the copy into the caller's (pageable, often freshly mapped) buffer
// split over the host threads, each chunk counting its converged points
// (residual <= 1e-9 (1 + |x| + |y| + |z|)) on the way.  Returns that count.
long long deliver_points(Lane *ctx, const double *dres, double *dst, long long keep, cudaStream_t st) {
  const size_t bytes = static_cast<size_t>(keep) * 8 * sizeof(double);
  const double *pin = reinterpret_cast<const double *>(lane_pinned(ctx, bytes));
  JSI_CUDA(copy_async(ctx, const_cast<double *>(pin), dres, bytes, cudaMemcpyDeviceToHost, st));
  JSI_CUDA(cudaStreamSynchronize(st));
  constexpr long long kChunk = 8192;  // points (512 KiB) per host task
  const size_t nchunk = static_cast<size_t>((keep + kChunk - 1) / kChunk);
  std::atomic<long long> conv{0};
  parallel_for(ctx->hpool, nchunk, [&](size_t c) {
    const long long q0 = static_cast<long long>(c) * kChunk, q1 = std::min(keep, q0 + kChunk);
    std::memcpy(dst + q0 * 8, pin + q0 * 8, static_cast<size_t>(q1 - q0) * 8 * sizeof(double));
    long long m = 0;
    for (long long q = q0; q < q1; ++q) {
      const double *pt = pin + q * 8;
      const double scale = 1.0 + std::fabs(pt[0]) + std::fabs(pt[1]) + std::fabs(pt[2]);
      if (pt[7] <= 1e-9 * scale) ++m;
    }
    conv += m;
  });
  return conv.load();
}

template <typename T>
void run_intersection(Lane *ctx, const jsi_task *ta, const jsi_task *tb, const jsi_inter_params *p,
                      jsi_inter_result *out, FinalRound<T> *fin = nullptr, bool cover = false, bool screen = false) {
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  const SurfaceRec &sa = get_surface(ctx, ta->surface);
  const SurfaceRec &sb = get_surface(ctx, tb->surface);
  const SurfView<T> va = view<T>(sa), vb = view<T>(sb);
  const bool use_k = p->use_k != 0;
  // Initial spans per side (intersection.cu:344-347).
  const T tiny = sizeof(T) == 4 ? T(1.0e-12f) : T(1.0e-12);
  T span_u[3] = {T(1), T(1), T(1)}, span_v[3] = {T(1), T(1), T(1)};
  span_u[1] = std::max(std::fabs(T(ta->ustop) - T(ta->ustart)), tiny);
  span_v[1] = std::max(std::fabs(T(ta->vstop) - T(ta->vstart)), tiny);
  span_u[2] = std::max(std::fabs(T(tb->ustop) - T(tb->ustart)), tiny);
  span_v[2] = std::max(std::fabs(T(tb->vstop) - T(tb->vstart)), tiny);
  const int side_a = ta->side == 2 ? 2 : 1, side_b = tb->side == 2 ? 2 : 1;

  RegionRec<T> roots[2] = {{T(ta->ustart), T(ta->vstart), T(ta->ustop), T(ta->vstop)},
                           {T(tb->ustart), T(tb->vstart), T(tb->ustop), T(tb->vstop)}};
  RegionRec<T> *dreg = ar.get<RegionRec<T>>(2);
  int *dmap = ar.get<int>(2);
  const int zeros[2] = {0, 0};
  JSI_CUDA(copy_async(ctx, dreg, roots, sizeof(roots), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, dmap, zeros, sizeof(zeros), cudaMemcpyHostToDevice, st));
  SideRound<T> A = make_side<T>(ar, make_geom(ta->nuv, p1_of(sa)), 1, true, dreg);
  SideRound<T> B = make_side<T>(ar, make_geom(tb->nuv, p1_of(sb)), 1, true, dreg + 1);
  const int *map1 = dmap, *map2 = dmap + 1;
  long long nslots = 1;
  int nuv = p->nuv_refine;
  long long written = 0;
  std::vector<unsigned long long> hkeys;
  for (int round = 1; round <= p->rounds; ++round) {
    const int sau = round == 1 ? side_a : 1, sbu = round == 1 ? side_b : 2;
    const bool screen_now = screen && round == 1 && !cover;
    if (!screen_now) {
      build_side(ctx, va, A, true, use_k, span_u[sau], span_v[sau], cover);
      build_side(ctx, vb, B, true, use_k, span_u[sbu], span_v[sbu], cover);
    }
    const int ij_bits = std::max(1, bit_width(static_cast<unsigned long long>(
                                        std::max(A.g.W * A.g.W, B.g.W * B.g.W) - 1)));
    const int slot_bits = std::max(1, bit_width(static_cast<unsigned long long>(nslots - 1)));
    if (2 * ij_bits + slot_bits > 64) fail(JSI_ERR_CAPACITY, "pair key does not fit 64 bits");
    unsigned long long *keys = nullptr;
    long long n = 0, tests = 0;
    if (screen_now) {
      if constexpr (std::is_same<T, double>::value) {
        const double span0[2][2] = {{span_u[sau], span_v[sau]}, {span_u[sbu], span_v[sbu]}};
        inter_screen_round(ctx, sa, sb, A, B, use_k, span0, map1, map2, ij_bits, slot_bits, out, &keys, &n, &tests);
      }
    }
    if (round == 1) {
      T *pads = reinterpret_cast<T *>(ctx->h_small);
      JSI_CUDA(copy_async(ctx, &pads[0], A.pad, sizeof(T), cudaMemcpyDeviceToHost, st));
      JSI_CUDA(copy_async(ctx, &pads[1], B.pad, sizeof(T), cudaMemcpyDeviceToHost, st));
      JSI_CUDA(cudaStreamSynchronize(st));
      out->pad[0] = static_cast<double>(pads[0]);
      out->pad[1] = static_cast<double>(pads[1]);
    }
    if (!screen_now) {
      const unsigned long long tile_pairs = static_cast<unsigned long long>(nslots) * A.g.ntiles * B.g.ntiles;
      if (tile_pairs > kMaxInterTilePairs) fail(JSI_ERR_CAPACITY, "%llu tile pairs exceed the screen's list", tile_pairs);
      unsigned long long *surv = ar.get<unsigned long long>(tile_pairs);
      reset_stats(ctx);
      timed(ctx, "inter_cull", [&] {
        launch_inter_cull(A, B, map1, map2, static_cast<int>(nslots), surv, tile_pairs, ctx->d_stats, st);
      });
      pull_stats(ctx);
      const unsigned long long nsurv = ctx->h_stats->survivors;
      unsigned long long key_cap =
          std::max<unsigned long long>(1ull << 16, std::min<unsigned long long>(nsurv * 64, 1ull << 24));
      keys = ar.get<unsigned long long>(key_cap);
      for (int attempt = 0;; ++attempt) {
        timed(ctx, "inter_leaf", [&] {
          launch_inter_leaf(A, B, map1, map2, surv, nsurv, ij_bits, keys, key_cap, ctx->d_stats, st);
        });
        pull_stats(ctx);
        ScreenStats &hs = *ctx->h_stats;
        if (hs.candidates <= key_cap) break;
        if (attempt >= 1) fail(JSI_ERR_CAPACITY, "overlap list overflow");
        key_cap = hs.candidates;
        keys = ar.get<unsigned long long>(key_cap);
        hs.candidates = 0;
        hs.pair_tests = 0;
        hs.work = 0;
        JSI_CUDA(copy_async(ctx, ctx->d_stats, &hs, sizeof(ScreenStats), cudaMemcpyHostToDevice, st));
      }
      n = static_cast<long long>(ctx->h_stats->candidates);
      tests = static_cast<long long>(ctx->h_stats->pair_tests);
      add_units(ctx, "inter_leaf", static_cast<double>(tests));
      add_units(ctx, "inter_cull", static_cast<double>(tile_pairs));
    }
    out->counts[round - 1] = n;
    out->pair_tests[round - 1] = tests;
    out->regions1[round - 1] = A.nreg;
    out->regions2[round - 1] = B.nreg;
    out->rounds_run = round;
    unsigned long long *sorted = keys;
    if (n > 1) {
      // (slot, i, j) order: slots concatenated in slot order, i-major, j ascending
      // (intersection.cu:299-306).
      const int end_bit = 2 * ij_bits + slot_bits;
      unsigned long long *alt = ar.get<unsigned long long>(n);
      size_t tmp_bytes = 0;
      cub::DoubleBuffer<unsigned long long> db(keys, alt);
      JSI_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, static_cast<int>(n), 0, end_bit, st));
      void *tmp = ar.alloc(tmp_bytes);
      timed(ctx, "sort_pairs", [&] {
        JSI_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, static_cast<int>(n), 0, end_bit, st));
      });
      sorted = db.Current();
    }
    if (out->trace_pairs && n > 0) {
      hkeys.resize(n);
      JSI_CUDA(copy_async(ctx, hkeys.data(), sorted, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
      JSI_CUDA(cudaStreamSynchronize(st));
      const unsigned long long mij = (1ull << ij_bits) - 1ull;
      for (long long q = 0; q < n; ++q) {
        if (written + q < out->trace_cap) {
          int *tp = out->trace_pairs + (written + q) * 3;
          tp[0] = static_cast<int>(hkeys[q] >> (2 * ij_bits));
          tp[1] = static_cast<int>((hkeys[q] >> ij_bits) & mij);
          tp[2] = static_cast<int>(hkeys[q] & mij);
        }
      }
    }
    written += n;
    if (round == p->rounds || n == 0) {
      if (p->points && n > 0 && (out->points || fin)) {
        // Intersection points from every final pair (minimum-norm Gauss-Newton).
        double dom[8];
        newton_domain(ta, tb, dom);
        double *ddom = ar.get<double>(8);
        double *dres = ar.get<double>(static_cast<size_t>(n) * 8);
        JSI_CUDA(copy_async(ctx, ddom, dom, sizeof(dom), cudaMemcpyHostToDevice, st));
        timed(ctx, "newton", [&] {
          launch_newton_inter(view<double>(sa), view<double>(sb), A.regions, B.regions, map1, map2, A.g.nuv, B.g.nuv,
                              sorted, n, ij_bits, ddom, dres, st);
        }, double(n));
        if (fin) {
          fin->points = dres;
          fin->n = n;
          fin->reg1 = A.regions;
          fin->reg2 = B.regions;
          fin->map1 = map1;
          fin->map2 = map2;
          fin->nuv1 = A.g.nuv;
          fin->nuv2 = B.g.nuv;
          fin->keys = sorted;
          fin->ij_bits = ij_bits;
        }
        const long long keep = out->points ? std::min<long long>(n, out->points_cap) : 0;
        out->points_written = keep;
        out->points_converged = keep > 0 ? deliver_points(ctx, dres, out->points, keep, st) : 0;
        if (keep == 0) JSI_CUDA(cudaStreamSynchronize(st));
      }
      break;
    }
    if (n > p->halve_threshold && nuv > p->min_nuv) nuv /= 2;  // intersection.cu:370
    if (n > (1ll << 31) - 1) fail(JSI_ERR_CAPACITY, "too many pairs for the next round");
    // Pair-preserving jobs and (slot, cell) dedup per side on the device.
    RegionRec<T> *next1, *next2;
    int *nmap1, *nmap2, r1, r2;
    next_regions<T>(ctx, sorted, n, ij_bits, slot_bits, A, B, map1, map2, cover, &next1, &next2, &nmap1, &nmap2, &r1,
                    &r2);
    // Refinement rounds of small regions run the fused region kernel (no
    // basis tables or sample grid).
    const Geom g1 = make_geom(nuv, p1_of(sa)), g2 = make_geom(nuv, p1_of(sb));
    A = make_side<T>(ar, g1, r1, true, next1, !(g1.nuv <= kRegNuv && g1.p1max <= kRegP1));
    B = make_side<T>(ar, g2, r2, true, next2, !(g2.nuv <= kRegNuv && g2.p1max <= kRegP1));
    map1 = nmap1;
    map2 = nmap2;
    nslots = n;
  }
  out->trace_written = written;
}

// ---------------------------------------------------------------------------
// Certified distance interval (bounds mode)
// ---------------------------------------------------------------------------

// Per coordinate c, bounds on |S_uu[c]| and |S_vv[c]| over a surface, from
// the raw record (knots U, knots V, control points, weights if rational).
//
// Non-rational: the second-derivative control nets (derivative control
// points applied twice per direction: Q_i = p (P_{i+1} - P_i) /
// (U_{i+p+1} - U_{i+1}), R_i = (p - 1)(Q_{i+1} - Q_i) / (U_{i+p+1} -
// U_{i+2}); a zero knot span gives a zero term) bound the second
// derivatives by the convex hull property.
//
// Rational (positive weights): S = A / w with A = sum N_i N_j w_ij (P_ij - m)
// + m w, m the centre of the control net's bounding box.  Differentiating
// (S - m) w = A' twice along u gives
//   S_u  = (A'_u - w_u (S - m)) / w,
//   S_uu = (A'_uu - 2 w_u S_u - w_uu (S - m)) / w,
// and with |S - m| <= h (the net's half range: S lies in the net's convex
// hull), w >= min w_ij, and the derivative nets of the homogeneous net
// (w (P - m), w) bounding A'_u, A'_uu, w_u, w_uu, every term is bounded.
// Each net entry carries a magnitude (the same recurrence on absolute
// values), and 1e-14 of it (about 45 units in the last place) covers the
// double rounding of the differences; the results are widened by 1e-12.
//
// Over control points i0..i1 (u) x j0..j1 (v) only, the bounds hold on the
// knot spans those points alone define: a span (su, sv) takes
// [su - p, su] x [sv - q, sv] (on it the u derivative nets that do not vanish
// are Q_{su-p..su-1} and R_{su-p..su-2}, which read only those points, and
// S lies in their convex hull).
void second_derivative_bounds_range(const int ivec[7], const float *data, int i0, int i1, int j0, int j1,
                                    double m2u[3], double m2v[3]) {
  const int p = ivec[1], nu = ivec[2], nku = ivec[3], q = ivec[4], nv = ivec[5], nkv = ivec[6];
  const bool rat = (ivec[0] & 2) != 0;
  const size_t ncp = static_cast<size_t>(nu) * nv;
  const float *U = data, *V = U + nku, *P = V + nkv;  // P[(j * nu + i) * 3 + c], u fastest
  const float *W = rat ? P + 3 * ncp : nullptr;
  const int lu = i1 - i0 + 1, lv = j1 - j0 + 1;
  auto at = [&](int i, int j) { return static_cast<size_t>(j0 + j) * nu + (i0 + i); };
  constexpr int kC = 4;
  double mid[3] = {0.0, 0.0, 0.0}, half[3] = {0.0, 0.0, 0.0}, wmin = 1.0;
  if (rat) {
    for (int c = 0; c < 3; ++c) {
      float lo = P[3 * at(0, 0) + c], hi = lo;
      for (int j = 0; j < lv; ++j)
        for (int i = 0; i < lu; ++i) {
          lo = std::min(lo, P[3 * at(i, j) + c]);
          hi = std::max(hi, P[3 * at(i, j) + c]);
        }
      mid[c] = 0.5 * (static_cast<double>(lo) + static_cast<double>(hi));  // exact
      half[c] = 0.5 * (static_cast<double>(hi) - static_cast<double>(lo));  // exact
    }
    wmin = W[at(0, 0)];
    for (int j = 0; j < lv; ++j)
      for (int i = 0; i < lu; ++i) wmin = std::min(wmin, static_cast<double>(W[at(i, j)]));
  }
  // One homogeneous net entry (w (P - m), w) and its magnitude.
  auto entry = [&](size_t k, double h[kC], double a[kC]) {
    const double w = rat ? static_cast<double>(W[k]) : 1.0;
    for (int c = 0; c < 3; ++c) {
      h[c] = rat ? w * (static_cast<double>(P[3 * k + c]) - mid[c]) : static_cast<double>(P[3 * k + c]);
      a[c] = std::fabs(h[c]);
    }
    h[3] = w;
    a[3] = std::fabs(w);
  };
  // m1 / m2: max |first / second derivative net entry| + its rounding slack.
  auto line_bound = [](const std::vector<double> &h, const std::vector<double> &a, const float *K, int deg, int n,
                       double m1[kC], double m2[kC]) {
    if (deg < 1 || n < 2) return;
    std::vector<double> Q(kC * (n - 1)), QA(kC * (n - 1));
    for (int i = 0; i < n - 1; ++i) {
      const double den = static_cast<double>(K[i + deg + 1]) - K[i + 1];
      for (int c = 0; c < kC; ++c) {
        Q[kC * i + c] = den != 0.0 ? deg * (h[kC * (i + 1) + c] - h[kC * i + c]) / den : 0.0;
        QA[kC * i + c] = den != 0.0 ? deg * (a[kC * (i + 1) + c] + a[kC * i + c]) / std::fabs(den) : 0.0;
        m1[c] = std::max(m1[c], std::fabs(Q[kC * i + c]) + 1e-14 * QA[kC * i + c]);
      }
    }
    if (deg < 2 || n < 3) return;
    for (int i = 0; i < n - 2; ++i) {
      const double den = static_cast<double>(K[i + deg + 1]) - K[i + 2];
      if (den == 0.0) continue;
      for (int c = 0; c < kC; ++c) {
        const double r = (deg - 1) * (Q[kC * (i + 1) + c] - Q[kC * i + c]) / den;
        const double ra = (deg - 1) * (QA[kC * (i + 1) + c] + QA[kC * i + c]) / std::fabs(den);
        m2[c] = std::max(m2[c], std::fabs(r) + 1e-14 * ra);
      }
    }
  };
  double m1u[kC] = {0, 0, 0, 0}, m2u_[kC] = {0, 0, 0, 0}, m1v[kC] = {0, 0, 0, 0}, m2v_[kC] = {0, 0, 0, 0};
  std::vector<double> h, a;
  for (int j = 0; j < lv; ++j) {
    h.assign(kC * lu, 0.0);
    a.assign(kC * lu, 0.0);
    for (int i = 0; i < lu; ++i) entry(at(i, j), &h[kC * i], &a[kC * i]);
    line_bound(h, a, U + i0, p, lu, m1u, m2u_);
  }
  for (int i = 0; i < lu; ++i) {
    h.assign(kC * lv, 0.0);
    a.assign(kC * lv, 0.0);
    for (int j = 0; j < lv; ++j) entry(at(i, j), &h[kC * j], &a[kC * j]);
    line_bound(h, a, V + j0, q, lv, m1v, m2v_);
  }
  for (int c = 0; c < 3; ++c) {
    double bu = m2u_[c], bv = m2v_[c];
    if (rat) {
      const double s1u = (m1u[c] + m1u[3] * half[c]) / wmin, s1v = (m1v[c] + m1v[3] * half[c]) / wmin;
      bu = (m2u_[c] + 2.0 * m1u[3] * s1u + m2u_[3] * half[c]) / wmin;
      bv = (m2v_[c] + 2.0 * m1v[3] * s1v + m2v_[3] * half[c]) / wmin;
    }
    m2u[c] = bu * (1.0 + 1e-12);
    m2v[c] = bv * (1.0 + 1e-12);
  }
}

void second_derivative_bounds_host(const int ivec[7], const float *data, double m2u[3], double m2v[3]) {
  second_derivative_bounds_range(ivec, data, 0, ivec[2] - 1, 0, ivec[5] - 1, m2u, m2v);
}

// A resident surface's raw record read back.
std::vector<float> raw_record(Lane *L, const SurfaceRec &s) {
  const size_t ncp = static_cast<size_t>(s.ivec[2]) * s.ivec[5];
  std::vector<float> raw(static_cast<size_t>(s.ivec[3]) + s.ivec[6] + (s.rat ? 4 : 3) * ncp);
  JSI_CUDA(copy_async(L, raw.data(), s.U32, raw.size() * sizeof(float), cudaMemcpyDeviceToHost, L->stream));
  JSI_CUDA(cudaStreamSynchronize(L->stream));
  return raw;
}

// Per knot span (su, sv), su in [p, ncpu - 1], sv in [q, ncpv - 1]: the
// bounds over that span's own control points, as two Vec4 rows (m2u, m2v)
// at index (sv - q) * (ncpu - p) + (su - p); zero for an empty span.
std::vector<Vec4<double>> span_curvature_table(const int ivec[7], const float *data) {
  const int p = ivec[1], nu = ivec[2], nku = ivec[3], q = ivec[4], nv = ivec[5];
  const float *U = data, *V = data + nku;
  const int nsu = nu - p, nsv = nv - q;
  if (static_cast<long long>(nsu) * nsv > (1ll << 20)) fail(JSI_ERR_CAPACITY, "%d x %d knot spans", nsu, nsv);
  std::vector<Vec4<double>> tab(2 * static_cast<size_t>(nsu) * nsv, Vec4<double>{0, 0, 0, 0});
  for (int sv = q; sv < nv; ++sv)
    for (int su = p; su < nu; ++su) {
      if (!(U[su + 1] > U[su]) || !(V[sv + 1] > V[sv])) continue;
      double mu[3], mv[3];
      second_derivative_bounds_range(ivec, data, su - p, su, sv - q, sv, mu, mv);
      const size_t k = 2 * (static_cast<size_t>(sv - q) * nsu + (su - p));
      tab[k] = Vec4<double>{mu[0], mu[1], mu[2], 0.0};
      tab[k + 1] = Vec4<double>{mv[0], mv[1], mv[2], 0.0};
    }
  return tab;
}

// Breakpoints of one parameter direction of a task rectangle [a, b] for the
// bounds mode's first round: every distinct interior knot where the surface
// may be only C0 (multiplicity >= the degree; every knot at degree 1), so
// that no cell straddles a kink, plus every g-th other knot, g chosen to
// keep the pieces near 16.
std::vector<double> knot_pieces(const float *K, int nk, int deg, double a, double b) {
  std::vector<std::pair<double, int>> in;  // distinct interior knots and their multiplicities
  for (int k = 0; k < nk; ++k) {
    const double x = K[k];
    if (!(x > a && x < b)) continue;
    if (!in.empty() && in.back().first == x) ++in.back().second;
    else in.push_back({x, 1});
  }
  const size_t g = std::max<size_t>(1, (in.size() + 1 + 15) / 16);
  std::vector<double> cuts{a};
  for (size_t k = 0; k < in.size(); ++k)
    if (in[k].second >= std::max(deg, 1) || (k + 1) % g == 0) cuts.push_back(in[k].first);
  cuts.push_back(b);
  std::sort(cuts.begin(), cuts.end());
  cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
  if (cuts.size() - 1 > 64) fail(JSI_ERR_UNSUPPORTED, "more than 64 C0 pieces in one direction");
  return cuts;
}

// Allowance for the FP64 evaluation of a surface point and for the centre /
// half-span rounding of a cell box: the evaluation's rounding stays below
// 2^-45 of the largest control-point coordinate (a few dozen roundings of
// terms bounded by it, the basis being a partition of unity); 2^-40 of it is
// a 32x margin.
double eval_allowance(const SurfaceRec &s) {
  if (s.rat) {
    // Rational: the homogeneous sums' rounding stays below 2^-45 of
    // max |w P| (coordinates) and of max w (weight); the quotient's error is
    // at most (e_A + |S| e_w) / w with w >= min w and |S| <= max |P|.
    const double c = std::max(s.cmax[0], std::max(s.cmax[1], s.cmax[2]));
    const double m = std::max(s.wcmax[0], std::max(s.wcmax[1], s.wcmax[2])) + c * s.wmax;
    return std::ldexp(m / s.wmin, -40);
  }
  return std::ldexp(std::max(s.cmax[0], std::max(s.cmax[1], s.cmax[2])), -40);
}

void run_bounds(Lane *ctx, const jsi_task *ta, const jsi_task *tb, const jsi_bounds_params *p,
                jsi_bounds_result *out) {
  Arena &ar = ctx->arena;
  cudaStream_t st = ctx->stream;
  const SurfaceRec &sa = get_surface(ctx, ta->surface);
  const SurfaceRec &sb = get_surface(ctx, tb->surface);
  if ((sa.rat && !(sa.wmin > 0)) || (sb.rat && !(sb.wmin > 0)))
    fail(JSI_ERR_UNSUPPORTED, "the bounds mode needs positive weights");
  if (sa.zero || sb.zero) fail(JSI_ERR_UNSUPPORTED, "the bounds mode needs surfaces that evaluate");
  // Upper bound: two surface points from the FP64 query with Newton.
  jsi_dist_params dp;
  jsi_dist_params_default(&dp);
  dp.precision = JSI_PREC_FP64;
  dp.newton = 1;
  jsi_dist_result dr;
  std::memset(&dr, 0, sizeof(dr));
  run_distance<double, double>(ctx, ta, tb, &dp, &dr);
  const double ea = eval_allowance(sa), eb = eval_allowance(sb);
  double ub = dr.newton_distance * (1.0 + 0x1p-50) + std::sqrt(3.0) * 1.000001 * (ea + eb);
  ub = std::nextafter(ub, INFINITY);
  out->ub = ub;
  for (int c = 0; c < 2; ++c) {
    out->uv1[c] = dr.uv1[c];
    out->uv2[c] = dr.uv2[c];
  }
  for (int c = 0; c < 3; ++c) {
    out->point1[c] = dr.point1[c];
    out->point2[c] = dr.point2[c];
  }
  // Pairs are kept while their gap can be below the prune level
  // (1 - rel_tol) ub: a dropped pair's gap exceeds it, so
  // lb = min(smallest kept gap, prune level) stays a lower bound, and the
  // kept set empties once the boxes are tighter than the tolerance.  ub (and
  // with it the prune level) drops each round to the closest corner-sample
  // pair seen.
  const double allowance = std::sqrt(3.0) * 1.000001 * (ea + eb);
  // Curvature bounds per knot span (each span's own control points), looked
  // up per region by the pad kernel.
  const std::vector<float> rawa = raw_record(ctx, sa), rawb = raw_record(ctx, sb);
  const std::vector<Vec4<double>> taba = span_curvature_table(sa.ivec, rawa.data());
  const std::vector<Vec4<double>> tabb = span_curvature_table(sb.ivec, rawb.data());
  Vec4<double> *dtab[2] = {ar.get<Vec4<double>>(taba.size()), ar.get<Vec4<double>>(tabb.size())};
  JSI_CUDA(copy_async(ctx, dtab[0], taba.data(), taba.size() * sizeof(Vec4<double>), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, dtab[1], tabb.data(), tabb.size() * sizeof(Vec4<double>), cudaMemcpyHostToDevice, st));
  const SurfView<double> va = view<double>(sa), vb = view<double>(sb);

  // First round: each rectangle cut at its knots into pieces (every C0 knot,
  // the others thinned to about 16 pieces per direction), the first-round
  // width shared out over the pieces, and every piece of one side paired with
  // every piece of the other.  No cell then straddles a kink, and each
  // piece's pads come from its own spans.
  auto pieces = [&](const std::vector<float> &raw, const SurfaceRec &s, const jsi_task *t,
                    std::vector<RegionRec<double>> &out) {
    const float *U = raw.data(), *V = U + s.ivec[3];
    const std::vector<double> cu = knot_pieces(U, s.ivec[3], s.ivec[1], t->ustart, t->ustop);
    const std::vector<double> cv = knot_pieces(V, s.ivec[6], s.ivec[4], t->vstart, t->vstop);
    for (size_t j = 0; j + 1 < cv.size(); ++j)
      for (size_t i = 0; i + 1 < cu.size(); ++i) out.push_back({cu[i], cv[j], cu[i + 1], cv[j + 1]});
    const int np = static_cast<int>(std::max(cu.size(), cv.size()) - 1);
    return std::max(3, (t->nuv - 1 + np - 1) / np + 1);
  };
  std::vector<RegionRec<double>> ra, rb;
  const int nuva = pieces(rawa, sa, ta, ra), nuvb = pieces(rawb, sb, tb, rb);
  const long long na = static_cast<long long>(ra.size()), nb = static_cast<long long>(rb.size());
  long long nslots = na * nb;
  std::vector<int> hmap(2 * nslots);
  for (long long k = 0; k < nslots; ++k) {
    hmap[k] = static_cast<int>(k / nb);
    hmap[nslots + k] = static_cast<int>(k % nb);
  }
  RegionRec<double> *dreg = ar.get<RegionRec<double>>(na + nb);
  int *dmap = ar.get<int>(2 * nslots);
  JSI_CUDA(copy_async(ctx, dreg, ra.data(), na * sizeof(RegionRec<double>), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, dreg + na, rb.data(), nb * sizeof(RegionRec<double>), cudaMemcpyHostToDevice, st));
  JSI_CUDA(copy_async(ctx, dmap, hmap.data(), hmap.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  // Per-coordinate pads: a Vec4 per region in place of the scalar.
  auto bounds_side = [&](const Geom &g, int nreg, RegionRec<double> *regions) {
    SideRound<double> S = make_side<double>(ar, g, nreg, true, regions);
    S.pad = ar.get<double>(static_cast<size_t>(nreg) * 4);
    return S;
  };
  SideRound<double> A = bounds_side(make_geom(nuva, p1_of(sa)), static_cast<int>(na), dreg);
  SideRound<double> B = bounds_side(make_geom(nuvb, p1_of(sb)), static_cast<int>(nb), dreg + na);
  const int *map1 = dmap, *map2 = dmap + nslots;
  double lb = 0.0;
  for (int round = 1; round <= p->max_rounds; ++round) {
    for (int side = 0; side < 2; ++side) {
      SideRound<double> &S = side ? B : A;
      const SurfView<double> &v = side ? vb : va;
      timed(ctx, "basis", [&] { launch_basis(v, S, st, Batch{}, static_cast<const SurfView<double> *>(nullptr), true); }, 2.0 * S.nreg * S.g.nuv);
      timed(ctx, "samples", [&] { launch_samples(v, S, false, st); }, double(S.nreg) * S.g.nuv * S.g.nuv);
      timed(ctx, "pad", [&] { launch_pad_bound(S, v, dtab[side], side ? eb : ea, st); });
      timed(ctx, "cells", [&] { launch_cells(S, true, st); }, double(S.nreg) * S.g.W * S.g.W);
    }
    const unsigned long long tile_pairs = static_cast<unsigned long long>(nslots) * A.g.ntiles * B.g.ntiles;
    if (tile_pairs > kMaxTilePairs) fail(JSI_ERR_CAPACITY, "%llu tile pairs exceed the screen's list", tile_pairs);
    const int ij_bits = std::max(1, bit_width(static_cast<unsigned long long>(
                                            std::max(A.g.W * A.g.W, B.g.W * B.g.W) - 1)));
    const int slot_bits = std::max(1, bit_width(static_cast<unsigned long long>(nslots - 1)));
    if (2 * ij_bits + slot_bits > 64) fail(JSI_ERR_CAPACITY, "pair key does not fit 64 bits");
    unsigned long long *surv = ar.get<unsigned long long>(tile_pairs);
    const double prune = std::nextafter((1.0 - p->rel_tol) * ub, 0.0);
    const double ub2 = std::nextafter(prune * prune, INFINITY);
    reset_stats(ctx);
    timed(ctx, "bound_cull", [&] {
      launch_bound_cull(A, B, map1, map2, static_cast<int>(nslots), ub2, surv, tile_pairs, ctx->d_stats, st);
    });
    pull_stats(ctx);
    const unsigned long long nsurv = ctx->h_stats->survivors;
    unsigned long long key_cap =
        std::max<unsigned long long>(1ull << 16, std::min<unsigned long long>(nsurv * 64, 1ull << 24));
    unsigned long long *keys = ar.get<unsigned long long>(key_cap);
    for (int attempt = 0;; ++attempt) {
      timed(ctx, "bound_leaf", [&] {
        launch_bound_leaf(A, B, map1, map2, surv, nsurv, ij_bits, ub2, keys, key_cap, ctx->d_stats, st);
      });
      pull_stats(ctx);
      ScreenStats &hs = *ctx->h_stats;
      if (hs.candidates <= key_cap) break;
      if (attempt >= 1) fail(JSI_ERR_CAPACITY, "bounds pair list overflow");
      key_cap = hs.candidates;
      keys = ar.get<unsigned long long>(key_cap);
      hs.candidates = 0;
      hs.pair_tests = 0;
      hs.work = 0;
      hs.lb_bits = 0x7ff0000000000000ull;
      hs.ub_bits = 0x7ff0000000000000ull;
      JSI_CUDA(copy_async(ctx, ctx->d_stats, &hs, sizeof(ScreenStats), cudaMemcpyHostToDevice, st));
    }
    const long long n = static_cast<long long>(ctx->h_stats->candidates);
    double g2;
    const unsigned long long gb = ctx->h_stats->lb_bits;
    std::memcpy(&g2, &gb, sizeof(g2));
    // Every point pair lies in some cell pair; a pair whose gap exceeds ub
    // cannot hold the minimum, so the smallest kept gap bounds it from below.
    // (The pair holding the ub points is always kept, so n >= 1.)
    const double lr = n > 0 ? std::nextafter(std::sqrt(g2), 0.0) : prune;
    lb = std::max(lb, std::min(lr, prune));
    double c2;
    const unsigned long long cb = ctx->h_stats->ub_bits;
    std::memcpy(&c2, &cb, sizeof(c2));
    if (n > 0 && c2 < INFINITY) {
      const double uc = std::nextafter(std::nextafter(std::sqrt(c2), INFINITY) + allowance, INFINITY);
      ub = std::min(ub, uc);
    }
    lb = std::min(lb, ub);
    out->kept[round - 1] = n;
    out->pair_tests[round - 1] = static_cast<long long>(ctx->h_stats->pair_tests);
    out->lb_round[round - 1] = lb;
    out->rounds_run = round;
    add_units(ctx, "bound_leaf", static_cast<double>(ctx->h_stats->pair_tests));
    if (n == 0 || ub - lb <= p->rel_tol * ub) {
      out->certified = 1;
      break;
    }
    if (round == p->max_rounds || n == 0 || n > p->max_pairs) break;
    unsigned long long *sorted = keys;
    if (n > 1) {
      const int end_bit = 2 * ij_bits + slot_bits;
      unsigned long long *alt = ar.get<unsigned long long>(n);
      size_t tmp_bytes = 0;
      cub::DoubleBuffer<unsigned long long> db(keys, alt);
      JSI_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, static_cast<int>(n), 0, end_bit, st));
      void *tmp = ar.alloc(tmp_bytes);
      timed(ctx, "sort_pairs", [&] {
        JSI_CUDA(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, static_cast<int>(n), 0, end_bit, st));
      });
      sorted = db.Current();
    }
    RegionRec<double> *next1, *next2;
    int *nmap1, *nmap2, r1, r2;
    next_regions<double>(ctx, sorted, n, ij_bits, slot_bits, A, B, map1, map2, true, &next1, &next2, &nmap1, &nmap2,
                         &r1, &r2);
    A = bounds_side(make_geom(p->nuv_refine, p1_of(sa)), r1, next1);
    B = bounds_side(make_geom(p->nuv_refine, p1_of(sb)), r2, next2);
    map1 = nmap1;
    map2 = nmap2;
    nslots = n;
  }
  out->lb = lb;
  out->ub = ub;
}

// ---------------------------------------------------------------------------
// Intersection curves: refined points linked into polylines
// ---------------------------------------------------------------------------

struct CurvePoint {
  double x[3];
  double uvst[4];
  double t[3];  // unit tangent
};

// Uniform hash grid over the points (cell = link tolerance).
class PointGrid {
 public:
  PointGrid(const std::vector<CurvePoint> &pts, double cell) : pts_(pts), cell_(cell) {
    for (size_t q = 0; q < pts.size(); ++q) cells_[key(pts[q].x)].push_back(static_cast<int>(q));
  }
  template <typename Fn>
  void near(const double *x, Fn &&fn) const {
    const long long ix = cellc(x[0]), iy = cellc(x[1]), iz = cellc(x[2]);
    for (long long a = ix - 1; a <= ix + 1; ++a)
      for (long long b = iy - 1; b <= iy + 1; ++b)
        for (long long c = iz - 1; c <= iz + 1; ++c) {
          auto it = cells_.find(pack(a, b, c));
          if (it == cells_.end()) continue;
          for (int q : it->second) fn(q);
        }
  }

 private:
  long long cellc(double v) const { return static_cast<long long>(std::floor(v / cell_)); }
  static long long pack(long long a, long long b, long long c) {
    return ((a & 0x1fffff) << 42) | ((b & 0x1fffff) << 21) | (c & 0x1fffff);
  }
  long long key(const double *x) const { return pack(cellc(x[0]), cellc(x[1]), cellc(x[2])); }
  const std::vector<CurvePoint> &pts_;
  double cell_;
  std::unordered_map<long long, std::vector<int>> cells_;
};

double dist3(const double *a, const double *b) {
  const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
  return std::sqrt(dx * dx + dy * dy + dz * dz);
}

// Walks from point c along direction d (unit): each step goes to the nearest
// unvisited point ahead within tol; points nearer than it along the curve
// (ahead or behind) are absorbed, and so are repeats of a point (closer than
// 1e-6 tol: several cell pairs refine to the same curve point, and a step
// onto a repeat would take an arbitrary direction).
std::vector<int> walk_curve(const std::vector<CurvePoint> &pts, const PointGrid &grid, std::vector<char> &visited,
                            int c, double d[3], double tol) {
  std::vector<int> path;
  for (;;) {
    int best = -1;
    double bd = INFINITY;
    grid.near(pts[c].x, [&](int o) {
      if (visited[o]) return;
      const double v[3] = {pts[o].x[0] - pts[c].x[0], pts[o].x[1] - pts[c].x[1], pts[o].x[2] - pts[c].x[2]};
      const double dist = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      if (dist <= 1e-6 * tol) {
        visited[o] = 1;  // the same point again
        return;
      }
      if (dist > tol) return;
      const double along = v[0] * d[0] + v[1] * d[1] + v[2] * d[2];
      if (along > 0.3 * dist && dist < bd) {
        bd = dist;
        best = o;
      }
    });
    if (best < 0) break;
    grid.near(pts[c].x, [&](int o) {
      if (visited[o] || o == best) return;
      const double v[3] = {pts[o].x[0] - pts[c].x[0], pts[o].x[1] - pts[c].x[1], pts[o].x[2] - pts[c].x[2]};
      const double dist = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      const double along = v[0] * d[0] + v[1] * d[1] + v[2] * d[2];
      if (dist < bd && std::fabs(along) >= 0.7 * dist) visited[o] = 1;
    });
    visited[best] = 1;
    path.push_back(best);
    const double v[3] = {pts[best].x[0] - pts[c].x[0], pts[best].x[1] - pts[c].x[1], pts[best].x[2] - pts[c].x[2]};
    const double s = v[0] * pts[best].t[0] + v[1] * pts[best].t[1] + v[2] * pts[best].t[2] >= 0.0 ? 1.0 : -1.0;
    for (int k = 0; k < 3; ++k) d[k] = s * pts[best].t[k];
    c = best;
  }
  return path;
}

void link_curves(const std::vector<CurvePoint> &pts, double tol, std::vector<std::vector<int>> &curves,
                 std::vector<int> &closed) {
  if (pts.empty() || !(tol > 0.0)) return;
  PointGrid grid(pts, tol);
  std::vector<char> visited(pts.size(), 0);
  for (size_t s = 0; s < pts.size(); ++s) {
    if (visited[s]) continue;
    visited[s] = 1;
    double d[3] = {pts[s].t[0], pts[s].t[1], pts[s].t[2]};
    std::vector<int> fwd = walk_curve(pts, grid, visited, static_cast<int>(s), d, tol);
    const bool loop = fwd.size() >= 3 && dist3(pts[fwd.back()].x, pts[s].x) <= tol;
    std::vector<int> curve;
    if (!loop) {
      double e[3] = {-pts[s].t[0], -pts[s].t[1], -pts[s].t[2]};
      std::vector<int> bwd = walk_curve(pts, grid, visited, static_cast<int>(s), e, tol);
      curve.assign(bwd.rbegin(), bwd.rend());
    }
    curve.push_back(static_cast<int>(s));
    curve.insert(curve.end(), fwd.begin(), fwd.end());
    if (curve.size() >= 2) {
      curves.push_back(std::move(curve));
      closed.push_back(loop ? 1 : 0);
    }
  }
}

// The FP64 intersection query with Newton points, tangents on the device,
// then the links on the host.
void run_curves(Lane *L, const jsi_task *ta, const jsi_task *tb, const jsi_curve_params *p, jsi_curve_result *out) {
  jsi_inter_result ir;
  std::memset(&ir, 0, sizeof(ir));
  jsi_inter_params ip = p->inter;
  ip.points = 1;
  FinalRound<double> fin;
  run_intersection<double>(L, ta, tb, &ip, &ir, &fin, true);
  const double *dpts = fin.points;
  const long long np = fin.n;
  std::vector<CurvePoint> pts;
  std::vector<double> scales;
  if (np > 0 && dpts) {
    const SurfaceRec &sa = get_surface(L, ta->surface);
    const SurfaceRec &sb = get_surface(L, tb->surface);
    double *dtan = L->arena.get<double>(static_cast<size_t>(np) * 5);
    timed(L, "curve_tangents", [&] {
      launch_curve_tangents(view<double>(sa), view<double>(sb), fin.reg1, fin.reg2, fin.map1, fin.map2, fin.nuv1,
                            fin.nuv2, fin.keys, fin.ij_bits, dpts, np, dtan, L->stream);
    });
    std::vector<double> hp(static_cast<size_t>(np) * 8), ht(static_cast<size_t>(np) * 5);
    JSI_CUDA(copy_async(L, hp.data(), dpts, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    JSI_CUDA(copy_async(L, ht.data(), dtan, ht.size() * sizeof(double), cudaMemcpyDeviceToHost, L->stream));
    JSI_CUDA(cudaStreamSynchronize(L->stream));
    for (long long q = 0; q < np; ++q) {
      const double *x = hp.data() + q * 8, *t = ht.data() + q * 5;
      const double scale = 1.0 + std::fabs(x[0]) + std::fabs(x[1]) + std::fabs(x[2]);
      if (!(x[7] <= 1e-9 * scale) || t[3] == 0.0) continue;  // not converged / no tangent
      CurvePoint cp;
      for (int k = 0; k < 3; ++k) {
        cp.x[k] = x[k];
        cp.t[k] = t[k];
      }
      for (int k = 0; k < 4; ++k) cp.uvst[k] = x[3 + k];
      pts.push_back(cp);
      scales.push_back(t[4]);
    }
  }
  out->points_found = static_cast<long long>(pts.size());
  // Default tolerance: 4 x the median size of the cells the points were
  // refined from (on the covering grid consecutive points come from
  // neighbouring cells).
  double tol = p->link_tol;
  if (!(tol > 0.0) && !scales.empty()) {
    std::nth_element(scales.begin(), scales.begin() + scales.size() / 2, scales.end());
    tol = 4.0 * scales[scales.size() / 2];
  }
  out->link_tol = tol;
  std::vector<std::vector<int>> curves;
  std::vector<int> closed;
  link_curves(pts, tol, curves, closed);
  long long nv = 0;
  for (const auto &cv : curves) nv += static_cast<long long>(cv.size());
  out->vertices = nv;
  out->curves = static_cast<long long>(curves.size());
  if (nv > out->vertex_cap || out->curves > out->curve_cap || (nv > 0 && (!out->vertex || !out->curve_start)))
    fail(JSI_ERR_CAPACITY, "%lld vertices / %lld curves do not fit the buffers (%lld / %lld)", nv, out->curves,
         out->vertex_cap, out->curve_cap);
  long long w = 0;
  for (size_t k = 0; k < curves.size(); ++k) {
    out->curve_start[k] = w;
    if (out->curve_closed) out->curve_closed[k] = closed[k];
    for (int q : curves[k]) {
      double *v = out->vertex + w * 7;
      for (int c = 0; c < 3; ++c) v[c] = pts[q].x[c];
      for (int c = 0; c < 4; ++c) v[3 + c] = pts[q].uvst[c];
      ++w;
    }
  }
  if (out->curve_start) out->curve_start[curves.size()] = w;
}



void check_precision(int prec, bool screen_built) {
  if (prec != JSI_PREC_V5_FP32 && prec != JSI_PREC_FP64 && prec != JSI_PREC_FP32_SCREEN)
    fail(JSI_ERR_INVALID, "unknown precision %d", prec);
  if (prec == JSI_PREC_FP32_SCREEN && !screen_built) fail(JSI_ERR_UNSUPPORTED, "FP32-screen form not built for this query");
}

// Lane set-up / tear-down.
void lane_init(Lane &L, int device, size_t block, size_t budget, const std::map<int, SurfaceRec> *surfaces,
               std::atomic<size_t> *shared = nullptr, size_t shared_cap = 0) {
  L.device = device;
  L.surfaces = surfaces;
  L.arena.configure(block, budget, shared, shared_cap);
  JSI_CUDA(cudaSetDevice(device));
  JSI_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
  JSI_CUDA(cudaEventCreate(&L.ev0));
  JSI_CUDA(cudaEventCreate(&L.ev1));
  JSI_CUDA(cudaMalloc(&L.d_stats, sizeof(ScreenStats)));
  JSI_CUDA(cudaMallocHost(&L.h_stats, sizeof(ScreenStats)));
  JSI_CUDA(cudaMallocHost(&L.h_small, 8 * sizeof(unsigned long long)));
}

void lane_free(Lane &L) {
  if (L.stream) cudaStreamSynchronize(L.stream);
  for (auto &p : L.pending) {
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  L.pending.clear();
  for (auto e : L.event_pool) cudaEventDestroy(e);
  L.event_pool.clear();
  if (L.d_stats) cudaFree(L.d_stats);
  if (L.h_stats) cudaFreeHost(L.h_stats);
  if (L.h_small) cudaFreeHost(L.h_small);
  L.h_small = nullptr;
  for (auto &g : L.graphs)
    if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
  L.graphs.clear();
  if (L.h_pin) cudaFreeHost(L.h_pin);
  L.h_pin = nullptr;
  L.h_pin_bytes = 0;
  if (L.ev0) cudaEventDestroy(L.ev0);
  if (L.ev1) cudaEventDestroy(L.ev1);
  if (L.stream) cudaStreamDestroy(L.stream);
  L.d_stats = nullptr;
  L.h_stats = nullptr;
  L.ev0 = L.ev1 = nullptr;
  L.stream = nullptr;
}

void validate_dist(jsi_dist_params &p, const jsi_task *a, const jsi_task *b) {
  if (p.k < 1 || p.k > kMaxK) fail(JSI_ERR_INVALID, "k = %d outside [1, %d]", p.k, kMaxK);
  if (p.rounds < 1 || p.rounds > JSI_MAX_ROUNDS) fail(JSI_ERR_INVALID, "rounds = %d", p.rounds);
  if (p.nuv_refine < 2 || p.nuv_refine > 4096) fail(JSI_ERR_INVALID, "nuv_refine = %d", p.nuv_refine);
  check_precision(p.precision, true);
  check_task<float>(a);
  check_task<float>(b);
}

void validate_inter(jsi_inter_params &p, const jsi_task *a, const jsi_task *b) {
  if (p.rounds < 1 || p.rounds > JSI_MAX_ROUNDS) fail(JSI_ERR_INVALID, "rounds = %d", p.rounds);
  if (p.nuv_refine < 2 || p.nuv_refine > 4096) fail(JSI_ERR_INVALID, "nuv_refine = %d", p.nuv_refine);
  if (p.min_nuv < 2) fail(JSI_ERR_INVALID, "min_nuv = %d", p.min_nuv);
  check_precision(p.precision, true);
  check_task<float>(a);
  check_task<float>(b);
}

// One distance query on one lane (arena rewound, device time in out->device_ms).
void exec_distance(Lane *L, const jsi_task *a, const jsi_task *b, const jsi_dist_params &p, jsi_dist_result *out) {
  int *tp = out->trace_pairs;
  const long long tc = out->trace_cap;
  int *cp = out->cand_pairs;
  double *cd = out->cand_d2;
  const long long cc = out->cand_cap;
  std::memset(out, 0, sizeof(*out));
  out->trace_pairs = tp;
  out->trace_cap = tc;
  out->cand_pairs = cp;
  out->cand_d2 = cd;
  out->cand_cap = cc;
  out->newton_distance = -1.0;
  JSI_CUDA(cudaSetDevice(L->device));
  L->arena.reset();
  JSI_CUDA(cudaEventRecord(L->ev0, L->stream));
  if (p.precision == JSI_PREC_V5_FP32)
    run_distance<float, float>(L, a, b, &p, out);
  else if (p.precision == JSI_PREC_FP64)
    run_distance<double, double>(L, a, b, &p, out);
  else
    run_distance<double, float>(L, a, b, &p, out);
  JSI_CUDA(cudaEventRecord(L->ev1, L->stream));
  JSI_CUDA(cudaEventSynchronize(L->ev1));
  JSI_CUDA(cudaEventElapsedTime(&out->device_ms, L->ev0, L->ev1));
  resolve_timing(L);
}

void exec_intersection(Lane *L, const jsi_task *a, const jsi_task *b, const jsi_inter_params &p,
                       jsi_inter_result *out) {
  int *tp = out->trace_pairs;
  const long long tc = out->trace_cap;
  double *pts = out->points;
  const long long pc = out->points_cap;
  int *sp = out->screen_pairs;
  const long long sc = out->screen_cap;
  std::memset(out, 0, sizeof(*out));
  out->trace_pairs = tp;
  out->trace_cap = tc;
  out->points = pts;
  out->points_cap = pc;
  out->screen_pairs = sp;
  out->screen_cap = sc;
  JSI_CUDA(cudaSetDevice(L->device));
  L->arena.reset();
  JSI_CUDA(cudaEventRecord(L->ev0, L->stream));
  // FP32_SCREEN: the first round screens in FP32 and re-checks in FP64, so
  // every round's pairs equal the FP64 form's.
  if (p.precision == JSI_PREC_V5_FP32)
    run_intersection<float>(L, a, b, &p, out);
  else
    run_intersection<double>(L, a, b, &p, out, nullptr, false, p.precision == JSI_PREC_FP32_SCREEN);
  JSI_CUDA(cudaEventRecord(L->ev1, L->stream));
  JSI_CUDA(cudaEventSynchronize(L->ev1));
  JSI_CUDA(cudaEventElapsedTime(&out->device_ms, L->ev0, L->ev1));
  resolve_timing(L);
}

int run_guarded(std::string &err, const std::function<void()> &fn);

// A lockstep batch on one lane; every item gets the batch's device time.
// Items flagged by the batch (a list overflowed) are re-run alone.
void exec_distance_batch(Lane *L, std::vector<BatchItem> &items, const jsi_dist_params &p) {
  JSI_CUDA(cudaSetDevice(L->device));
  L->arena.reset();
  for (auto &it : items) {
    int *tp = it.out->trace_pairs;
    const long long tc = it.out->trace_cap;
    std::memset(it.out, 0, sizeof(*it.out));
    it.out->trace_pairs = tp;
    it.out->trace_cap = tc;
    it.out->newton_distance = -1.0;
    it.status = JSI_OK;
  }
  JSI_CUDA(cudaEventRecord(L->ev0, L->stream));
  int rerun = 0;
  if (p.precision == JSI_PREC_V5_FP32)
    rerun = run_distance_batch<float, float>(L, items, p);
  else if (p.precision == JSI_PREC_FP64)
    rerun = run_distance_batch<double, double>(L, items, p);
  else
    rerun = run_distance_batch<double, float>(L, items, p);
  JSI_CUDA(cudaEventRecord(L->ev1, L->stream));
  JSI_CUDA(cudaEventSynchronize(L->ev1));
  float ms = 0.0f;
  JSI_CUDA(cudaEventElapsedTime(&ms, L->ev0, L->ev1));
  L->batch_reruns += rerun;
  for (auto &it : items) {
    if (it.status == JSI_OK) {
      it.out->device_ms = ms;
      continue;
    }
    it.status = run_guarded(it.error, [&] { exec_distance(L, it.a, it.b, p, it.out); });
  }
}

int run_guarded(std::string &err, const std::function<void()> &fn) {
  try {
    fn();
    return JSI_OK;
  } catch (const StatusError &e) {
    err = e.msg;
    return e.status;
  } catch (const CudaError &e) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at line %d", static_cast<int>(e.err),
             cudaGetErrorString(e.err), e.what, e.line);
    err = buf;
    return JSI_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    err = "host allocation failed";
    return JSI_ERR_NOMEM;
  }
}

std::vector<int> job_surfaces(const Job &j) {
  if (j.kind != 2) return {j.a.surface, j.b.surface};
  std::vector<int> ids;
  ids.reserve(2 * j.items.size());
  for (const auto &it : j.items) {
    ids.push_back(it.a->surface);
    ids.push_back(it.b->surface);
  }
  return ids;
}

void release_refs(jsi_context *ctx, const Job &j) {
  std::lock_guard<std::mutex> lk(ctx->surf_mu);
  for (int id : job_surfaces(j)) {
    auto it = ctx->surface_refs.find(id);
    if (it != ctx->surface_refs.end() && --it->second <= 0) ctx->surface_refs.erase(it);
  }
}

// Worker: takes queued queries in arrival order and runs them on its lane.
void worker_loop(jsi_context *ctx, Lane *L) {
  cudaSetDevice(L->device);
  for (;;) {
    std::shared_ptr<Job> job;
    {
      std::unique_lock<std::mutex> lk(ctx->qmu);
      ctx->qcv.wait(lk, [&] { return ctx->stopping || !ctx->queue.empty(); });
      if (ctx->queue.empty()) return;  // stopping and drained
      job = ctx->queue.front();
      ctx->queue.pop_front();
      ++ctx->busy;
    }
    job->status = run_guarded(job->error, [&] {
      {
        std::lock_guard<std::mutex> lk(ctx->surf_mu);
        JSI_CUDA(cudaStreamWaitEvent(L->stream, ctx->upload_ev, 0));
      }
      if (job->kind == 0)
        exec_distance(L, &job->a, &job->b, job->dp, &job->dres);
      else if (job->kind == 1)
        exec_intersection(L, &job->a, &job->b, job->ip, &job->ires);
      else
        exec_distance_batch(L, job->items, job->dp);
      if (!job->end_ev) JSI_CUDA(cudaEventCreate(&job->end_ev));
      JSI_CUDA(cudaEventRecord(job->end_ev, L->stream));
    });
    release_refs(ctx, *job);
    if (L->arena.held() > ctx->lane_keep) L->arena.trim(ctx->lane_keep);
    {
      std::lock_guard<std::mutex> lk(ctx->qmu);
      job->done = true;
      --ctx->busy;
    }
    ctx->dcv.notify_all();
  }
}

void stop_workers(jsi_context *ctx) {
  {
    std::lock_guard<std::mutex> lk(ctx->qmu);
    ctx->stopping = true;
  }
  ctx->qcv.notify_all();
  for (auto &t : ctx->threads) t.join();
  ctx->threads.clear();
  // Per-kernel timing totals outlive the lanes (kept on the main lane).
  for (auto &L : ctx->lanes) {
    for (auto &kv : L->kernel_ms) {
      auto &acc = ctx->main.kernel_ms[kv.first];
      acc.first += kv.second.first;
      acc.second += kv.second.second;
    }
    for (auto &kv : L->kernel_units) ctx->main.kernel_units[kv.first] += kv.second;
  }
  for (auto &L : ctx->lanes) lane_free(*L);
  ctx->lanes.clear();
  ctx->stopping = false;
}

void start_workers(jsi_context *ctx, int n) {
  // Lanes grow their arenas in 512 MiB blocks as used, all drawing on the
  // budget left beside the resident surfaces (or each up to lane_bytes when
  // the caller set it); after a query a lane keeps at most an even share.
  const size_t left = ctx->budget > ctx->resident ? ctx->budget - ctx->resident : 0;
  const size_t cap = ctx->lane_bytes ? ctx->lane_bytes : left;
  ctx->lane_keep = n > 0 ? std::max<size_t>(size_t(512) << 20, left / n) : 0;
  for (int q = 0; q < n; ++q) {
    auto L = std::make_unique<Lane>();
    lane_init(*L, ctx->device, std::min(cap, size_t(512) << 20), cap, &ctx->surfaces, &ctx->lane_held, left);
    L->surfaces_mu = &ctx->surf_mu;
    L->graphs_on = ctx->batch_graphs;
    L->timing = ctx->main.timing.load();  // per-kernel timing follows the context's setting
    ctx->lanes.push_back(std::move(L));
  }
  for (auto &L : ctx->lanes) ctx->threads.emplace_back(worker_loop, ctx, L.get());
}

long long enqueue(jsi_context *ctx, std::shared_ptr<Job> job) {
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    const std::vector<int> ids = job_surfaces(*job);
    for (int id : ids)
      if (!ctx->surfaces.count(id)) fail(JSI_ERR_INVALID, "unknown surface id %d", id);
    std::lock_guard<std::mutex> ls(ctx->surf_mu);
    for (int id : ids) ++ctx->surface_refs[id];
  }
  long long t;
  {
    std::lock_guard<std::mutex> lk(ctx->qmu);
    t = ctx->next_ticket++;
    ctx->jobs[t] = job;
    ctx->queue.push_back(job);
  }
  ctx->qcv.notify_one();
  return t;
}

}  // namespace

extern "C" {

int jsi_abi_version(void) { return JSI_B200_ABI_VERSION; }

const char *jsi_status_string(int status) {
  switch (status) {
    case JSI_OK: return "ok";
    case JSI_ERR_INVALID: return "invalid argument";
    case JSI_ERR_CUDA: return "CUDA error";
    case JSI_ERR_NOMEM: return "out of device memory / budget";
    case JSI_ERR_CAPACITY: return "capacity exceeded";
    case JSI_ERR_SURFACE: return "malformed surface";
    case JSI_ERR_TIMEOUT: return "device wait timed out";
    case JSI_ERR_UNSUPPORTED: return "unsupported";
    case JSI_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char *jsi_last_error(const jsi_context *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int jsi_create(const jsi_config *cfg, jsi_context **out) {
  if (!out) return JSI_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return JSI_ERR_NO_DEVICE;
  }
  const int dev = cfg ? cfg->device : 0;
  if (dev < 0 || dev >= ndev) return JSI_ERR_INVALID;
  jsi_context *ctx = new (std::nothrow) jsi_context();
  if (!ctx) return JSI_ERR_NOMEM;
  ctx->device = dev;
  const size_t arena = (cfg && cfg->arena_bytes) ? cfg->arena_bytes : (size_t(2) << 30);
  ctx->budget = (cfg && cfg->hbm_budget_bytes) ? cfg->hbm_budget_bytes : (size_t(120) << 30);
  const int st = guarded(ctx, [&]() {
    lane_init(ctx->main, dev, arena, ctx->budget, &ctx->surfaces);
    JSI_CUDA(cudaMallocHost(reinterpret_cast<void **>(&ctx->ring), kRingSeg * kRingSegs));
    JSI_CUDA(cudaMalloc(reinterpret_cast<void **>(&ctx->dring), kRingSeg * kRingSegs));
    for (auto &e : ctx->ring_ev) {
      JSI_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      JSI_CUDA(cudaEventRecord(e, ctx->main.stream));
    }
    JSI_CUDA(cudaEventCreateWithFlags(&ctx->upload_ev, cudaEventDisableTiming));
    JSI_CUDA(cudaEventRecord(ctx->upload_ev, ctx->main.stream));
    {
      // Upload-path host threads beside the caller: up to 7 by default,
      // JSI_HOST_THREADS (0..63) overrides.
      const int hw = static_cast<int>(std::thread::hardware_concurrency());
      int nt = std::min(7, std::max(0, hw - 1));
      if (const char *v = std::getenv("JSI_HOST_THREADS"); v && *v)
        nt = static_cast<int>(std::min(63L, std::max(0L, std::strtol(v, nullptr, 10))));
      if (nt > 0) ctx->hpool = std::make_unique<HostPool>(nt);
      ctx->main.hpool = ctx->hpool.get();
    }
    return JSI_OK;
  });
  if (st != JSI_OK) {
    jsi_destroy(ctx);
    return st;
  }
  *out = ctx;
  return JSI_OK;
}

int jsi_destroy(jsi_context *ctx) {
  if (!ctx) return JSI_ERR_INVALID;
  cudaSetDevice(ctx->device);
  stop_workers(ctx);
  if (ctx->main.stream) cudaStreamSynchronize(ctx->main.stream);
  ctx->surfaces.clear();  // pooled blocks go with the pool
  for (auto &e : ctx->ring_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->upload_ev) cudaEventDestroy(ctx->upload_ev);
  if (ctx->ring) cudaFreeHost(ctx->ring);
  if (ctx->dring) cudaFree(ctx->dring);
  for (auto &b : ctx->host_blocks) cudaFreeHost(reinterpret_cast<void *>(b.first));
  ctx->host_blocks.clear();
  lane_free(ctx->main);
  delete ctx;
  return JSI_OK;
}

int jsi_host_alloc(jsi_context *ctx, unsigned long long bytes, void **ptr) {
  if (!ctx || !ptr || bytes == 0) return JSI_ERR_INVALID;
  *ptr = nullptr;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    JSI_CUDA(cudaSetDevice(ctx->device));
    void *p = nullptr;
    if (cudaMallocHost(&p, static_cast<size_t>(bytes)) != cudaSuccess) {
      cudaGetLastError();
      fail(JSI_ERR_NOMEM, "cudaMallocHost of %llu bytes failed", bytes);
    }
    ctx->host_blocks[reinterpret_cast<uintptr_t>(p)] = static_cast<size_t>(bytes);
    *ptr = p;
    return JSI_OK;
  });
}

int jsi_host_free(jsi_context *ctx, void *ptr) {
  if (!ctx || !ptr) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->host_blocks.find(reinterpret_cast<uintptr_t>(ptr));
  if (it == ctx->host_blocks.end()) return record(ctx, JSI_ERR_INVALID, "not a block of jsi_host_alloc");
  // Uploads copy from these blocks asynchronously on the main stream.
  if (ctx->main.stream) cudaStreamSynchronize(ctx->main.stream);
  cudaFreeHost(ptr);
  ctx->host_blocks.erase(it);
  return JSI_OK;
}

int jsi_surface_upload(jsi_context *ctx, const int ivec[7], const float *data, int ndata, jsi_surface_id *out) {
  if (!ctx || !out) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    JSI_CUDA(cudaSetDevice(ctx->device));
    SurfaceRec s = upload_resident(ctx, ivec, data, ndata);
    ctx->resident += s.bytes;
    const int id = ctx->next_id++;
    std::lock_guard<std::mutex> ls(ctx->surf_mu);
    ctx->surfaces[id] = s;
    *out = id;
    return JSI_OK;
  });
}

int jsi_surface_release(jsi_context *ctx, jsi_surface_id id) {
  if (!ctx) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  std::lock_guard<std::mutex> ls(ctx->surf_mu);
  auto it = ctx->surfaces.find(id);
  if (it == ctx->surfaces.end()) return record(ctx, JSI_ERR_INVALID, "unknown surface id");
  if (ctx->surface_refs.count(id)) return record(ctx, JSI_ERR_INVALID, "surface is used by a queued query");
  // No query holds the surface: its block returns to the pool at once (a
  // later upload into it is ordered after this one's copies on the main
  // stream).
  ctx->resident -= it->second.bytes;
  ctx->pool.put(it->second.block, it->second.block_bytes);
  ctx->surfaces.erase(it);
  return JSI_OK;
}

int jsi_surface_release_many(jsi_context *ctx, int n, const jsi_surface_id *ids) {
  if (!ctx || n < 0 || (n > 0 && !ids)) return JSI_ERR_INVALID;
  for (int q = 0; q < n; ++q) {
    const int st = jsi_surface_release(ctx, ids[q]);
    if (st != JSI_OK) return st;
  }
  return JSI_OK;
}

int jsi_surface_domains(jsi_context *ctx, int n, const jsi_surface_id *ids, float *rects) {
  if (!ctx || n < 0 || (n > 0 && (!ids || !rects))) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (int q = 0; q < n; ++q) {
    auto it = ctx->surfaces.find(ids[q]);
    if (it == ctx->surfaces.end()) return record(ctx, JSI_ERR_INVALID, "unknown surface id");
    std::memcpy(rects + 4 * static_cast<size_t>(q), it->second.dom, sizeof(it->second.dom));
  }
  return JSI_OK;
}

int jsi_surface_upload_many(jsi_context *ctx, int n, const int *ivecs, const float *const *datas, const int *ndatas,
                            jsi_surface_id *out) {
  if (!ctx || n < 0 || (n > 0 && (!ivecs || !datas || !ndatas || !out))) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  int done = 0;
  const int st = guarded(ctx, [&]() {
    JSI_CUDA(cudaSetDevice(ctx->device));
    std::vector<PendingSurface> in;
    in.reserve(n);
    for (int q = 0; q < n; ++q) in.push_back(PendingSurface{ivecs + 7 * q, datas[q], ndatas[q]});
    std::vector<SurfaceRec> recs;
    recs.reserve(n);
    try {
      upload_resident_many(ctx, in, recs);
    } catch (...) {
      for (auto &r : recs) ctx->pool.put(r.block, r.block_bytes);  // none becomes resident
      throw;
    }
    std::lock_guard<std::mutex> ls(ctx->surf_mu);
    for (; done < n; ++done) {
      ctx->resident += recs[done].bytes;
      const int id = ctx->next_id++;
      ctx->surfaces[id] = recs[done];
      out[done] = id;
    }
    return JSI_OK;
  });
  for (int q = done; q < n; ++q) out[q] = 0;
  return st;
}

int jsi_resident_bytes(const jsi_context *ctx, unsigned long long *out) {
  if (!ctx || !out) return JSI_ERR_INVALID;
  *out = ctx->resident;
  return JSI_OK;
}

int jsi_context_stream(jsi_context *ctx, void **stream) {
  if (!ctx || !stream) return JSI_ERR_INVALID;
  *stream = static_cast<void *>(ctx->main.stream);
  return JSI_OK;
}

int jsi_transfer_bytes(const jsi_context *ctx, unsigned long long *h2d, unsigned long long *d2h) {
  if (!ctx || !h2d || !d2h) return JSI_ERR_INVALID;
  *h2d = ctx->main.h2d_bytes;
  *d2h = ctx->main.d2h_bytes;
  for (auto &L : ctx->lanes) {
    *h2d += L->h2d_bytes;
    *d2h += L->d2h_bytes;
  }
  return JSI_OK;
}

int jsi_kernel_timing(jsi_context *ctx, int enable) {
  if (!ctx) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto set = [&](Lane &L) {
    std::lock_guard<std::mutex> ls(L.stats_mu);
    L.timing = enable != 0;
    L.kernel_ms.clear();
    L.kernel_units.clear();
    // Events of unresolved launches go back to the pool (re-recording an
    // event that is still pending on the stream is allowed).
    for (auto &pe : L.pending) {
      L.event_pool.push_back(pe.second.first);
      L.event_pool.push_back(pe.second.second);
    }
    L.pending.clear();
  };
  set(ctx->main);
  for (auto &L : ctx->lanes) set(*L);
  return JSI_OK;
}

int jsi_kernel_time(jsi_context *ctx, const char *name, double *total_ms, long long *launches) {
  if (!ctx || !name || !total_ms || !launches) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  *total_ms = 0.0;
  *launches = 0;
  auto add = [&](Lane &L) {
    std::lock_guard<std::mutex> ls(L.stats_mu);
    auto it = L.kernel_ms.find(name);
    if (it != L.kernel_ms.end()) {
      *total_ms += it->second.first;
      *launches += it->second.second;
    }
  };
  add(ctx->main);
  for (auto &L : ctx->lanes) add(*L);
  return JSI_OK;
}

int jsi_kernel_units(jsi_context *ctx, const char *name, double *units) {
  if (!ctx || !name || !units) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  *units = 0.0;
  auto add = [&](Lane &L) {
    std::lock_guard<std::mutex> ls(L.stats_mu);
    auto it = L.kernel_units.find(name);
    if (it != L.kernel_units.end()) *units += it->second;
  };
  add(ctx->main);
  for (auto &L : ctx->lanes) add(*L);
  return JSI_OK;
}

const char *jsi_kernel_names(jsi_context *ctx) {
  if (!ctx) return "";
  std::lock_guard<std::mutex> lk(ctx->mu);
  std::map<std::string, int> names;
  for (auto &kv : ctx->main.kernel_ms) names[kv.first] = 1;
  for (auto &L : ctx->lanes) {
    std::lock_guard<std::mutex> ls(L->stats_mu);
    for (auto &kv : L->kernel_ms) names[kv.first] = 1;
  }
  ctx->kernel_names.clear();
  for (auto &kv : names) {
    if (!ctx->kernel_names.empty()) ctx->kernel_names += ",";
    ctx->kernel_names += kv.first;
  }
  return ctx->kernel_names.c_str();
}

int jsi_launch_count(unsigned long long *out) {
  if (!out) return JSI_ERR_INVALID;
  *out = jsi::launch_count();
  return JSI_OK;
}

void jsi_dist_params_default(jsi_dist_params *p) {
  if (!p) return;
  p->nuv_refine = 16;
  p->k = 8;
  p->rounds = 4;
  p->precision = JSI_PREC_V5_FP32;
  p->newton = 0;
}

void jsi_inter_params_default(jsi_inter_params *p) {
  if (!p) return;
  p->nuv_refine = 16;
  p->use_k = 1;
  p->rounds = 6;
  p->halve_threshold = 512;
  p->min_nuv = 4;
  p->precision = JSI_PREC_V5_FP32;
  p->points = 0;
}

int jsi_min_distance(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_dist_params *params,
                     jsi_dist_result *out) {
  if (!ctx || !a || !b || !out) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    jsi_dist_params p;
    jsi_dist_params_default(&p);
    if (params) p = *params;
    validate_dist(p, a, b);
    exec_distance(&ctx->main, a, b, p, out);
    return JSI_OK;
  });
}

void jsi_curve_params_default(jsi_curve_params *p) {
  if (!p) return;
  jsi_inter_params_default(&p->inter);
  p->inter.precision = JSI_PREC_FP64;
  p->inter.points = 1;
  p->link_tol = 0.0;
}

int jsi_intersection_curves(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_curve_params *params,
                            jsi_curve_result *out) {
  if (!ctx || !a || !b || !out) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    jsi_curve_params p;
    jsi_curve_params_default(&p);
    if (params) p = *params;
    p.inter.precision = JSI_PREC_FP64;
    validate_inter(p.inter, a, b);
    if (!(p.link_tol >= 0.0)) fail(JSI_ERR_INVALID, "link_tol must be >= 0");
    out->points_found = out->vertices = out->curves = 0;
    out->link_tol = 0.0;
    out->device_ms = 0.0f;
    Lane *L = &ctx->main;
    JSI_CUDA(cudaSetDevice(L->device));
    L->arena.reset();
    JSI_CUDA(cudaEventRecord(L->ev0, L->stream));
    run_curves(L, a, b, &p, out);
    JSI_CUDA(cudaEventRecord(L->ev1, L->stream));
    JSI_CUDA(cudaEventSynchronize(L->ev1));
    JSI_CUDA(cudaEventElapsedTime(&out->device_ms, L->ev0, L->ev1));
    resolve_timing(L);
    return JSI_OK;
  });
}

void jsi_bounds_params_default(jsi_bounds_params *p) {
  if (!p) return;
  p->nuv_refine = 8;
  p->max_rounds = 10;
  p->rel_tol = 1e-6;
  p->max_pairs = 1ll << 22;
}

int jsi_surface_curvature_bounds(const int *ivec, const float *data, int ndata, const double *rect, double *m2u,
                                 double *m2v) {
  if (!ivec || !data || !m2u || !m2v) return JSI_ERR_INVALID;
  try {
    check_surface(ivec, data, ndata);
    SurfaceRec s;
    surface_header(s, ivec, data);
    if (s.rat && !(s.wmin > 0)) return JSI_ERR_UNSUPPORTED;
    if (!rect) {
      second_derivative_bounds_host(ivec, data, m2u, m2v);
      return JSI_OK;
    }
    // The bounds mode's per-region rule: the largest per-span bound over the
    // spans the rectangle touches, its upper ends looked up just below.
    const int p = ivec[1], q = ivec[4], nsu = ivec[2] - p;
    const std::vector<Vec4<double>> tab = span_curvature_table(ivec, data);
    std::vector<double> U(data, data + ivec[3]), V(data + ivec[3], data + ivec[3] + ivec[6]);
    auto span = [](const std::vector<double> &K, int deg, double u) {
      const int n = static_cast<int>(K.size()) - deg - 1;
      if (u <= K[deg]) return deg;
      if (u >= K[n]) return n - 1;
      int k = deg;
      while (k + 1 < n && K[k + 1] <= u) ++k;
      return k;
    };
    const double ulo = std::min(rect[0], rect[2]), uhi = std::max(rect[0], rect[2]);
    const double vlo = std::min(rect[1], rect[3]), vhi = std::max(rect[1], rect[3]);
    const int su0 = span(U, p, ulo), su1 = span(U, p, uhi > ulo ? std::nextafter(uhi, ulo) : uhi);
    const int sv0 = span(V, q, vlo), sv1 = span(V, q, vhi > vlo ? std::nextafter(vhi, vlo) : vhi);
    for (int c = 0; c < 3; ++c) m2u[c] = m2v[c] = 0.0;
    for (int sv = sv0; sv <= sv1; ++sv)
      for (int su = su0; su <= su1; ++su) {
        const size_t k = 2 * (static_cast<size_t>(sv - q) * nsu + (su - p));
        const double a[3] = {tab[k].x, tab[k].y, tab[k].z}, b[3] = {tab[k + 1].x, tab[k + 1].y, tab[k + 1].z};
        for (int c = 0; c < 3; ++c) {
          m2u[c] = std::max(m2u[c], a[c]);
          m2v[c] = std::max(m2v[c], b[c]);
        }
      }
    return JSI_OK;
  } catch (const StatusError &e) {
    return e.status;
  } catch (const std::bad_alloc &) {
    return JSI_ERR_NOMEM;
  }
}

int jsi_distance_bounds(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_bounds_params *params,
                        jsi_bounds_result *out) {
  if (!ctx || !a || !b || !out) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    jsi_bounds_params p;
    jsi_bounds_params_default(&p);
    if (params) p = *params;
    if (p.nuv_refine < 2 || p.nuv_refine > 64) fail(JSI_ERR_INVALID, "nuv_refine = %d", p.nuv_refine);
    if (p.max_rounds < 1 || p.max_rounds > JSI_MAX_ROUNDS) fail(JSI_ERR_INVALID, "max_rounds = %d", p.max_rounds);
    if (!(p.rel_tol >= 0.0)) fail(JSI_ERR_INVALID, "rel_tol must be >= 0");
    if (p.max_pairs < 1) fail(JSI_ERR_INVALID, "max_pairs = %lld", p.max_pairs);
    check_task<double>(a);
    check_task<double>(b);
    std::memset(out, 0, sizeof(*out));
    Lane *L = &ctx->main;
    JSI_CUDA(cudaSetDevice(L->device));
    L->arena.reset();
    JSI_CUDA(cudaEventRecord(L->ev0, L->stream));
    run_bounds(L, a, b, &p, out);
    JSI_CUDA(cudaEventRecord(L->ev1, L->stream));
    JSI_CUDA(cudaEventSynchronize(L->ev1));
    JSI_CUDA(cudaEventElapsedTime(&out->device_ms, L->ev0, L->ev1));
    resolve_timing(L);
    return JSI_OK;
  });
}

int jsi_intersect(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_inter_params *params,
                  jsi_inter_result *out) {
  if (!ctx || !a || !b || !out) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    jsi_inter_params p;
    jsi_inter_params_default(&p);
    if (params) p = *params;
    validate_inter(p, a, b);
    exec_intersection(&ctx->main, a, b, p, out);
    return JSI_OK;
  });
}

int jsi_workers(jsi_context *ctx, int n, unsigned long long lane_bytes) {
  if (!ctx || n < 0 || n > 256) return JSI_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(ctx->qmu);
    if (!ctx->queue.empty() || ctx->busy) return record(ctx, JSI_ERR_INVALID, "queries are still queued");
  }
  stop_workers(ctx);
  ctx->lane_bytes = lane_bytes;
  return guarded(ctx, [&]() {
    start_workers(ctx, n);
    return JSI_OK;
  });
}

int jsi_submit_distance(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_dist_params *params,
                        int *trace_pairs, long long trace_cap, jsi_ticket *out) {
  if (!ctx || !a || !b || !out) return JSI_ERR_INVALID;
  return guarded(ctx, [&]() {
    if (ctx->lanes.empty()) fail(JSI_ERR_INVALID, "no worker lanes (call jsi_workers first)");
    auto job = std::make_shared<Job>();
    job->kind = 0;
    job->a = *a;
    job->b = *b;
    jsi_dist_params_default(&job->dp);
    if (params) job->dp = *params;
    validate_dist(job->dp, a, b);
    job->dres.trace_pairs = trace_pairs;
    job->dres.trace_cap = trace_cap;
    *out = enqueue(ctx, job);
    return JSI_OK;
  });
}

int jsi_submit_intersect(jsi_context *ctx, const jsi_task *a, const jsi_task *b, const jsi_inter_params *params,
                         int *trace_pairs, long long trace_cap, jsi_ticket *out) {
  if (!ctx || !a || !b || !out) return JSI_ERR_INVALID;
  return guarded(ctx, [&]() {
    if (ctx->lanes.empty()) fail(JSI_ERR_INVALID, "no worker lanes (call jsi_workers first)");
    auto job = std::make_shared<Job>();
    job->kind = 1;
    job->a = *a;
    job->b = *b;
    jsi_inter_params_default(&job->ip);
    if (params) job->ip = *params;
    validate_inter(job->ip, a, b);
    job->ires.trace_pairs = trace_pairs;
    job->ires.trace_cap = trace_cap;
    job->ires.points = nullptr;
    job->ires.points_cap = 0;
    *out = enqueue(ctx, job);
    return JSI_OK;
  });
}

int jsi_wait(jsi_context *ctx, jsi_ticket ticket, int timeout_ms, jsi_dist_result *dist, jsi_inter_result *inter) {
  if (!ctx) return JSI_ERR_INVALID;
  std::shared_ptr<Job> job;
  {
    std::unique_lock<std::mutex> lk(ctx->qmu);
    auto it = ctx->jobs.find(ticket);
    if (it == ctx->jobs.end()) return record(ctx, JSI_ERR_INVALID, "unknown ticket");
    job = it->second;
    auto ready = [&] { return job->done; };
    if (timeout_ms < 0)
      ctx->dcv.wait(lk, ready);
    else if (!ctx->dcv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
      return JSI_ERR_TIMEOUT;
    ctx->jobs.erase(ticket);
  }
  if (dist && job->kind == 0) *dist = job->dres;
  if (inter && job->kind == 1) *inter = job->ires;
  if (job->status != JSI_OK) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_error = job->error;
  }
  return job->status;
}

int jsi_queue_depth(jsi_context *ctx, int *queued, int *running) {
  if (!ctx || !queued || !running) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->qmu);
  *queued = static_cast<int>(ctx->queue.size());
  *running = ctx->busy;
  return JSI_OK;
}

int jsi_batch_chunk(jsi_context *ctx, int chunk) {
  if (!ctx || chunk < 0 || chunk > 65535) return JSI_ERR_INVALID;
  ctx->batch_chunk = chunk;
  return JSI_OK;
}

int jsi_batch_graphs(jsi_context *ctx, int enable, long long *replays) {
  if (!ctx) return JSI_ERR_INVALID;
  if (enable >= 0) {
    ctx->batch_graphs = enable != 0;
    for (auto &L : ctx->lanes) L->graphs_on = ctx->batch_graphs;
  }
  if (replays) {
    long long t = 0;
    for (auto &L : ctx->lanes) t += L->graph_replays;
    *replays = t;
  }
  return JSI_OK;
}

int jsi_autotune_batch(jsi_context *ctx, int n, const jsi_task *a, const jsi_task *b, const jsi_dist_params *params,
                       int *chunk_out, float *ms_out) {
  if (!ctx || n < 1 || !a || !b) return JSI_ERR_INVALID;
  if (ctx->lanes.empty()) return record(ctx, JSI_ERR_INVALID, "no worker lanes (call jsi_workers first)");
  jsi_dist_params p;
  jsi_dist_params_default(&p);
  if (params) p = *params;
  std::array<int, 4> shape{};
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    const int st = guarded(ctx, [&]() {
      validate_dist(p, &a[0], &b[0]);
      auto ia = ctx->surfaces.find(a[0].surface), ib = ctx->surfaces.find(b[0].surface);
      if (ia == ctx->surfaces.end() || ib == ctx->surfaces.end()) fail(JSI_ERR_INVALID, "unknown surface id");
      shape = {a[0].nuv, b[0].nuv, shape_of(ia->second), shape_of(ib->second)};
      for (int q = 1; q < n; ++q) {
        auto qa = ctx->surfaces.find(a[q].surface), qb = ctx->surfaces.find(b[q].surface);
        if (qa == ctx->surfaces.end() || qb == ctx->surfaces.end()) fail(JSI_ERR_INVALID, "unknown surface id");
        const std::array<int, 4> s2 = {a[q].nuv, b[q].nuv, shape_of(qa->second), shape_of(qb->second)};
        if (s2 != shape) fail(JSI_ERR_INVALID, "autotune queries differ in shape");
      }
      return JSI_OK;
    });
    if (st != JSI_OK) return st;
  }
  const std::array<int, 7> key = {shape[0], shape[1], shape[2], shape[3], p.k, p.rounds, p.precision};
  ctx->tuned_chunk.erase(key);
  const int saved = ctx->batch_chunk;
  std::vector<jsi_dist_result> out(n);
  int best = saved > 0 ? saved : 64;
  float best_ms = INFINITY;
  // Candidates: powers of two up to the largest per-lane share of the batch.
  const int nl = static_cast<int>(ctx->lanes.size());
  const int most = std::max(1, (n + nl - 1) / nl);
  for (int chunk = 8; chunk <= std::max(8, most); chunk *= 2) {
    ctx->batch_chunk = chunk;
    float ms = 0.0f;
    int st = JSI_OK;
    for (int rep = 0; rep < 3 && st == JSI_OK; ++rep) {  // one warm run, then the faster of two
      std::memset(out.data(), 0, sizeof(jsi_dist_result) * out.size());
      float t = 0.0f;
      st = jsi_min_distance_batch(ctx, n, a, b, &p, out.data(), nullptr, &t);
      if (rep == 1 || (rep == 2 && t < ms)) ms = t;
    }
    if (st != JSI_OK) {
      ctx->batch_chunk = saved;
      return st;
    }
    if (ms < best_ms) {
      best_ms = ms;
      best = chunk;
    }
  }
  ctx->batch_chunk = saved;
  ctx->tuned_chunk[key] = best;
  if (chunk_out) *chunk_out = best;
  if (ms_out) *ms_out = best_ms;
  return JSI_OK;
}

int jsi_batch_reruns(jsi_context *ctx, long long *out) {
  if (!ctx || !out) return JSI_ERR_INVALID;
  long long t = 0;
  for (auto &L : ctx->lanes) t += L->batch_reruns;
  *out = t;
  return JSI_OK;
}

int jsi_submit_distance_batch(jsi_context *ctx, int n, const jsi_task *a, const jsi_task *b,
                              const jsi_dist_params *params, jsi_dist_result *out, int *status, jsi_ticket *ticket) {
  if (!ctx || n < 0 || (n > 0 && (!a || !b || !out)) || !ticket) return JSI_ERR_INVALID;
  if (ctx->lanes.empty()) return record(ctx, JSI_ERR_INVALID, "no worker lanes (call jsi_workers first)");
  jsi_dist_params p;
  jsi_dist_params_default(&p);
  if (params) p = *params;
  auto pb = std::make_unique<PendingBatch>();
  pb->out = out;
  pb->status = status;
  pb->first_err = JSI_OK;
  PendingBatch &B = *pb;
  auto set_status = [&](int q, int st) {
    if (status) status[q] = st;
    if (st != JSI_OK && B.first_err == JSI_OK) B.first_err = st;
  };
  // Start of the batch's device span: an event on the main stream after the
  // uploads issued before this call.  Lane streams are not touched here (a
  // lane may be capturing a CUDA graph); each job waits for the uploads on
  // its own lane before it starts.
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    const int st = guarded(ctx, [&]() {
      JSI_CUDA(cudaSetDevice(ctx->device));
      JSI_CUDA(cudaEventCreate(&B.ev0));
      JSI_CUDA(cudaEventRecord(B.ev0, ctx->main.stream));
      return JSI_OK;
    });
    if (st != JSI_OK) return st;
  }
  const bool lockstep = ctx->batch_chunk > 0 && p.k >= 1 && p.k <= kBatchK && p.rounds >= 1 &&
                        p.rounds <= kBatchRounds;
  auto job_of = [&](jsi_ticket t) {
    std::lock_guard<std::mutex> lk(ctx->qmu);
    auto it = ctx->jobs.find(t);
    return it != ctx->jobs.end() ? it->second : std::shared_ptr<Job>();
  };
  if (lockstep) {
    // Group by first-round nuv and zero flags of both sides; degrees and
    // rational flags may differ within a group (a mixed lockstep batch).
    // shapes[q] keeps each query's shape key for the autotuner's table.
    std::map<std::array<int, 4>, std::vector<int>> groups;
    std::vector<std::array<int, 2>> shapes(static_cast<size_t>(n));
    for (int q = 0; q < n; ++q) {
      std::string err;
      std::array<int, 4> key{};
      const int st = run_guarded(err, [&] {
        validate_dist(p, &a[q], &b[q]);
        std::lock_guard<std::mutex> lk(ctx->mu);
        auto ia = ctx->surfaces.find(a[q].surface), ib = ctx->surfaces.find(b[q].surface);
        if (ia == ctx->surfaces.end() || ib == ctx->surfaces.end()) fail(JSI_ERR_INVALID, "unknown surface id");
        key = {a[q].nuv, b[q].nuv, ia->second.zero, ib->second.zero};
        shapes[q] = {shape_of(ia->second), shape_of(ib->second)};
      });
      if (st != JSI_OK) {
        set_status(q, st);
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->last_error = err;
        continue;
      }
      groups[key].push_back(q);
    }
    const int nl = static_cast<int>(ctx->lanes.size());
    for (auto &g : groups) {
      const int m = static_cast<int>(g.second.size());
      const int q0 = g.second[0];
      const std::array<int, 7> tk = {g.first[0], g.first[1], shapes[q0][0], shapes[q0][1], p.k, p.rounds, p.precision};
      auto tit = ctx->tuned_chunk.find(tk);
      const int chunk = tit != ctx->tuned_chunk.end() ? tit->second : ctx->batch_chunk;
      const int per = std::max(1, std::min(chunk, (m + nl - 1) / nl));
      for (int s0 = 0; s0 < m; s0 += per) {
        auto job = std::make_shared<Job>();
        job->kind = 2;
        job->dp = p;
        for (int t = s0; t < std::min(m, s0 + per); ++t) {
          const int q = g.second[t];
          BatchItem it;
          it.a = &a[q];
          it.b = &b[q];
          it.out = &out[q];
          job->items.push_back(it);
        }
        jsi_ticket t = 0;
        const int st = guarded(ctx, [&]() {
          t = enqueue(ctx, job);
          return JSI_OK;
        });
        if (st != JSI_OK) {
          for (int u = s0; u < std::min(m, s0 + per); ++u) set_status(g.second[u], st);
          continue;
        }
        B.tickets.push_back(t);
        B.solo.push_back(-1);
        B.batch_jobs.push_back(job);
        B.all_jobs.push_back(job);
      }
    }
  } else {
    for (int q = 0; q < n; ++q) {
      jsi_ticket t = 0;
      const int st = jsi_submit_distance(ctx, &a[q], &b[q], &p, out[q].trace_pairs, out[q].trace_cap, &t);
      if (st != JSI_OK) {
        set_status(q, st);
        continue;
      }
      B.tickets.push_back(t);
      B.solo.push_back(q);
      if (auto j = job_of(t)) B.all_jobs.push_back(j);
    }
  }
  {
    std::lock_guard<std::mutex> lk(ctx->qmu);
    *ticket = ctx->next_ticket++;
    ctx->batches[*ticket] = std::move(pb);
  }
  return JSI_OK;
}

int jsi_poll_distance_batch(jsi_context *ctx, jsi_ticket ticket, int *done) {
  if (!ctx || !done) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->qmu);
  auto it = ctx->batches.find(ticket);
  if (it == ctx->batches.end()) return record(ctx, JSI_ERR_INVALID, "unknown batch ticket");
  int all = 1;
  for (auto &j : it->second->all_jobs)
    if (!j->done) all = 0;
  *done = all;
  return JSI_OK;
}

int jsi_wait_distance_batch(jsi_context *ctx, jsi_ticket ticket, float *device_ms) {
  if (!ctx) return JSI_ERR_INVALID;
  std::unique_ptr<PendingBatch> pb;
  {
    std::lock_guard<std::mutex> lk(ctx->qmu);
    auto it = ctx->batches.find(ticket);
    if (it == ctx->batches.end()) return record(ctx, JSI_ERR_INVALID, "unknown batch ticket");
    pb = std::move(it->second);
    ctx->batches.erase(it);
  }
  PendingBatch &B = *pb;
  jsi_dist_result *out = B.out;
  auto set_status = [&](int q, int st) {
    if (B.status) B.status[q] = st;
    if (st != JSI_OK && B.first_err == JSI_OK) B.first_err = st;
  };
  size_t bj = 0;
  for (size_t w = 0; w < B.tickets.size(); ++w) {
    if (B.solo[w] >= 0) {
      set_status(B.solo[w], jsi_wait(ctx, B.tickets[w], -1, &out[B.solo[w]], nullptr));
      continue;
    }
    const int st = jsi_wait(ctx, B.tickets[w], -1, nullptr, nullptr);
    Job &job = *B.batch_jobs[bj++];
    for (auto &it : job.items) {
      const int q = static_cast<int>(it.out - out);
      const int sq = st != JSI_OK ? st : it.status;
      set_status(q, sq);
      if (sq != JSI_OK && !it.error.empty()) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->last_error = it.error;
      }
    }
  }
  // Device span: from the start event to the last job's end (each job's end
  // event is recorded on its lane's stream after its work).
  std::lock_guard<std::mutex> lk(ctx->mu);
  const int st = guarded(ctx, [&]() {
    float span = 0.0f;
    for (auto &j : B.all_jobs) {
      if (!j->end_ev) continue;
      JSI_CUDA(cudaEventSynchronize(j->end_ev));
      float ms = 0.0f;
      JSI_CUDA(cudaEventElapsedTime(&ms, B.ev0, j->end_ev));
      span = std::max(span, ms);
    }
    if (device_ms) *device_ms = span;
    return JSI_OK;
  });
  return B.first_err != JSI_OK ? B.first_err : st;
}

int jsi_query_batch(jsi_context *ctx, int n, const int *kinds, const jsi_task *a, const jsi_task *b,
                    const jsi_dist_params *dp, const jsi_inter_params *ip, jsi_dist_result *dist_out,
                    jsi_inter_result *inter_out, int *status, float *device_ms) {
  if (!ctx || n < 0 || (n > 0 && (!kinds || !a || !b))) return JSI_ERR_INVALID;
  if (ctx->lanes.empty()) return record(ctx, JSI_ERR_INVALID, "no worker lanes (call jsi_workers first)");
  std::vector<int> di, ii;
  for (int q = 0; q < n; ++q) {
    if (kinds[q] == 0) di.push_back(q);
    else if (kinds[q] == 1) ii.push_back(q);
    else return record(ctx, JSI_ERR_INVALID, "query kind must be 0 (distance) or 1 (intersection)");
  }
  if ((!di.empty() && !dist_out) || (!ii.empty() && !inter_out)) return JSI_ERR_INVALID;
  int first_err = JSI_OK;
  auto set_status = [&](int q, int st) {
    if (status) status[q] = st;
    if (st != JSI_OK && first_err == JSI_OK) first_err = st;
  };
  cudaEvent_t ev0 = nullptr;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    const int st = guarded(ctx, [&]() {
      JSI_CUDA(cudaSetDevice(ctx->device));
      JSI_CUDA(cudaEventCreate(&ev0));
      JSI_CUDA(cudaEventRecord(ev0, ctx->main.stream));
      return JSI_OK;
    });
    if (st != JSI_OK) return st;
  }
  // Intersections first, the largest first-round grids first, so that the
  // long jobs start early and the distance batches fill the lanes last.
  std::sort(ii.begin(), ii.end(), [&](int x, int y) {
    const long long wx = 1ll * a[x].nuv * a[x].nuv + 1ll * b[x].nuv * b[x].nuv;
    const long long wy = 1ll * a[y].nuv * a[y].nuv + 1ll * b[y].nuv * b[y].nuv;
    return wx != wy ? wx > wy : x < y;
  });
  jsi_inter_params ipv;
  jsi_inter_params_default(&ipv);
  if (ip) ipv = *ip;
  std::vector<std::pair<int, jsi_ticket>> itick;
  std::vector<std::shared_ptr<Job>> ijobs;
  for (int q : ii) {
    jsi_ticket t = 0;
    std::shared_ptr<Job> job;
    const int st = guarded(ctx, [&]() {
      validate_inter(ipv, &a[q], &b[q]);
      job = std::make_shared<Job>();
      job->kind = 1;
      job->a = a[q];
      job->b = b[q];
      job->ip = ipv;
      const jsi_inter_result &tpl = inter_out[q];
      job->ires.trace_pairs = tpl.trace_pairs;
      job->ires.trace_cap = tpl.trace_cap;
      job->ires.points = tpl.points;
      job->ires.points_cap = tpl.points_cap;
      job->ires.screen_pairs = tpl.screen_pairs;
      job->ires.screen_cap = tpl.screen_cap;
      t = enqueue(ctx, job);
      return JSI_OK;
    });
    if (st != JSI_OK) {
      set_status(q, st);
      continue;
    }
    itick.push_back({q, t});
    ijobs.push_back(job);
  }
  // Distance queries: the lockstep batches of jsi_submit_distance_batch over
  // compacted copies of their tasks and results.
  const int nd = static_cast<int>(di.size());
  std::vector<jsi_task> da(nd), db(nd);
  std::vector<jsi_dist_result> dres(nd);
  std::vector<int> dst(nd, JSI_OK);
  for (int e = 0; e < nd; ++e) {
    da[e] = a[di[e]];
    db[e] = b[di[e]];
    dres[e] = dist_out[di[e]];
  }
  jsi_ticket dt = 0;
  int dsub = JSI_OK;
  if (nd > 0) dsub = jsi_submit_distance_batch(ctx, nd, da.data(), db.data(), dp, dres.data(), dst.data(), &dt);
  for (auto &qt : itick) set_status(qt.first, jsi_wait(ctx, qt.second, -1, nullptr, &inter_out[qt.first]));
  float dms = 0.0f;
  if (nd > 0) {
    int dw = dsub;
    if (dsub == JSI_OK) dw = jsi_wait_distance_batch(ctx, dt, &dms);
    for (int e = 0; e < nd; ++e) {
      dist_out[di[e]] = dres[e];
      set_status(di[e], dsub != JSI_OK ? dsub : dst[e]);
    }
    if (dw != JSI_OK && first_err == JSI_OK) first_err = dw;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  const int st = guarded(ctx, [&]() {
    float span = dms;  // the distance batch's span starts after ev0
    for (auto &j : ijobs) {
      if (!j->end_ev) continue;
      JSI_CUDA(cudaEventSynchronize(j->end_ev));
      float ms = 0.0f;
      JSI_CUDA(cudaEventElapsedTime(&ms, ev0, j->end_ev));
      span = std::max(span, ms);
    }
    if (device_ms) *device_ms = span;
    return JSI_OK;
  });
  cudaEventDestroy(ev0);
  return first_err != JSI_OK ? first_err : st;
}

int jsi_min_distance_batch(jsi_context *ctx, int n, const jsi_task *a, const jsi_task *b,
                           const jsi_dist_params *params, jsi_dist_result *out, int *status, float *device_ms) {
  jsi_ticket t = 0;
  const int st = jsi_submit_distance_batch(ctx, n, a, b, params, out, status, &t);
  if (st != JSI_OK) return st;
  return jsi_wait_distance_batch(ctx, t, device_ms);
}

}  // extern "C"

namespace {
template <typename T>
int eval_grid_impl(jsi_context *ctx, const int ivec[7], const float *data, int ndata, T ustep, T vstep, T ustart,
                   T vstart, int nuv, T *results) {
  if (!ctx || !results) return JSI_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return guarded(ctx, [&]() {
    if (nuv < 1 || nuv > 8192) fail(JSI_ERR_INVALID, "nuv = %d", nuv);
    Lane *L = &ctx->main;
    JSI_CUDA(cudaSetDevice(ctx->device));
    L->arena.reset();
    SurfaceRec s = upload_surface(L, ivec, data, ndata, &L->arena);
    const size_t n = static_cast<size_t>(nuv) * nuv * 18;
    T *d = L->arena.get<T>(n);
    launch_records(view<T>(s), ustep, vstep, ustart, vstart, nuv, d, L->stream);
    JSI_CUDA(cudaGetLastError());
    JSI_CUDA(copy_async(L, results, d, n * sizeof(T), cudaMemcpyDeviceToHost, L->stream));
    JSI_CUDA(cudaStreamSynchronize(L->stream));
    return JSI_OK;
  });
}
}  // namespace

extern "C" {

int jsi_eval_grid(jsi_context *ctx, const int ivec[7], const float *data, int ndata, float ustep, float vstep,
                  float ustart, float vstart, int nuv, float *results) {
  return eval_grid_impl<float>(ctx, ivec, data, ndata, ustep, vstep, ustart, vstart, nuv, results);
}

int jsi_eval_grid_f64(jsi_context *ctx, const int ivec[7], const float *data, int ndata, double ustep,
                      double vstep, double ustart, double vstart, int nuv, double *results) {
  return eval_grid_impl<double>(ctx, ivec, data, ndata, ustep, vstep, ustart, vstart, nuv, results);
}

}  // extern "C"
