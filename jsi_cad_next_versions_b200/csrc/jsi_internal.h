// Internal declarations shared by the kernels and the host orchestration.
//
// Layout in HBM (per round, per side):
//   regions  RegionRec<T>[R]              parameter rectangle of each unique region
//   spans    int[R][2][nuv]               knot span of every grid line (u lines, then v lines)
//   basis    T[R][2][nuv][3][p1max]       basis values and 1st/2nd derivatives per line
//   samples  T4[R][nuv*nuv]               P of every sample (x, y, z, 0), u fastest
//   kmax     ordered bits[R][3]           max |Puu|, |Puv|, |Pvv| over the grid (curvature padding)
//   cells    T4 centre[R][cpr], T4 half[R][cpr]
//            tile-major: cpr = ntiles*te*te; tile (ty, tx) holds cells
//            iv in [ty*te, ty*te+te), iu in [tx*te, tx*te+te) clipped to W
//   tiles    T4 lo[R][ntiles], T4 hi[R][ntiles], T4 hmax[R][ntiles]
// Cell id (the reference's bbox id) = iv * W + iu with W = nuv - 1.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace jsi {

constexpr int kMaxDeg = 25;   // degrees >= kMaxDeg evaluate to zero records (evaluation.cu:13,272)
constexpr int kMaxTile = 8;   // tile edge in cells
constexpr int kMaxK = 1024;   // largest top-k supported
constexpr int kSelectCap = 4096;  // entries the top-k select can sort on chip

template <typename T>
struct alignas(4 * sizeof(T) > 16 ? 16 : 4 * sizeof(T)) Vec4 {
  T x, y, z, w;
};

// Surface as the kernels see it.  cpw = control points with weight,
// (x, y, z, w) per point, u fastest; w = 1 for non-rational surfaces.
template <typename T>
struct SurfView {
  int degu, degv, ncpu, ncpv, nku, nkv;
  int rat;   // rational
  int zero;  // every record is zero (evaluation.cu:271-272)
  int du, dv;
  const T *U;
  const T *V;
  const Vec4<T> *cpw;
};

// Unsigned encodings that order like the float / double they encode
// (non-negative: bits with the sign bit set; negative: complemented bits), so
// integer atomicMin / atomicMax compute exact float minima / maxima.
template <typename T>
struct OrdBits;
template <>
struct OrdBits<float> {
  using type = unsigned;
};
template <>
struct OrdBits<double> {
  using type = unsigned long long;
};

template <typename T>
struct RegionRec {
  T u0, v0, u1, v1;
};

// Sampling geometry shared by all regions of one side in one round.
struct Geom {
  int nuv;    // samples per direction
  int W;      // cells per direction
  int te;     // tile edge
  int tw;     // tiles per direction
  int ntiles; // tw * tw
  int cpr;    // padded cells per region = ntiles * te * te
  int p1max;  // basis stride (max degree + 1)
  int stw;    // supertiles (8 x 8 tiles) per direction
  int nst;    // stw * stw
};

inline Geom make_geom(int nuv, int p1max) {
  Geom g;
  g.nuv = nuv;
  g.W = nuv - 1;
  g.te = g.W < kMaxTile ? g.W : kMaxTile;
  if (g.te < 1) g.te = 1;
  g.tw = (g.W + g.te - 1) / g.te;
  g.ntiles = g.tw * g.tw;
  g.cpr = g.ntiles * g.te * g.te;
  g.p1max = p1max;
  g.stw = (g.tw + kMaxTile - 1) / kMaxTile;
  g.nst = g.stw * g.stw;
  return g;
}

// One side's data of one round.
template <typename T>
struct SideRound {
  Geom g;
  int nreg;
  RegionRec<T> *regions;
  int *spans;
  T *basis;
  Vec4<T> *samples;
  unsigned long long *kmax;  // 3 per region, ordered bits of non-negative T
  T *pad;                    // curvature padding per region
  Vec4<T> *center;
  Vec4<T> *half;
  Vec4<T> *tlo;
  Vec4<T> *thi;
  Vec4<T> *thmax;
  Vec4<T> *stlo;  // supertile bounds [R][nst] (built on demand)
  Vec4<T> *sthi;
  const int *dnreg;  // when set: the region count lives on the device (batched rounds)
  // When set (batched rounds): supertile bounds folded in by the cell
  // kernels as encoded [R][nst][4] minima / maxima (OrdBits), used in place
  // of stlo / sthi.
  typename OrdBits<T>::type *stmin;
  typename OrdBits<T>::type *stmax;
};

// Candidate of the distance screen.
template <typename T>
struct DistCand {
  T d2;
  int slot, i, j;
};

// Counters one screening round accumulates on the device.
struct ScreenStats {
  unsigned long long tile_pairs;    // tile pairs examined
  unsigned long long survivors;     // tile pairs that passed the bound
  unsigned long long pair_tests;    // cell pairs tested
  unsigned long long candidates;    // cell pairs that passed the screen
  unsigned int tau_bits;            // float bits of the current distance threshold
  int status;                       // 0 ok, otherwise a jsi_status
  int nsel;                         // pairs kept by the select
  int nreg1, nreg2;                 // unique regions built for the next round
  int pad_;
  unsigned long long work;          // work counter of the persistent leaf kernels
  unsigned long long st_survivors;  // supertile pairs that passed the bound
  unsigned long long nhead;         // tile pairs in the threshold pass's list (batched rounds)
  int nslots;                       // slots of this round (batched rounds)
  int pad2_;
  unsigned long long lb_bits;       // bounds mode: smallest kept squared box gap (double bits)
  unsigned long long ub_bits;       // bounds mode: smallest corner-sample squared distance (double bits)
  unsigned long long checked;       // intersection FP32 screen: candidates the FP64 re-check kept
  unsigned long long rechecked;     // intersection FP32 screen: samples re-evaluated for the exact compute_K maxima
};

// Lockstep batch of queries that share one shape: query q runs in
// blockIdx.y = q and finds every per-query array at the query-0 address plus
// q * qs bytes (one slab per query, identical layouts).  n = 1, qs = 0 is the
// single-query launch.
struct Batch {
  int n = 1;
  long long qs = 0;
};

// Count arguments with this value are read from the device (ScreenStats).
constexpr unsigned long long kFromDevice = ~0ull;

// Batched distance form: limits and the per-query record it leaves in the
// query's slab (read back with one strided copy per batch).
constexpr int kBatchRounds = 8;  // rounds a batched query may run
constexpr int kBatchK = 8;       // largest k of the batched form
constexpr int kStatusCapacity = -4;  // JSI_ERR_CAPACITY

template <typename TP>
struct DistRecord {
  long long tests[kBatchRounds];
  long long cands[kBatchRounds];
  unsigned long long survivors[kBatchRounds];
  unsigned long long examined[kBatchRounds];  // tile pairs whose bound or representative was evaluated
  unsigned long long st_kept[kBatchRounds];   // supertile pairs that passed their bound
  int npairs[kBatchRounds];
  int status[kBatchRounds];
  DistCand<TP> top[kBatchRounds][kBatchK];
  double newton[kBatchK * 11];
};

// A surviving tile pair: (row = slot * ntiles1 + t1) << 32 | t2.
__host__ __device__ inline unsigned long long pack_tile_pair(unsigned row, unsigned t2) {
  return (static_cast<unsigned long long>(row) << 32) | t2;
}

// ---- launchers (jsi_kernels.cu) ----
// Every distance-path launcher takes an optional Batch (default: one query).
// In a batch the per-query arrays sit in slabs qs bytes apart; surfaces come
// from the slabs through the vdev pointers; counts given as kFromDevice (or a
// negative slot count -max) are read from each query's ScreenStats, with the
// host value (or cap) only bounding the grid.
unsigned long long launch_count();  // kernels launched so far (all contexts)
void add_launches(unsigned long long n);  // kernels a replayed CUDA graph launched
// cover: sample the covering grid (nuv samples over the whole rectangle, the
// last on its end) of the bounds mode instead of the reference's grid.
// values_only: leave the derivative rows zero (the distance path reads the
// basis values alone).
template <typename T>
void launch_basis(const SurfView<T> &s, const SideRound<T> &sr, cudaStream_t st, const Batch &bt = Batch{},
                  const SurfView<T> *vdev = nullptr, bool cover = false, bool values_only = false);
template <typename T>
void launch_samples(const SurfView<T> &s, const SideRound<T> &sr, bool need_k, cudaStream_t st,
                    const Batch &bt = Batch{}, const SurfView<T> *vdev = nullptr);
template <typename T>
void launch_pad(const SideRound<T> &sr, bool use_k, T span_u0, T span_v0, cudaStream_t st);
template <typename T>
void launch_cells(const SideRound<T> &sr, bool intersect, cudaStream_t st, const Batch &bt = Batch{});
// Limits of the fused region kernel: samples per direction and basis stride
// (degree + 1).
constexpr int kRegNuv = 16;
constexpr int kRegP1 = 9;
// Intersection sides of small regions (nuv <= 16, degree <= 8): basis,
// samples, compute_K padding, cells and tile ranges of every region in one
// launch, bit-identical to launch_basis + launch_samples + launch_pad +
// launch_cells (the basis tables and sample grid are not written).
template <typename T>
bool region_cells_fits(const SideRound<T> &sr);
template <typename T>
void launch_region_cells(const SurfView<T> &s, const SideRound<T> &sr, bool need_k, T span_u0, T span_v0, bool cover,
                         cudaStream_t st);
template <typename T>
void launch_records(const SurfView<T> &s, T ustep, T vstep, T ustart, T vstart, int nuv, T *out, cudaStream_t st);

// Whether the single-level threshold seed can fold anything: a block folds
// the k-th of its 256 threads' minima, and only threads t2 < ntiles of side
// B see a tile pair, so with fewer than k tiles on that side (4 at nuv 16,
// where k = 8) no block folds and the launch would change nothing.
inline bool dist_tau_folds(const Geom &gb, int k) { return k <= 256 && gb.ntiles >= k; }

// screen = true (float only): FP32-screen thresholds with centre-error bound e.
template <typename T>
void launch_dist_tau(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                     int k, ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt = Batch{});
template <typename T>
void launch_dist_cull(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                      unsigned long long *surv, unsigned *surv_lb, unsigned long long surv_cap, ScreenStats *stats,
                      bool screen, float e, cudaStream_t st, const Batch &bt = Batch{});
// sorted: surv is ordered by surv_lb (a warp stops at the first bound above
// tau); otherwise tile pairs whose bound exceeds tau are skipped.
// collect = 0: only tighten tau (no candidates); 1: append pairs with d2 <= tau.
template <typename T>
void launch_dist_leaf(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                      const unsigned long long *surv, const unsigned *surv_lb, unsigned long long nsurv,
                      unsigned long long surv_cap, bool sorted, int k, int collect, DistCand<T> *cand,
                      unsigned long long cand_cap, ScreenStats *stats, bool screen, float e, cudaStream_t st,
                      const Batch &bt = Batch{});
// Supertile level of the distance screen: bounds of 8 x 8 tiles, threshold
// seed and cull over supertile pairs, expansion of the surviving supertile
// pairs into tile pairs (threshold pass, then cull with the bound keys).
template <typename T>
void launch_supertiles(const SideRound<T> &sr, cudaStream_t st, const Batch &bt = Batch{});
template <typename T>
void launch_dist_tau_st(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                        int k, ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt = Batch{});
template <typename T>
void launch_dist_cull_st(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                         unsigned long long *surv, unsigned long long cap, ScreenStats *stats, bool screen, float e,
                         cudaStream_t st, const Batch &bt = Batch{});
template <typename T>
void launch_dist_expand(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                        const unsigned long long *st_surv, unsigned long long nst_surv, unsigned long long st_cap,
                        int k, int cull, unsigned long long *surv, unsigned *surv_lb, unsigned long long cap,
                        ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt = Batch{});
// Exact k-th d2 (k <= 8) of each of the first nhead tile pairs, folded into tau.
template <typename T>
void launch_dist_head(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                      const unsigned long long *surv, unsigned long long nhead, unsigned long long head_cap, int k,
                      ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt = Batch{});
// FP32-screen form: FP32 samples from FP64 basis tables; FP64 re-check.
void launch_samples_screen(const SurfView<float> &s, const SideRound<double> &basis_side, const SideRound<float> &out,
                           cudaStream_t st, const Batch &bt = Batch{}, const SurfView<float> *vdev = nullptr);
// Resident surface layout from raw float records staged on the device: the
// record copied into its block, FP64 knots, FP32/FP64 (x, y, z, w) nets.
struct SurfacePrep {
  const float *src;  // staged record
  float *raw;        // the record in the surface's block
  double *U64, *V64;
  Vec4<float> *cpw32;
  Vec4<double> *cpw64;
  long long ndata, ncp;
  int nku, nkv, rat, pad_;
};
// jobs: device array of n entries; most = the largest max(ndata, ncp).
void launch_surface_prep(const SurfacePrep *jobs, int n, long long most, cudaStream_t st);
// Distance cells straight from the basis tables (no sample grid in HBM):
// centres and tile ranges of out, bit-identical to launch_samples(_screen) +
// launch_cells.  TB = basis precision, TC = cell precision.
// mixed: the queries of the batch differ in degree or rational flag (s then
// only carries the largest degrees): the kernel that reads every query's
// degree and flag from vdev is used.
template <typename TB, typename TC>
void launch_cells_fused(const SurfView<TC> &s, const SideRound<TB> &bs, const SideRound<TC> &out, cudaStream_t st,
                        const Batch &bt = Batch{}, const SurfView<TC> *vdev = nullptr, bool mixed = false);
// stats set: the candidate count is read on the device (capped at cap).
void launch_dist_verify(const SurfView<double> &sa, const SurfView<double> &sb, const SideRound<double> &a,
                        const SideRound<double> &b, const int *map1, const int *map2, const DistCand<float> *cand,
                        long long n, DistCand<double> *out, cudaStream_t st, const Batch &bt = Batch{},
                        const SurfView<double> *va = nullptr, const SurfView<double> *vb = nullptr,
                        const ScreenStats *stats = nullptr, unsigned long long cap = 0);
template <typename T>
void launch_dist_select(const DistCand<T> *cand, unsigned long long cand_cap, int k, DistCand<T> *out,
                        ScreenStats *stats, cudaStream_t st, const Batch &bt = Batch{});
template <typename T>
void launch_dist_next(const DistCand<T> *top, ScreenStats *stats, const SideRound<T> &a, const SideRound<T> &b,
                      const int *map1, const int *map2, int nuv_next, RegionRec<T> *next1, RegionRec<T> *next2,
                      int *nmap1, int *nmap2, cudaStream_t st, const Batch &bt = Batch{});
// Batched rounds: record a round and restart the counters; choose the
// threshold-pass list (at most head_cap tile pairs, about `want` with the
// smallest bounds when more survive).
template <typename TP>
void launch_dist_close(ScreenStats *stats, const DistCand<TP> *top, DistRecord<TP> *rec, int round,
                       unsigned long long surv_cap, unsigned long long cand_cap, bool last, cudaStream_t st,
                       const Batch &bt);

// The refinement rounds of a batched distance query in one launch (one block
// of kRefineThreads per query, every round of the query inside it): the
// round's regions evaluated into shared memory (basis, samples, cell centres
// and tile ranges, the same operations as k_basis + k_cells_fused), the
// exact k smallest (d2, slot, i, j) over the slots' cell pairs with tile
// pairs pruned by their box gap against the k-th of the closest tile pairs,
// the next round's regions with (slot, cell) dedup (k_dist_next) and the
// round's record (k_dist_close).  Needs nuv <= kRefineNuv and k <= kBatchK.
constexpr int kRefineNuv = 16;
constexpr int kRefineThreads = 256;
template <typename T>
struct RefineRound {
  const RegionRec<T> *reg1, *reg2;  // this round's regions (side A / B)
  const int *map1, *map2;           // slot -> region
  DistCand<T> *top;                 // the round's kept pairs
  RegionRec<T> *next1, *next2;      // the next round's regions (null in the last round)
  int *nmap1, *nmap2;
  Vec4<T> *cen1, *cen2;             // the round's cell centres, (nuv - 1)^2 per region
};
template <typename T>
struct RefineArgs {
  RefineRound<T> r[kBatchRounds];  // indexed by round - 1
  int first, last;                 // rounds first..last (1-based, first >= 2)
  int nuv, k;
};
template <typename T>
void launch_dist_refine(const SurfView<T> &sa, const SurfView<T> &sb, const SurfView<T> *va, const SurfView<T> *vb,
                        ScreenStats *stats, DistRecord<T> *rec, const RefineArgs<T> &args, cudaStream_t st,
                        const Batch &bt);
void launch_dist_pick(const unsigned long long *surv, const unsigned *surv_lb, unsigned long long surv_cap,
                      unsigned long long *head, unsigned long long head_cap, unsigned want, ScreenStats *stats,
                      cudaStream_t st, const Batch &bt);

template <typename T>
void launch_inter_cull(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                       unsigned long long *surv, unsigned long long surv_cap, ScreenStats *stats, cudaStream_t st);
template <typename T>
void launch_inter_leaf(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                       const unsigned long long *surv, unsigned long long nsurv, int ij_bits,
                       unsigned long long *keys, unsigned long long key_cap, ScreenStats *stats, cudaStream_t st);
// FP32 screen of the intersection query (one round): FP32 samples (and, with
// need_k, curvature terms with rigorous bounds: khi per sample, klo per
// region) from the FP64 basis tables; exact FP64 curvature maxima from the
// samples whose bound reaches the maximum (into bs.kmax, count += samples
// re-evaluated); overlap screen widened per axis by w plus both regions' FP64
// paddings; FP64 re-check of the candidate keys into out (stats->checked),
// from the round's FP64 cells.
void launch_iscreen_samples(const SurfView<float> &s, const SideRound<double> &bs, const SideRound<float> &out,
                            bool need_k, Vec4<float> *khi, unsigned *klo, double g, const double cmax[3],
                            const double wcmax[3], double wmax, cudaStream_t st);
void launch_kmax_recheck(const SurfView<double> &s, const SideRound<double> &bs, const Vec4<float> *khi,
                         const unsigned *klo, unsigned long long *count, cudaStream_t st);
void launch_inter_cull_screen(const SideRound<float> &a, const SideRound<float> &b, const int *map1, const int *map2,
                              int nslots, unsigned long long *surv, unsigned long long surv_cap, ScreenStats *stats,
                              const float w[3], const double *pad64a, const double *pad64b, cudaStream_t st);
void launch_inter_leaf_screen(const SideRound<float> &a, const SideRound<float> &b, const int *map1, const int *map2,
                              const unsigned long long *surv, unsigned long long nsurv, int ij_bits,
                              unsigned long long *keys, unsigned long long key_cap, ScreenStats *stats,
                              const float w[3], const double *pad64a, const double *pad64b, cudaStream_t st);
// The same re-check from the FP64 cells of the round (a.center / a.half, with
// a.pad): a lookup per candidate instead of eight point evaluations.
void launch_inter_verify_cells(const SideRound<double> &a, const SideRound<double> &b, const int *map1,
                               const int *map2, const unsigned long long *keys, unsigned long long n, int ij_bits,
                               unsigned long long *out, unsigned long long cap, ScreenStats *stats, cudaStream_t st);
// Dedup of the next round's regions from sorted (slot, i, j) keys.
void launch_inter_prep(const unsigned long long *keys, long long n, int ij_bits, unsigned long long *key2, int *idx,
                       unsigned *flag1, cudaStream_t st);
void launch_flag_runs(const unsigned long long *sorted, long long n, unsigned *flags, cudaStream_t st);
template <typename T>
void launch_inter_side1(const unsigned long long *keys, long long n, int ij_bits, const unsigned *flag1,
                        const unsigned *ex1, const SideRound<T> &cur, const int *map1, RegionRec<T> *next,
                        int *nmap1, cudaStream_t st, bool cover = false);
template <typename T>
void launch_inter_side2(const unsigned long long *key2s, const int *idxs, long long n, int ij_bits,
                        const unsigned *flag2, const unsigned *ex2, const SideRound<T> &cur, const int *map2,
                        RegionRec<T> *next, int *nmap2, cudaStream_t st, bool cover = false);

// Bounds mode (certified distance interval), FP64 sides built on the
// covering grid: rigorous cell padding per region and coordinate, then tile pairs / cell
// pairs whose box gap (rounded down) can be <= ub, ub2 = ub^2 rounded up; the
// leaf appends (slot, i, j) keys like the intersection leaf and folds the
// smallest kept squared gap into stats->lb_bits.
// Unit tangents and source-cell scales (tx, ty, tz, ok, scale) of the
// intersection curve at refined points (8 doubles each: x, y, z, u, v, s, t,
// residual, in the order of the final round's pair keys).
void launch_curve_tangents(const SurfView<double> &sa, const SurfView<double> &sb, const RegionRec<double> *reg1,
                           const RegionRec<double> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                           const unsigned long long *keys, int ij_bits, const double *pts, long long n, double *out,
                           cudaStream_t st);
// sr.pad must hold 4 doubles per region (a Vec4 pad per region, x, y, z).
// Per-region pads of the bounds mode from a per-knot-span table of
// curvature bounds (two Vec4 per span: m2u, m2v).
void launch_pad_bound(const SideRound<double> &sr, const SurfView<double> &v, const Vec4<double> *tab, double eps,
                      cudaStream_t st);
void launch_bound_cull(const SideRound<double> &a, const SideRound<double> &b, const int *map1, const int *map2,
                       int nslots, double ub2, unsigned long long *surv, unsigned long long surv_cap,
                       ScreenStats *stats, cudaStream_t st);
void launch_bound_leaf(const SideRound<double> &a, const SideRound<double> &b, const int *map1, const int *map2,
                       const unsigned long long *surv, unsigned long long nsurv, int ij_bits, double ub2,
                       unsigned long long *keys, unsigned long long key_cap, ScreenStats *stats, cudaStream_t st);

// FP64 Newton refinement.  dom = {u0, u1, v0, v1, s0, s1, t0, t1} (the query
// rectangles).  Distance: 11 doubles per candidate (d, u, v, s, t, P1, P2);
// intersection: 8 doubles per pair (x, y, z, u, v, s, t, residual).
// stats set: the candidate count is the device slot count of the last round.
template <typename TP>
void launch_newton_dist(const SurfView<double> &sa, const SurfView<double> &sb, const RegionRec<TP> *reg1,
                        const RegionRec<TP> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                        const DistCand<TP> *top, int n, const double *dom, double *out, cudaStream_t st,
                        const Batch &bt = Batch{}, const SurfView<double> *va = nullptr,
                        const SurfView<double> *vb = nullptr, const ScreenStats *stats = nullptr);
template <typename TP>
void launch_newton_inter(const SurfView<double> &sa, const SurfView<double> &sb, const RegionRec<TP> *reg1,
                         const RegionRec<TP> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                         const unsigned long long *keys, long long n, int ij_bits, const double *dom, double *out,
                         cudaStream_t st);

}  // namespace jsi
