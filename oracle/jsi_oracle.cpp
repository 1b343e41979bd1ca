// CPU oracle: a restatement of the reference VERSION5 query path.
//
// TEST INFRASTRUCTURE ONLY (see jsi_oracle.h).  Every routine names the
// reference lines it follows; paths are relative to JSI_CAD_NEXT_VERSION5/.
// Compiled with -ffp-contract=off so that each written product and sum is
// rounded on its own, as the reference's x86-64 build does.
#include "jsi_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <unordered_map>
#include <vector>

namespace {

constexpr int kMaxDeg = 25;  // src/evaluation/evaluation.cu:13

template <typename T>
struct Surface {
  int flags = 0, degu = 0, degv = 0, ncpu = 0, ncpv = 0, nku = 0, nkv = 0;
  bool flat = false, rat = false;
  int du = 0, dv = 0;
  std::vector<T> U, V, CP, W;
};

// EGADS header decode, src/evaluation/evaluation.cu:239-257.
template <typename T>
Surface<T> load_surface(const int *ivec, const float *data) {
  Surface<T> s;
  s.flags = ivec[0];
  s.flat = (ivec[0] & 1) != 0;
  s.rat = (ivec[0] & 2) != 0;
  s.degu = ivec[1];
  s.ncpu = ivec[2];
  s.nku = ivec[3];
  s.degv = ivec[4];
  s.ncpv = ivec[5];
  s.nkv = ivec[6];
  s.du = std::min(2, s.degu);
  s.dv = std::min(2, s.degv);
  s.U.assign(data, data + s.nku);
  s.V.assign(data + s.nku, data + s.nku + s.nkv);
  const float *cp = data + s.nku + s.nkv;
  const size_t ncp = static_cast<size_t>(s.ncpu) * s.ncpv;
  s.CP.assign(cp, cp + 3 * ncp);
  if (s.rat) s.W.assign(cp + 3 * ncp, cp + 4 * ncp);
  return s;
}

// Knot-span binary search, src/evaluation/evaluation.cu:152-166.
template <typename T>
int find_span(int nk, int p, T u, const T *knots) {
  if (u <= knots[p]) return p;
  const int n = nk - p - 1;
  if (u >= knots[n]) return n - 1;
  int lo = p, hi = n;
  int mid = (lo + hi) / 2;
  while (u < knots[mid] || u >= knots[mid + 1]) {
    if (u < knots[mid])
      hi = mid;
    else
      lo = mid;
    mid = (lo + hi) / 2;
  }
  return mid;
}

// Non-zero basis functions and their derivatives up to order nd, the
// published algorithm A2.3 of Piegl & Tiller, "The NURBS Book", as used by
// src/evaluation/evaluation.cu:168-219.  ders[k][j] = k-th derivative of
// N_{span-p+j, p}.
template <typename T>
void basis_ders(int span, int p, T u, const T *knots, int nd, T ders[3][kMaxDeg + 1]) {
  T ndu[kMaxDeg + 1][kMaxDeg + 1];
  T left[kMaxDeg + 1], right[kMaxDeg + 1];
  T a[2][kMaxDeg + 1];
  ndu[0][0] = T(1);
  for (int j = 1; j <= p; ++j) {
    left[j] = u - knots[span + 1 - j];
    right[j] = knots[span + j] - u;
    T saved = T(0);
    for (int r = 0; r < j; ++r) {
      ndu[j][r] = right[r + 1] + left[j - r];
      const T tmp = ndu[r][j - 1] / ndu[j][r];
      ndu[r][j] = saved + right[r + 1] * tmp;
      saved = left[j - r] * tmp;
    }
    ndu[j][j] = saved;
  }
  for (int j = 0; j <= p; ++j) ders[0][j] = ndu[j][p];
  for (int r = 0; r <= p; ++r) {
    int s1 = 0, s2 = 1;
    a[0][0] = T(1);
    for (int k = 1; k <= nd; ++k) {
      T d = T(0);
      const int rk = r - k, pk = p - k;
      if (r >= k) {
        a[s2][0] = a[s1][0] / ndu[pk + 1][rk];
        d = a[s2][0] * ndu[rk][pk];
      }
      const int j1 = (rk >= -1) ? 1 : -rk;
      const int j2 = (r - 1 <= pk) ? k - 1 : p - r;
      for (int j = j1; j <= j2; ++j) {
        a[s2][j] = (a[s1][j] - a[s1][j - 1]) / ndu[pk + 1][rk + j];
        d += a[s2][j] * ndu[rk + j][pk];
      }
      if (r <= pk) {
        a[s2][k] = -a[s1][k - 1] / ndu[pk + 1][r];
        d += a[s2][k] * ndu[r][pk];
      }
      ders[k][r] = d;
      std::swap(s1, s2);
    }
  }
  int fac = p;
  for (int k = 1; k <= nd; ++k) {
    for (int j = 0; j <= p; ++j) ders[k][j] *= static_cast<T>(fac);
    fac *= p - k;
  }
}

// Homogeneous -> Euclidean derivatives up to order 2 for a 4-wide record
// stride (x, y, z, w), the der_count = 2, dim = 3, stride = 4 case of
// src/evaluation/evaluation.cu:77-130.  Record order in h: 0 P, 1 Pu, 2 Pv,
// 3 Puu, 4 Puv, 5 Pvv (4 values each).
template <typename T>
void quotient_rule2(T h[24]) {
  const T inv = T(1) / h[3];
  for (int q = 0; q < 24; ++q) h[q] *= inv;
  const T ws = -h[7], wt = -h[11];
  for (int c = 0; c < 3; ++c) {
    h[4 + c] += ws * h[c];
    h[8 + c] += wt * h[c];
  }
  const T wss = -h[15], wst = -h[19], wtt = -h[23];
  for (int c = 0; c < 3; ++c) {
    const T F = h[c], Fs = h[4 + c], Ft = h[8 + c];
    h[12 + c] += wss * F + T(2) * ws * Fs;
    h[16 + c] += wst * F + wt * Fs + ws * Ft;
    h[20 + c] += wtt * F + T(2) * wt * Ft;
  }
}

// One parameter point, src/evaluation/evaluation.cu:259-356.  out = 18
// values P, Pu, Pv, Puu, Puv, Pvv.  The contraction runs, for each derivative
// pair (k in u, l in v), a u-direction sum over the p+1 columns for every one
// of the q+1 rows, then a v-direction sum over the rows, in that order.
template <typename T>
void eval_point(const Surface<T> &s, T u, T v, T out[18]) {
  for (int q = 0; q < 18; ++q) out[q] = T(0);
  if (!s.flat && (s.flags & 12) != 0) return;
  if (s.degu >= kMaxDeg || s.degv >= kMaxDeg) return;
  T Nu[3][kMaxDeg + 1], Nv[3][kMaxDeg + 1];
  const int spanu = find_span(s.nku, s.degu, u, s.U.data());
  basis_ders(spanu, s.degu, u, s.U.data(), s.du, Nu);
  const int spanv = find_span(s.nkv, s.degv, v, s.V.data());
  basis_ders(spanv, s.degv, v, s.V.data(), s.dv, Nv);
  const int cu0 = spanu - s.degu, cv0 = spanv - s.degv;

  // (l, k) enumeration order of the reference: m = 0:(0,0) 1:(0,1) 2:(0,2)
  // 3:(1,0) 4:(1,1) 5:(2,0) with k the u order; the record order swaps m=2
  // and m=3 at the end.
  const int ku[6] = {0, 1, 2, 0, 1, 0};
  const int lv[6] = {0, 0, 0, 1, 1, 2};
  const int slot_of_m[6] = {0, 1, 3, 2, 4, 5};
  if (!s.rat) {
    for (int m = 0; m < 6; ++m) {
      const int k = ku[m], l = lv[m];
      if (l > s.dv || k > s.du) continue;
      T acc[3] = {T(0), T(0), T(0)};
      for (int r = 0; r <= s.degv; ++r) {
        T row[3] = {T(0), T(0), T(0)};
        const size_t base = static_cast<size_t>(s.ncpu) * (cv0 + r);
        for (int c = 0; c <= s.degu; ++c) {
          const size_t idx = base + cu0 + c;
          row[0] += Nu[k][c] * s.CP[3 * idx];
          row[1] += Nu[k][c] * s.CP[3 * idx + 1];
          row[2] += Nu[k][c] * s.CP[3 * idx + 2];
        }
        acc[0] += Nv[l][r] * row[0];
        acc[1] += Nv[l][r] * row[1];
        acc[2] += Nv[l][r] * row[2];
      }
      const int o = 3 * slot_of_m[m];
      out[o] = acc[0];
      out[o + 1] = acc[1];
      out[o + 2] = acc[2];
    }
    return;
  }
  T h[24];
  for (int q = 0; q < 24; ++q) h[q] = T(0);
  for (int m = 0; m < 6; ++m) {
    const int k = ku[m], l = lv[m];
    if (l > s.dv || k > s.du) continue;
    T acc[4] = {T(0), T(0), T(0), T(0)};
    for (int r = 0; r <= s.degv; ++r) {
      T row[4] = {T(0), T(0), T(0), T(0)};
      const size_t base = static_cast<size_t>(s.ncpu) * (cv0 + r);
      for (int c = 0; c <= s.degu; ++c) {
        const size_t idx = base + cu0 + c;
        const T nw = Nu[k][c] * s.W[idx];
        row[0] += nw * s.CP[3 * idx];
        row[1] += nw * s.CP[3 * idx + 1];
        row[2] += nw * s.CP[3 * idx + 2];
        row[3] += nw;
      }
      for (int c = 0; c < 4; ++c) acc[c] += Nv[l][r] * row[c];
    }
    const int o = 4 * slot_of_m[m];
    for (int c = 0; c < 4; ++c) h[o + c] = acc[c];
  }
  quotient_rule2(h);
  for (int m = 0; m < 6; ++m)
    for (int c = 0; c < 3; ++c) out[3 * m + c] = h[4 * m + c];
}

// Grid driver, src/evaluation/evaluation.cu:358-369.
template <typename T>
void eval_grid(const Surface<T> &s, T ustep, T vstep, T ustart, T vstart, int nuv, T *out) {
  for (int idy = 0; idy < nuv; ++idy)
    for (int idx = 0; idx < nuv; ++idx)
      eval_point(s, ustep * static_cast<T>(idx) + ustart, vstep * static_cast<T>(idy) + vstart,
                 out + static_cast<size_t>(idx + idy * nuv) * 18);
}

template <typename T>
T lowest();
template <>
float lowest<float>() { return -FLT_MAX; }
template <>
double lowest<double>() { return -DBL_MAX; }

// Curvature constant, src/common/common.cu:149-172.
template <typename T>
T compute_k(const T *rec, int n) {
  T muu = lowest<T>(), muv = lowest<T>(), mvv = lowest<T>();
  const size_t cnt = static_cast<size_t>(n) * n;
  for (size_t q = 0; q < cnt; ++q) {
    const T *r = rec + q * 18;
    const T uu = std::max(std::fabs(r[9]), std::max(std::fabs(r[10]), std::fabs(r[11])));
    const T uv = std::max(std::fabs(r[12]), std::max(std::fabs(r[13]), std::fabs(r[14])));
    const T vv = std::max(std::fabs(r[15]), std::max(std::fabs(r[16]), std::fabs(r[17])));
    muu = std::max(muu, uu);
    muv = std::max(muv, uv);
    mvv = std::max(mvv, vv);
  }
  const int side = n > 1 ? n - 1 : 1;
  const T ss = static_cast<T>(side * side);
  return (muu / ss + T(2) * muv / ss + mvv / ss) / T(8);
}

struct Rect {
  double u0, v0, u1, v1;
};

template <typename T>
struct Region {
  T u0, v0, u1, v1;
  int nuv;
  int side;
  std::vector<T> center;  // 3 per cell
  std::vector<T> radius;  // 3 per cell (intersection only)
};

// Per-cell boxes from the four corner samples: distance flavour
// src/distance_analysis/distance_analysis.cu:45-86 (k = 0) and intersection
// flavour src/intersection/intersection.cu:106-148 (radius += padding).
template <typename T>
void build_cells(const T *rec, int nuv, bool with_radius, T padding, std::vector<T> &center, std::vector<T> &radius) {
  const int w = nuv - 1;
  const size_t ncell = static_cast<size_t>(w) * w;
  center.assign(3 * ncell, T(0));
  if (with_radius) radius.assign(3 * ncell, T(0));
  for (int iv = 0; iv < w; ++iv) {
    for (int iu = 0; iu < w; ++iu) {
      const size_t id = static_cast<size_t>(iv) * w + iu;
      const size_t p0 = static_cast<size_t>(iv) * nuv + iu, p1 = p0 + 1, p2 = p0 + nuv, p3 = p2 + 1;
      for (int c = 0; c < 3; ++c) {
        const T a = rec[p0 * 18 + c], b = rec[p1 * 18 + c], e = rec[p2 * 18 + c], f = rec[p3 * 18 + c];
        const T lo = std::min(a, std::min(b, std::min(e, f)));
        const T hi = std::max(a, std::max(b, std::max(e, f)));
        if (with_radius) {
          center[3 * id + c] = (lo + hi) / T(2);
          radius[3 * id + c] = (hi - lo) / T(2) + padding;
        } else {
          // (lo - k + hi + k) / 2 with k = 0.
          center[3 * id + c] = (lo - T(0) + hi + T(0)) / T(2);
        }
      }
    }
  }
}

// Span bookkeeping of the intersection query (intersection.cu:344-347) and
// the padding rule (intersection.cu:187-205).
template <typename T>
struct Spans {
  T u[3] = {T(1), T(1), T(1)};
  T v[3] = {T(1), T(1), T(1)};
};

template <typename T>
T tiny_span();
template <>
float tiny_span<float>() { return 1.0e-12f; }
template <>
double tiny_span<double>() { return 1.0e-12; }

// Evaluate one region and build its cells: src/distance_analysis/distance_analysis.cu:88-116
// (distance, no padding) and src/intersection/intersection.cu:175-219 (intersection).
template <typename T>
void run_region(const Surface<T> &s, Region<T> &reg, bool intersect, bool use_k, const Spans<T> &spans,
                T *pad_out = nullptr) {
  const int nuv = reg.nuv;
  const T ustep = (reg.u1 - reg.u0) / static_cast<T>(nuv);
  const T vstep = (reg.v1 - reg.v0) / static_cast<T>(nuv);
  std::vector<T> rec(static_cast<size_t>(nuv) * nuv * 18);
  eval_grid(s, ustep, vstep, reg.u0, reg.v0, nuv, rec.data());
  T pad = T(0);
  if (intersect && use_k) {
    const T raw = compute_k(rec.data(), nuv);
    const int side = (reg.side == 2) ? 2 : 1;
    const T us = std::fabs(reg.u1 - reg.u0) / spans.u[side];
    const T vs = std::fabs(reg.v1 - reg.v0) / spans.v[side];
    const T ps = std::max(us, vs);
    pad = raw * ps * ps;
    if (!std::isfinite(pad) || pad < T(0)) pad = T(0);
  }
  if (pad_out) *pad_out = pad;
  build_cells(rec.data(), nuv, intersect, pad, reg.center, reg.radius);
}

// Child region of cell bbox: make_dist_refine_task (distance_analysis.cu:340-354)
// and make_intersect_refine_task (intersection.cu:311-325), same arithmetic.
template <typename T>
Region<T> child_region(const Region<T> &parent, int bbox, int side, int nuv) {
  const T ustep = (parent.u1 - parent.u0) / static_cast<T>(parent.nuv);
  const T vstep = (parent.v1 - parent.v0) / static_cast<T>(parent.nuv);
  const int w = parent.nuv - 1;
  const int x = bbox % w, y = bbox / w;
  Region<T> r;
  r.side = side;
  r.nuv = nuv;
  r.u0 = parent.u0 + ustep * static_cast<T>(x);
  r.u1 = r.u0 + ustep;
  r.v0 = parent.v0 + vstep * static_cast<T>(y);
  r.v1 = r.v0 + vstep;
  return r;
}

struct PairRef {
  int slot, i, j;
};

template <typename T>
struct DistPair {
  T d2;
  int slot, i, j;
};

// Total order of the distance top-k: distance_analysis.cu:226-231.
template <typename T>
bool dist_less(const DistPair<T> &a, const DistPair<T> &b) {
  if (a.d2 != b.d2) return a.d2 < b.d2;
  if (a.slot != b.slot) return a.slot < b.slot;
  if (a.i != b.i) return a.i < b.i;
  return a.j < b.j;
}

// Squared centre distance: distance_analysis.cu:202-207.
template <typename T>
inline T center_d2(const T *c1, const T *c2) {
  const T dx = c1[0] - c2[0];
  const T dy = c1[1] - c2[1];
  const T dz = c1[2] - c2[2];
  return dx * dx + dy * dy + dz * dz;
}

// Strict per-axis overlap: intersection.cu:46-63.
template <typename T>
inline bool boxes_overlap(const T *c1, const T *r1, const T *c2, const T *r2) {
  return std::fabs(c1[0] - c2[0]) < (r1[0] + r2[0]) && std::fabs(c1[1] - c2[1]) < (r1[1] + r2[1]) &&
         std::fabs(c1[2] - c2[2]) < (r1[2] + r2[2]);
}

// Global k smallest over all slot-local cell pairs (dist_collect_top_pairs,
// distance_analysis.cu:246-338), kept in a max-heap under the total order.
template <typename T>
std::vector<DistPair<T>> dist_top_pairs(const std::vector<const Region<T> *> &s1,
                                        const std::vector<const Region<T> *> &s2, int k) {
  const int limit = std::max(1, k);
  std::vector<DistPair<T>> heap;
  heap.reserve(limit + 1);
  auto cmp = [](const DistPair<T> &a, const DistPair<T> &b) { return dist_less(a, b); };
  for (size_t slot = 0; slot < s1.size(); ++slot) {
    const Region<T> &a = *s1[slot];
    const Region<T> &b = *s2[slot];
    const int n1 = static_cast<int>(a.center.size() / 3), n2 = static_cast<int>(b.center.size() / 3);
    for (int i = 0; i < n1; ++i) {
      for (int j = 0; j < n2; ++j) {
        DistPair<T> p{center_d2(&a.center[3 * i], &b.center[3 * j]), static_cast<int>(slot), i, j};
        if (static_cast<int>(heap.size()) < limit) {
          heap.push_back(p);
          std::push_heap(heap.begin(), heap.end(), cmp);
        } else if (dist_less(p, heap.front())) {
          std::pop_heap(heap.begin(), heap.end(), cmp);
          heap.back() = p;
          std::push_heap(heap.begin(), heap.end(), cmp);
        }
      }
    }
  }
  std::sort(heap.begin(), heap.end(), cmp);
  return heap;
}

template <typename T>
Region<T> root_region(const T *rect, int nuv, int side) {
  Region<T> r;
  r.u0 = rect[0];
  r.v0 = rect[1];
  r.u1 = rect[2];
  r.v1 = rect[3];
  r.nuv = nuv;
  r.side = side;
  return r;
}

// minimum_distance round loop, distance_analysis.cu:356-506, with pair
// preservation (JSI_CAD_PRESERVE_PAIR_RELATION=1) and duplicate-region reuse
// keyed by (slot, cell) per side (:426-465).
// Start parameters (u, v, s, t) of a final pair for the Newton refinement:
// the centres of its two cells, in double.
template <typename T>
void cell_start(const Region<T> &r1, int i, const Region<T> &r2, int j, double *x) {
  const int w1 = r1.nuv - 1, w2 = r2.nuv - 1;
  const double du1 = (double(r1.u1) - double(r1.u0)) / r1.nuv, dv1 = (double(r1.v1) - double(r1.v0)) / r1.nuv;
  const double du2 = (double(r2.u1) - double(r2.u0)) / r2.nuv, dv2 = (double(r2.v1) - double(r2.v0)) / r2.nuv;
  x[0] = double(r1.u0) + du1 * ((i % w1) + 0.5);
  x[1] = double(r1.v0) + dv1 * ((i / w1) + 0.5);
  x[2] = double(r2.u0) + du2 * ((j % w2) + 0.5);
  x[3] = double(r2.v0) + dv2 * ((j / w2) + 0.5);
}

template <typename T>
int dist_query(const int *ivec1, const float *data1, const T *rect1, const int *ivec2, const float *data2,
               const T *rect2, int nuv0, int nuv_refine, int k, int rounds, T *kth_d2, int *npairs, int *pairs_out,
               double *starts) {
  const Surface<T> sa = load_surface<T>(ivec1, data1);
  const Surface<T> sb = load_surface<T>(ivec2, data2);
  Spans<T> spans;
  std::vector<Region<T>> store1, store2;
  store1.push_back(root_region(rect1, nuv0, 1));
  store2.push_back(root_region(rect2, nuv0, 2));
  run_region(sa, store1[0], false, false, spans);
  run_region(sb, store2[0], false, false, spans);
  std::vector<const Region<T> *> ch1{&store1[0]}, ch2{&store2[0]};
  int nuv = nuv_refine;
  int round = 0;
  const int limit = std::max(1, k);
  for (int r = 0; r < rounds; ++r) {
    kth_d2[r] = T(0);
    npairs[r] = 0;
  }
  while (true) {
    ++round;
    auto best = dist_top_pairs(ch1, ch2, k);
    kth_d2[round - 1] = best.empty() ? T(0) : best.back().d2;
    npairs[round - 1] = static_cast<int>(best.size());
    for (size_t q = 0; q < best.size() && static_cast<int>(q) < limit; ++q) {
      pairs_out[(static_cast<size_t>(round - 1) * limit + q) * 3 + 0] = best[q].slot;
      pairs_out[(static_cast<size_t>(round - 1) * limit + q) * 3 + 1] = best[q].i;
      pairs_out[(static_cast<size_t>(round - 1) * limit + q) * 3 + 2] = best[q].j;
    }
    if (best.empty() || round == rounds) {
      if (starts)
        for (size_t q = 0; q < best.size(); ++q)
          cell_start(*ch1[best[q].slot], best[q].i, *ch2[best[q].slot], best[q].j, starts + 4 * q);
      break;
    }
    std::vector<Region<T>> next1, next2;
    std::unordered_map<uint64_t, size_t> idx1, idx2;
    std::vector<size_t> slot1, slot2;
    for (const auto &p : best) {
      const uint64_t key1 = (static_cast<uint64_t>(static_cast<uint32_t>(p.slot)) << 32) | static_cast<uint32_t>(p.i);
      const uint64_t key2 = (static_cast<uint64_t>(static_cast<uint32_t>(p.slot)) << 32) | static_cast<uint32_t>(p.j);
      auto it1 = idx1.emplace(key1, next1.size());
      if (it1.second) next1.push_back(child_region(*ch1[p.slot], p.i, 1, nuv));
      auto it2 = idx2.emplace(key2, next2.size());
      if (it2.second) next2.push_back(child_region(*ch2[p.slot], p.j, 2, nuv));
      slot1.push_back(it1.first->second);
      slot2.push_back(it2.first->second);
    }
    for (auto &reg : next1) run_region(sa, reg, false, false, spans);
    for (auto &reg : next2) run_region(sb, reg, false, false, spans);
    store1.swap(next1);
    store2.swap(next2);
    ch1.clear();
    ch2.clear();
    for (size_t q = 0; q < slot1.size(); ++q) {
      ch1.push_back(&store1[slot1[q]]);
      ch2.push_back(&store2[slot2[q]]);
    }
  }
  return round;
}

// intersection round loop, intersection.cu:338-475 (pair preservation,
// (slot, cell) dedup per side, nuv halving rule at :368-370).
template <typename T>
int inter_query(const int *ivec1, const float *data1, const T *rect1, const int *ivec2, const float *data2,
                const T *rect2, int nuv0, int nuv_refine, int use_k, int rounds, int halve_threshold, int min_nuv,
                long long max_pairs, long long *counts, int *pairs_out, long long pair_cap, long long *pairs_written,
                T *pads, double *starts, long long starts_cap) {
  const Surface<T> sa = load_surface<T>(ivec1, data1);
  const Surface<T> sb = load_surface<T>(ivec2, data2);
  Spans<T> spans;
  spans.u[1] = std::max(std::fabs(rect1[2] - rect1[0]), tiny_span<T>());
  spans.v[1] = std::max(std::fabs(rect1[3] - rect1[1]), tiny_span<T>());
  spans.u[2] = std::max(std::fabs(rect2[2] - rect2[0]), tiny_span<T>());
  spans.v[2] = std::max(std::fabs(rect2[3] - rect2[1]), tiny_span<T>());
  std::vector<Region<T>> store1, store2;
  store1.push_back(root_region(rect1, nuv0, 1));
  store2.push_back(root_region(rect2, nuv0, 2));
  T pad1 = T(0), pad2 = T(0);
  run_region(sa, store1[0], true, use_k != 0, spans, &pad1);
  run_region(sb, store2[0], true, use_k != 0, spans, &pad2);
  if (pads) {
    pads[0] = pad1;
    pads[1] = pad2;
  }
  std::vector<const Region<T> *> ch1{&store1[0]}, ch2{&store2[0]};
  int nuv = nuv_refine;
  int round = 0;
  long long written = 0;
  for (int r = 0; r < rounds; ++r) counts[r] = 0;
  while (true) {
    ++round;
    std::vector<PairRef> pairs;
    for (size_t slot = 0; slot < ch1.size(); ++slot) {
      const Region<T> &a = *ch1[slot];
      const Region<T> &b = *ch2[slot];
      const int n1 = static_cast<int>(a.center.size() / 3), n2 = static_cast<int>(b.center.size() / 3);
      for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j)
          if (boxes_overlap(&a.center[3 * i], &a.radius[3 * i], &b.center[3 * j], &b.radius[3 * j]))
            pairs.push_back({static_cast<int>(slot), i, j});
      if (static_cast<long long>(pairs.size()) > max_pairs) {
        if (pairs_written) *pairs_written = written;
        return -1;
      }
    }
    counts[round - 1] = static_cast<long long>(pairs.size());
    for (const auto &p : pairs) {
      if (written < pair_cap) {
        pairs_out[written * 3 + 0] = p.slot;
        pairs_out[written * 3 + 1] = p.i;
        pairs_out[written * 3 + 2] = p.j;
      }
      ++written;
    }
    if (round == rounds || pairs.empty()) {
      if (starts)
        for (size_t q = 0; q < pairs.size() && static_cast<long long>(q) < starts_cap; ++q)
          cell_start(*ch1[pairs[q].slot], pairs[q].i, *ch2[pairs[q].slot], pairs[q].j, starts + 4 * q);
      break;
    }
    if (static_cast<long long>(pairs.size()) > halve_threshold && nuv > min_nuv) nuv /= 2;
    std::vector<Region<T>> next1, next2;
    std::unordered_map<uint64_t, size_t> idx1, idx2;
    std::vector<size_t> slot1, slot2;
    slot1.reserve(pairs.size());
    slot2.reserve(pairs.size());
    for (const auto &p : pairs) {
      const uint64_t key1 = (static_cast<uint64_t>(static_cast<uint32_t>(p.slot)) << 32) | static_cast<uint32_t>(p.i);
      const uint64_t key2 = (static_cast<uint64_t>(static_cast<uint32_t>(p.slot)) << 32) | static_cast<uint32_t>(p.j);
      auto it1 = idx1.emplace(key1, next1.size());
      if (it1.second) next1.push_back(child_region(*ch1[p.slot], p.i, 1, nuv));
      auto it2 = idx2.emplace(key2, next2.size());
      if (it2.second) next2.push_back(child_region(*ch2[p.slot], p.j, 2, nuv));
      slot1.push_back(it1.first->second);
      slot2.push_back(it2.first->second);
    }
    for (auto &reg : next1) run_region(sa, reg, true, use_k != 0, spans);
    for (auto &reg : next2) run_region(sb, reg, true, use_k != 0, spans);
    store1.swap(next1);
    store2.swap(next2);
    ch1.clear();
    ch2.clear();
    for (size_t q = 0; q < slot1.size(); ++q) {
      ch1.push_back(&store1[slot1[q]]);
      ch2.push_back(&store2[slot2[q]]);
    }
  }
  if (pairs_written) *pairs_written = written;
  return round;
}

template <typename T>
void region_cells(const int *ivec, const float *data, const T *rect, int nuv, T padding, T *centers, T *radii) {
  const Surface<T> s = load_surface<T>(ivec, data);
  Region<T> reg = root_region(rect, nuv, 1);
  const T ustep = (reg.u1 - reg.u0) / static_cast<T>(nuv);
  const T vstep = (reg.v1 - reg.v0) / static_cast<T>(nuv);
  std::vector<T> rec(static_cast<size_t>(nuv) * nuv * 18);
  eval_grid(s, ustep, vstep, reg.u0, reg.v0, nuv, rec.data());
  std::vector<T> c, r;
  build_cells(rec.data(), nuv, radii != nullptr, padding, c, r);
  if (centers) std::memcpy(centers, c.data(), c.size() * sizeof(T));
  if (radii) std::memcpy(radii, r.data(), r.size() * sizeof(T));
}

// ---------------------------------------------------------------------------
// FP64 Newton refinement (no counterpart in the reference: it stops at cell
// centres).  Levenberg-Marquardt on |S1(u,v) - S2(s,t)|^2 and minimum-norm
// Gauss-Newton on S1 - S2 = 0, both inside the query rectangles.
// ---------------------------------------------------------------------------

void record_at(const Surface<double> &s, double u, double v, double r[18]) { eval_point(s, u, v, r); }

double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

double clamp(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Gaussian elimination with partial pivoting on an n x n system (n <= 4).
bool gauss_solve(double M[4][4], double r[4], int n) {
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int q = c + 1; q < n; ++q)
      if (std::fabs(M[q][c]) > std::fabs(M[piv][c])) piv = q;
    if (!(std::fabs(M[piv][c]) > 0.0)) return false;
    if (piv != c) {
      for (int q = 0; q < n; ++q) std::swap(M[c][q], M[piv][q]);
      std::swap(r[c], r[piv]);
    }
    for (int q = c + 1; q < n; ++q) {
      const double f = M[q][c] / M[c][c];
      for (int w = c; w < n; ++w) M[q][w] -= f * M[c][w];
      r[q] -= f * r[c];
    }
  }
  for (int c = n - 1; c >= 0; --c) {
    double acc = r[c];
    for (int q = c + 1; q < n; ++q) acc -= M[c][q] * r[q];
    r[c] = acc / M[c][c];
  }
  return true;
}

void lm_distance(const Surface<double> &sa, const Surface<double> &sb, const double dom[8], double x[4],
                 double out[11]) {
  double r1[18], r2[18];
  record_at(sa, x[0], x[1], r1);
  record_at(sb, x[2], x[3], r2);
  double D[3] = {r1[0] - r2[0], r1[1] - r2[1], r1[2] - r2[2]};
  double f = dot3(D, D);
  double lam = 1e-6;
  for (int it = 0; it < 60; ++it) {
    // half gradient and half Hessian of f (first and second derivatives of both patches)
    const double g[4] = {dot3(D, r1 + 3), dot3(D, r1 + 6), -dot3(D, r2 + 3), -dot3(D, r2 + 6)};
    double H[4][4];
    H[0][0] = dot3(r1 + 3, r1 + 3) + dot3(D, r1 + 9);
    H[0][1] = dot3(r1 + 3, r1 + 6) + dot3(D, r1 + 12);
    H[1][1] = dot3(r1 + 6, r1 + 6) + dot3(D, r1 + 15);
    H[0][2] = -dot3(r1 + 3, r2 + 3);
    H[0][3] = -dot3(r1 + 3, r2 + 6);
    H[1][2] = -dot3(r1 + 6, r2 + 3);
    H[1][3] = -dot3(r1 + 6, r2 + 6);
    H[2][2] = dot3(r2 + 3, r2 + 3) - dot3(D, r2 + 9);
    H[2][3] = dot3(r2 + 3, r2 + 6) - dot3(D, r2 + 12);
    H[3][3] = dot3(r2 + 6, r2 + 6) - dot3(D, r2 + 15);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < a; ++b) H[a][b] = H[b][a];
    bool moved = false;
    while (lam < 1e16) {
      double M[4][4], step[4];
      for (int a = 0; a < 4; ++a) {
        for (int b = 0; b < 4; ++b) M[a][b] = H[a][b];
        M[a][a] += lam * (std::fabs(H[a][a]) + 1e-30);
        step[a] = -g[a];
      }
      if (!gauss_solve(M, step, 4)) {
        lam *= 10.0;
        continue;
      }
      double y[4];
      for (int a = 0; a < 4; ++a) y[a] = clamp(x[a] + step[a], dom[2 * a], dom[2 * a + 1]);
      double q1[18], q2[18];
      record_at(sa, y[0], y[1], q1);
      record_at(sb, y[2], y[3], q2);
      const double E[3] = {q1[0] - q2[0], q1[1] - q2[1], q1[2] - q2[2]};
      const double fy = dot3(E, E);
      if (fy < f) {
        double dmax = 0.0;
        for (int a = 0; a < 4; ++a) {
          dmax = std::max(dmax, std::fabs(y[a] - x[a]));
          x[a] = y[a];
        }
        std::memcpy(r1, q1, sizeof(r1));
        std::memcpy(r2, q2, sizeof(r2));
        std::memcpy(D, E, sizeof(D));
        f = fy;
        lam = std::max(lam * 0.1, 1e-12);
        moved = dmax > 1e-15;
        break;
      }
      lam *= 10.0;
    }
    if (!moved) break;
  }
  out[0] = std::sqrt(f);
  for (int a = 0; a < 4; ++a) out[1 + a] = x[a];
  for (int c = 0; c < 3; ++c) {
    out[5 + c] = r1[c];
    out[8 + c] = r2[c];
  }
}

void gn_point(const Surface<double> &sa, const Surface<double> &sb, const double dom[8], double x[4],
              double out[8]) {
  double r1[18], r2[18], D[3];
  double prev = INFINITY;
  for (int it = 0; it < 40; ++it) {
    record_at(sa, x[0], x[1], r1);
    record_at(sb, x[2], x[3], r2);
    for (int c = 0; c < 3; ++c) D[c] = r1[c] - r2[c];
    // J = [S1u, S1v, -S2s, -S2t] (3 x 4); step = -J^T (J J^T)^-1 D
    const double J[3][4] = {{r1[3], r1[6], -r2[3], -r2[6]},
                            {r1[4], r1[7], -r2[4], -r2[7]},
                            {r1[5], r1[8], -r2[5], -r2[8]}};
    double M[4][4] = {}, y[4] = {D[0], D[1], D[2], 0.0};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double acc = 0.0;
        for (int q = 0; q < 4; ++q) acc += J[a][q] * J[b][q];
        M[a][b] = acc;
      }
    if (!gauss_solve(M, y, 3)) break;
    double dmax = 0.0;
    for (int q = 0; q < 4; ++q) {
      const double step = -(J[0][q] * y[0] + J[1][q] * y[1] + J[2][q] * y[2]);
      const double nx = clamp(x[q] + step, dom[2 * q], dom[2 * q + 1]);
      dmax = std::max(dmax, std::fabs(nx - x[q]));
      x[q] = nx;
    }
    // converged, or the steps stopped shrinking at rounding level
    if (dmax <= 1e-15 || (dmax <= 1e-12 && dmax > 0.5 * prev)) break;
    prev = dmax;
  }
  record_at(sa, x[0], x[1], r1);
  record_at(sb, x[2], x[3], r2);
  for (int c = 0; c < 3; ++c) {
    D[c] = r1[c] - r2[c];
    out[c] = 0.5 * (r1[c] + r2[c]);
  }
  for (int q = 0; q < 4; ++q) out[3 + q] = x[q];
  out[7] = std::sqrt(dot3(D, D));
}

}  // namespace

extern "C" {

void orc_newton_distance(const int *ivec1, const float *data1, const int *ivec2, const float *data2,
                         const double *dom, const double *x0, double *out) {
  const Surface<double> sa = load_surface<double>(ivec1, data1), sb = load_surface<double>(ivec2, data2);
  double x[4] = {x0[0], x0[1], x0[2], x0[3]};
  lm_distance(sa, sb, dom, x, out);
}

void orc_newton_point(const int *ivec1, const float *data1, const int *ivec2, const float *data2, const double *dom,
                      const double *x0, double *out) {
  const Surface<double> sa = load_surface<double>(ivec1, data1), sb = load_surface<double>(ivec2, data2);
  double x[4] = {x0[0], x0[1], x0[2], x0[3]};
  gn_point(sa, sb, dom, x, out);
}


void orc_eval_grid_f32(const int *ivec, const float *data, float ustep, float vstep, float ustart, float vstart,
                       int nuv, float *out) {
  eval_grid(load_surface<float>(ivec, data), ustep, vstep, ustart, vstart, nuv, out);
}

void orc_eval_grid_f64(const int *ivec, const float *data, double ustep, double vstep, double ustart, double vstart,
                       int nuv, double *out) {
  eval_grid(load_surface<double>(ivec, data), ustep, vstep, ustart, vstart, nuv, out);
}

float orc_compute_k_f32(const float *records, int nuv) { return compute_k(records, nuv); }
double orc_compute_k_f64(const double *records, int nuv) { return compute_k(records, nuv); }

int orc_dist_query_f32(const int *ivec1, const float *data1, const float *rect1, const int *ivec2,
                       const float *data2, const float *rect2, int nuv0, int nuv_refine, int k, int rounds,
                       float *kth_d2, int *npairs, int *pairs, double *starts) {
  return dist_query<float>(ivec1, data1, rect1, ivec2, data2, rect2, nuv0, nuv_refine, k, rounds, kth_d2, npairs,
                           pairs, starts);
}

int orc_dist_query_f64(const int *ivec1, const float *data1, const double *rect1, const int *ivec2,
                       const float *data2, const double *rect2, int nuv0, int nuv_refine, int k, int rounds,
                       double *kth_d2, int *npairs, int *pairs, double *starts) {
  return dist_query<double>(ivec1, data1, rect1, ivec2, data2, rect2, nuv0, nuv_refine, k, rounds, kth_d2, npairs,
                            pairs, starts);
}

int orc_inter_query_f32(const int *ivec1, const float *data1, const float *rect1, const int *ivec2,
                        const float *data2, const float *rect2, int nuv0, int nuv_refine, int use_k, int rounds,
                        int halve_threshold, int min_nuv, long long max_pairs, long long *counts, int *pairs,
                        long long pair_cap, long long *pairs_written, float *pads, double *starts,
                        long long starts_cap) {
  return inter_query<float>(ivec1, data1, rect1, ivec2, data2, rect2, nuv0, nuv_refine, use_k, rounds,
                            halve_threshold, min_nuv, max_pairs, counts, pairs, pair_cap, pairs_written, pads, starts,
                            starts_cap);
}

int orc_inter_query_f64(const int *ivec1, const float *data1, const double *rect1, const int *ivec2,
                        const float *data2, const double *rect2, int nuv0, int nuv_refine, int use_k, int rounds,
                        int halve_threshold, int min_nuv, long long max_pairs, long long *counts, int *pairs,
                        long long pair_cap, long long *pairs_written, double *pads, double *starts,
                        long long starts_cap) {
  return inter_query<double>(ivec1, data1, rect1, ivec2, data2, rect2, nuv0, nuv_refine, use_k, rounds,
                             halve_threshold, min_nuv, max_pairs, counts, pairs, pair_cap, pairs_written, pads, starts,
                             starts_cap);
}

void orc_region_cells_f32(const int *ivec, const float *data, const float *rect, int nuv, float padding,
                          float *centers, float *radii) {
  region_cells<float>(ivec, data, rect, nuv, padding, centers, radii);
}

void orc_region_cells_f64(const int *ivec, const float *data, const double *rect, int nuv, double padding,
                          double *centers, double *radii) {
  region_cells<double>(ivec, data, rect, nuv, padding, centers, radii);
}

}  // extern "C"
