// sm_100a kernels of the NURBS distance / intersection query path.
//
// Every kernel is a template over the arithmetic type T (float for the
// VERSION5-FP32 form, double for the plain FP64 form).  The library is built
// with --fmad=false so that each written product and sum is rounded on its
// own, in the operation order of the reference (JSI_CAD_NEXT_VERSION5); the
// FP32 results are therefore bit-identical to the reference's x86 build.
//
// Work decomposition (B200: 148 SMs, 32-wide warps):
//   k_basis     one thread per (region, direction, grid line)
//   k_samples   one thread per (region, sample)
//   k_cells     one warp per (region, tile): cells and the tile's bounds
//   distance    k_dist_tau -> k_dist_cull -> k_dist_leaf -> k_dist_select -> k_dist_next
//   intersect   k_inter_cull -> k_inter_leaf -> (device radix sort) -> k_inter_* dedup
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <type_traits>

#include "jsi_internal.h"

namespace jsi {

namespace {

constexpr unsigned kFull = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T tmin(T a, T b) {  // std::min
  return (b < a) ? b : a;
}
template <typename T>
__device__ __forceinline__ T tmax(T a, T b) {  // std::max
  return (a < b) ? b : a;
}
// Single-instruction min / max for the distance cells: they differ from
// std::min / std::max only in which zero (+0 / -0) they return on a tie and
// for NaN.  A distance centre is ((lo - 0) + hi) + 0, and the trailing + 0
// turns a -0 sum into +0, so the choice of zero never reaches a centre, and
// centres are never -0; coordinates are finite.
__device__ __forceinline__ float fmn(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double fmn(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float fmx(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double fmx(double a, double b) { return fmax(a, b); }

__device__ __forceinline__ unsigned long long ordered_bits(float x) { return __float_as_uint(x); }
__device__ __forceinline__ unsigned long long ordered_bits(double x) {
  return static_cast<unsigned long long>(__double_as_longlong(x));
}
template <typename T>
__device__ __forceinline__ T from_ordered(unsigned long long b);
template <>
__device__ __forceinline__ float from_ordered<float>(unsigned long long b) {
  return __uint_as_float(static_cast<unsigned>(b));
}
template <>
__device__ __forceinline__ double from_ordered<double>(unsigned long long b) {
  return __longlong_as_double(static_cast<long long>(b));
}

// Upper bound of a non-negative value as float bits (for the shared threshold).
__device__ __forceinline__ unsigned tau_bits_up(float x) { return __float_as_uint(x); }
__device__ __forceinline__ unsigned tau_bits_up(double x) { return __float_as_uint(__double2float_ru(x)); }

template <typename T>
__device__ __forceinline__ T tau_value(unsigned bits) {
  return static_cast<T>(__uint_as_float(bits));
}

// Warp-aggregated append: returns the slot of this lane or -1.
__device__ __forceinline__ long long warp_append(bool pred, unsigned long long *counter) {
  const unsigned mask = __ballot_sync(kFull, pred);
  if (mask == 0) return -1;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(counter, static_cast<unsigned long long>(__popc(mask)));
  base = __shfl_sync(kFull, base, leader);
  if (!pred) return -1;
  return static_cast<long long>(base + __popc(mask & ((1u << lane) - 1u)));
}

// ---- lockstep batches (see Batch): query = blockIdx.y, slab offset q * qs ----
__device__ __forceinline__ long long qoff(long long qs) { return static_cast<long long>(blockIdx.y) * qs; }

template <typename P>
__device__ __forceinline__ P *qsh(P *p, long long off) {
  return (p && off) ? reinterpret_cast<P *>(reinterpret_cast<uintptr_t>(p) + off) : p;
}

template <typename T>
__device__ __forceinline__ SideRound<T> qsh(SideRound<T> s, long long off) {
  if (!off) return s;
  s.regions = qsh(s.regions, off);
  s.spans = qsh(s.spans, off);
  s.basis = qsh(s.basis, off);
  s.samples = qsh(s.samples, off);
  s.kmax = qsh(s.kmax, off);
  s.pad = qsh(s.pad, off);
  s.center = qsh(s.center, off);
  s.half = qsh(s.half, off);
  s.tlo = qsh(s.tlo, off);
  s.thi = qsh(s.thi, off);
  s.thmax = qsh(s.thmax, off);
  s.stlo = qsh(s.stlo, off);
  s.sthi = qsh(s.sthi, off);
  s.dnreg = qsh(s.dnreg, off);
  s.stmin = qsh(s.stmin, off);
  s.stmax = qsh(s.stmax, off);
  return s;
}

__device__ __forceinline__ unsigned ord_enc(float x) {
  const unsigned b = __float_as_uint(x);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_dec(unsigned e) {
  return __uint_as_float((e & 0x80000000u) ? (e & 0x7fffffffu) : ~e);
}
__device__ __forceinline__ unsigned long long ord_enc(double x) {
  const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(x));
  return (b >> 63) ? ~b : (b | (1ull << 63));
}
__device__ __forceinline__ double ord_dec(unsigned long long e) {
  return __longlong_as_double(static_cast<long long>((e >> 63) ? (e & ~(1ull << 63)) : ~e));
}

// Supertile bounds of entry i: decoded from the folded minima / maxima when
// the side carries them, else the stored vectors.
template <typename T>
__device__ __forceinline__ void st_bounds(const SideRound<T> &s, long long i, Vec4<T> &lo, Vec4<T> &hi) {
  if (s.stmin) {
    const typename OrdBits<T>::type *mn = s.stmin + i * 4, *mx = s.stmax + i * 4;
    lo = Vec4<T>{ord_dec(mn[0]), ord_dec(mn[1]), ord_dec(mn[2]), T(0)};
    hi = Vec4<T>{ord_dec(mx[0]), ord_dec(mx[1]), ord_dec(mx[2]), T(0)};
  } else {
    lo = s.stlo[i];
    hi = s.sthi[i];
  }
}

// Folds a tile's centre range into its supertile's bounds (batched rounds).
template <typename T>
__device__ __forceinline__ void fold_supertile(const SideRound<T> &s, int r, int ty, int tx, const T lo[3],
                                               const T hi[3]) {
  const long long st = static_cast<long long>(r) * s.g.nst + (ty / kMaxTile) * s.g.stw + tx / kMaxTile;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    atomicMin(s.stmin + st * 4 + c, ord_enc(lo[c]));
    atomicMax(s.stmax + st * 4 + c, ord_enc(hi[c]));
  }
}

// Region count of a side: on the device in batched refinement rounds.
template <typename T>
__device__ __forceinline__ int nreg_of(const SideRound<T> &s) {
  return s.dnreg ? *s.dnreg : s.nreg;
}

// Slot count: nslots < 0 means the device count of this round.
__device__ __forceinline__ int nslots_of(int nslots, const ScreenStats *stats) {
  return nslots >= 0 ? nslots : stats->nslots;
}

// A list length given on the host, or (kFromDevice) the device count capped
// at the list's capacity.
__device__ __forceinline__ unsigned long long count_of(unsigned long long host, unsigned long long dev,
                                                       unsigned long long cap) {
  if (host != kFromDevice) return host;
  return dev < cap ? dev : cap;
}

// ---------------------------------------------------------------------------
// Knot spans and basis functions
// ---------------------------------------------------------------------------

// Knot-span binary search (evaluation.cu:152-166).
template <typename T>
__device__ int find_span(int nk, int p, T u, const T *knots) {
  if (u <= knots[p]) return p;
  const int n = nk - p - 1;
  if (u >= knots[n]) return n - 1;
  int lo = p, hi = n;
  int mid = (lo + hi) / 2;
  // The search interval halves every step; the bound only guards against
  // non-monotone knot data (NaN).
  for (int guard = 0; guard < 64 && (u < knots[mid] || u >= knots[mid + 1]); ++guard) {
    if (u < knots[mid])
      hi = mid;
    else
      lo = mid;
    mid = (lo + hi) / 2;
  }
  return mid;
}

// Non-zero basis functions and derivatives up to order nd: the published
// algorithm A2.3 (Piegl & Tiller, The NURBS Book), in the operation order of
// evaluation.cu:168-219.  MAXP bounds the degree + 1 held in registers /
// local memory.
template <typename T, int MAXP>
__device__ void basis_ders(int span, int p, T u, const T *knots, int nd, T *out, int stride) {
  T ndu[MAXP][MAXP];
  T left[MAXP], right[MAXP];
  T a[2][MAXP];
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
  for (int j = 0; j <= p; ++j) out[j] = ndu[j][p];
  for (int k = 1; k <= 2; ++k)
    for (int j = 0; j <= p; ++j) out[k * stride + j] = T(0);
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
      out[k * stride + r] = d;
      const int t = s1;
      s1 = s2;
      s2 = t;
    }
  }
  int fac = p;
  for (int k = 1; k <= nd; ++k) {
    for (int j = 0; j <= p; ++j) out[k * stride + j] *= static_cast<T>(fac);
    fac *= p - k;
  }
}

// A2.3 for a degree P known at compile time: the same operations in the same
// order as basis_ders (so the same bits), with every loop bound a constant,
// so that the triangle and the derivative rows stay in registers instead of
// a local-memory stack frame.
template <typename T, int P>
__device__ __forceinline__ void basis_ders_fixed(int span, T u, const T *knots, int nd, T *out, int stride) {
  T ndu[P + 1][P + 1];
  T left[P + 1], right[P + 1];
  T a[2][P + 1];
  ndu[0][0] = T(1);
#pragma unroll
  for (int j = 1; j <= P; ++j) {
    left[j] = u - knots[span + 1 - j];
    right[j] = knots[span + j] - u;
    T saved = T(0);
#pragma unroll
    for (int r = 0; r < j; ++r) {
      ndu[j][r] = right[r + 1] + left[j - r];
      const T tmp = ndu[r][j - 1] / ndu[j][r];
      ndu[r][j] = saved + right[r + 1] * tmp;
      saved = left[j - r] * tmp;
    }
    ndu[j][j] = saved;
  }
#pragma unroll
  for (int j = 0; j <= P; ++j) out[j] = ndu[j][P];
#pragma unroll
  for (int k = 1; k <= 2; ++k)
#pragma unroll
    for (int j = 0; j <= P; ++j) out[k * stride + j] = T(0);
#pragma unroll
  for (int r = 0; r <= P; ++r) {
    a[0][0] = T(1);
#pragma unroll
    for (int k = 1; k <= 2; ++k) {
      if (k > nd) break;
      const int s1 = (k - 1) & 1, s2 = k & 1;
      T d = T(0);
      const int rk = r - k, pk = P - k;
      if (r >= k) {
        a[s2][0] = a[s1][0] / ndu[pk + 1][rk];
        d = a[s2][0] * ndu[rk][pk];
      }
      const int j1 = (rk >= -1) ? 1 : -rk;
      const int j2 = (r - 1 <= pk) ? k - 1 : P - r;
#pragma unroll
      for (int j = j1; j <= j2; ++j) {
        a[s2][j] = (a[s1][j] - a[s1][j - 1]) / ndu[pk + 1][rk + j];
        d += a[s2][j] * ndu[rk + j][pk];
      }
      if (r <= pk) {
        a[s2][k] = -a[s1][k - 1] / ndu[pk + 1][r];
        d += a[s2][k] * ndu[r][pk];
      }
      out[k * stride + r] = d;
    }
  }
  int fac = P;
#pragma unroll
  for (int k = 1; k <= 2; ++k) {
    if (k > nd) break;
#pragma unroll
    for (int j = 0; j <= P; ++j) out[k * stride + j] *= static_cast<T>(fac);
    fac *= P - k;
  }
}

// basis_ders with the common degrees 1-5 on the register path above; other
// degrees (MAXP >= p + 1) on the general one.
template <typename T, int MAXP>
__device__ __forceinline__ void basis_ders_any(int span, int p, T u, const T *knots, int nd, T *out, int stride) {
  switch (p) {
    case 1: basis_ders_fixed<T, 1>(span, u, knots, nd, out, stride); return;
    case 2: basis_ders_fixed<T, 2>(span, u, knots, nd, out, stride); return;
    case 3: basis_ders_fixed<T, 3>(span, u, knots, nd, out, stride); return;
    case 4: basis_ders_fixed<T, 4>(span, u, knots, nd, out, stride); return;
    case 5: basis_ders_fixed<T, 5>(span, u, knots, nd, out, stride); return;
    default: basis_ders<T, MAXP>(span, p, u, knots, nd, out, stride); return;
  }
}

template <typename T, int MAXP>
__global__ void k_basis(SurfView<T> s, const SurfView<T> *vdev, const RegionRec<T> *regions, int nreg,
                        const int *dnreg, int nuv, int p1max, int *spans, T *basis, long long qs, int cover,
                        int max_ders) {
  const long long qo = qoff(qs);
  if (vdev) s = *qsh(vdev, qo);
  if (dnreg) nreg = *qsh(dnreg, qo);
  regions = qsh(regions, qo);
  spans = qsh(spans, qo);
  basis = qsh(basis, qo);
  const long long total = static_cast<long long>(nreg) * 2 * nuv;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int q = static_cast<int>(t % nuv);
    const int dir = static_cast<int>((t / nuv) % 2);
    const int r = static_cast<int>(t / (2LL * nuv));
    const RegionRec<T> reg = regions[r];
    const T lo = dir ? reg.v0 : reg.u0;
    const T hi = dir ? reg.v1 : reg.u1;
    // ustep = (ustop - ustart) / nuv; u = ustep * idx + ustart
    // (distance_analysis.cu:92-93, evaluation.cu:366).  The covering grid of
    // the bounds mode spaces nuv samples over the whole rectangle instead and
    // puts the last one on its end.
    const T step = cover ? (hi - lo) / static_cast<T>(nuv - 1) : (hi - lo) / static_cast<T>(nuv);
    const T x = (cover && q == nuv - 1) ? hi : step * static_cast<T>(q) + lo;
    const int p = dir ? s.degv : s.degu;
    const int nk = dir ? s.nkv : s.nku;
    const T *knots = dir ? s.V : s.U;
    // Derivative rows only where a caller reads them (the intersection's
    // curvature padding); the distance path reads the values alone, and
    // the derivative rows stay zero.
    const int nd = min(dir ? s.dv : s.du, max_ders);
    T *out = basis + t * 3 * p1max;
    if (s.zero) {
      spans[t] = p;
      for (int j = 0; j < 3 * p1max; ++j) out[j] = T(0);
      continue;
    }
    const int span = find_span(nk, p, x, knots);
    spans[t] = span;
    basis_ders_any<T, MAXP>(span, p, x, knots, nd, out, p1max);
  }
}

// ---------------------------------------------------------------------------
// Sample evaluation (evaluation.cu:259-356)
// ---------------------------------------------------------------------------

// Sum over the (q+1) x (p+1) window: for every row r, a u-direction sum over
// the columns, then the v-direction sum over the rows, as the reference
// orders it.  Non-rational: 3 channels.
template <typename T>
__device__ __forceinline__ void contract3(const SurfView<T> &s, int cu0, int cv0, const T *Nu, const T *Nv, T acc[3]) {
  acc[0] = acc[1] = acc[2] = T(0);
  for (int r = 0; r <= s.degv; ++r) {
    T row0 = T(0), row1 = T(0), row2 = T(0);
    const Vec4<T> *cp = s.cpw + static_cast<long long>(s.ncpu) * (cv0 + r) + cu0;
    for (int c = 0; c <= s.degu; ++c) {
      const Vec4<T> q = cp[c];
      const T n = Nu[c];
      row0 += n * q.x;
      row1 += n * q.y;
      row2 += n * q.z;
    }
    const T m = Nv[r];
    acc[0] += m * row0;
    acc[1] += m * row1;
    acc[2] += m * row2;
  }
}

// Rational: homogeneous 4 channels, row terms (N * w) * coordinate.
template <typename T>
__device__ __forceinline__ void contract4(const SurfView<T> &s, int cu0, int cv0, const T *Nu, const T *Nv, T acc[4]) {
  acc[0] = acc[1] = acc[2] = acc[3] = T(0);
  for (int r = 0; r <= s.degv; ++r) {
    T row0 = T(0), row1 = T(0), row2 = T(0), row3 = T(0);
    const Vec4<T> *cp = s.cpw + static_cast<long long>(s.ncpu) * (cv0 + r) + cu0;
    for (int c = 0; c <= s.degu; ++c) {
      const Vec4<T> q = cp[c];
      const T nw = Nu[c] * q.w;
      row0 += nw * q.x;
      row1 += nw * q.y;
      row2 += nw * q.z;
      row3 += nw;
    }
    const T m = Nv[r];
    acc[0] += m * row0;
    acc[1] += m * row1;
    acc[2] += m * row2;
    acc[3] += m * row3;
  }
}

// Homogeneous -> Euclidean up to order 2 (evaluation.cu:77-130 with
// dim = 3, der_count = 2, stride = 4).  h: P, Pu, Pv, Puu, Puv, Pvv x 4.
template <typename T>
__device__ __forceinline__ void quotient2(T h[24]) {
  const T inv = T(1) / h[3];
#pragma unroll
  for (int q = 0; q < 24; ++q) h[q] *= inv;
  const T ws = -h[7], wt = -h[11];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    h[4 + c] += ws * h[c];
    h[8 + c] += wt * h[c];
  }
  const T wss = -h[15], wst = -h[19], wtt = -h[23];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const T F = h[c], Fs = h[4 + c], Ft = h[8 + c];
    h[12 + c] += wss * F + T(2) * ws * Fs;
    h[16 + c] += wst * F + wt * Fs + ws * Ft;
    h[20 + c] += wtt * F + T(2) * wt * Ft;
  }
}

// Full 18-value record of one sample.
template <typename T>
__device__ void eval_record(const SurfView<T> &s, int spanu, const T *Nu, int spanv, const T *Nv, int p1, T out[18]) {
#pragma unroll
  for (int q = 0; q < 18; ++q) out[q] = T(0);
  if (s.zero) return;
  const int cu0 = spanu - s.degu, cv0 = spanv - s.degv;
  // (k, l) = derivative order in (u, v); record slots P, Pu, Pv, Puu, Puv, Pvv.
  const int ku[6] = {0, 1, 0, 2, 1, 0};
  const int lv[6] = {0, 0, 1, 0, 1, 2};
  // Factored over the control-net window: each net row is read once and its
  // u sums for the orders 0..du are formed once, then every derivative
  // combination takes its v step.  Each combination's sum is the same
  // operation sequence as contract3 / contract4 (the u sum over the columns
  // in order, then acc += N_v[r] * row in row order), so the bits are those
  // of the per-combination contraction.
  const int nch = s.rat ? 4 : 3;
  T acc[6][4];
#pragma unroll
  for (int m = 0; m < 6; ++m) acc[m][0] = acc[m][1] = acc[m][2] = acc[m][3] = T(0);
  for (int r = 0; r <= s.degv; ++r) {
    const Vec4<T> *cp = s.cpw + static_cast<long long>(s.ncpu) * (cv0 + r) + cu0;
    T row[3][4];
#pragma unroll
    for (int k = 0; k < 3; ++k) row[k][0] = row[k][1] = row[k][2] = row[k][3] = T(0);
    for (int c = 0; c <= s.degu; ++c) {
      const Vec4<T> q = cp[c];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        if (k > s.du) break;
        if (s.rat) {
          const T nw = Nu[k * p1 + c] * q.w;
          row[k][0] += nw * q.x;
          row[k][1] += nw * q.y;
          row[k][2] += nw * q.z;
          row[k][3] += nw;
        } else {
          const T n = Nu[k * p1 + c];
          row[k][0] += n * q.x;
          row[k][1] += n * q.y;
          row[k][2] += n * q.z;
        }
      }
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      if (ku[m] > s.du || lv[m] > s.dv) continue;
      const T mv = Nv[lv[m] * p1 + r];
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (c < nch) acc[m][c] += mv * row[ku[m]][c];
    }
  }
  if (!s.rat) {
#pragma unroll
    for (int m = 0; m < 6; ++m) {
      if (ku[m] > s.du || lv[m] > s.dv) continue;
      out[3 * m] = acc[m][0];
      out[3 * m + 1] = acc[m][1];
      out[3 * m + 2] = acc[m][2];
    }
    return;
  }
  T h[24];
#pragma unroll
  for (int q = 0; q < 24; ++q) h[q] = T(0);
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    if (ku[m] > s.du || lv[m] > s.dv) continue;
    h[4 * m] = acc[m][0];
    h[4 * m + 1] = acc[m][1];
    h[4 * m + 2] = acc[m][2];
    h[4 * m + 3] = acc[m][3];
  }
  quotient2(h);
#pragma unroll
  for (int m = 0; m < 6; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c) out[3 * m + c] = h[4 * m + c];
}

// Position only (bit-identical to the P of the full record).
template <typename T>
__device__ __forceinline__ void eval_point(const SurfView<T> &s, int spanu, const T *Nu, int spanv, const T *Nv,
                                           T P[3]) {
  P[0] = P[1] = P[2] = T(0);
  if (s.zero) return;
  const int cu0 = spanu - s.degu, cv0 = spanv - s.degv;
  if (!s.rat) {
    contract3(s, cu0, cv0, Nu, Nv, P);
    return;
  }
  T acc[4];
  contract4(s, cu0, cv0, Nu, Nv, acc);
  const T inv = T(1) / acc[3];
  P[0] = acc[0] * inv;
  P[1] = acc[1] * inv;
  P[2] = acc[2] * inv;
}

template <typename T>
__device__ __forceinline__ void atomic_max_bits(unsigned long long *addr, T v) {
  atomicMax(addr, ordered_bits(v));
}

template <typename T>
__global__ void k_samples(SurfView<T> s, const SurfView<T> *vdev, SideRound<T> sr, int need_k, long long qs) {
  const long long qo = qoff(qs);
  if (vdev) s = *qsh(vdev, qo);
  sr = qsh(sr, qo);
  const Geom g = sr.g;
  const int nuv = g.nuv;
  const long long per = static_cast<long long>(nuv) * nuv;
  const long long total = per * nreg_of(sr);
  const int p1 = g.p1max;
  for (long long base = blockIdx.x * static_cast<long long>(blockDim.x); base < total;
       base += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long t = base + threadIdx.x;
    const bool live = t < total;
    int r = 0;
    T kuu = T(0), kuv = T(0), kvv = T(0);
    if (live) {
      r = static_cast<int>(t / per);
      const int q = static_cast<int>(t % per);
      const int idx = q % nuv, idy = q / nuv;
      const long long lu = (static_cast<long long>(r) * 2 + 0) * nuv + idx;
      const long long lv = (static_cast<long long>(r) * 2 + 1) * nuv + idy;
      const T *Nu = sr.basis + lu * 3 * p1;
      const T *Nv = sr.basis + lv * 3 * p1;
      const int spanu = sr.spans[lu], spanv = sr.spans[lv];
      Vec4<T> out;
      if (need_k) {
        T rec[18];
        eval_record(s, spanu, Nu, spanv, Nv, p1, rec);
        out.x = rec[0];
        out.y = rec[1];
        out.z = rec[2];
        // max-abs component of Puu, Puv, Pvv (common.cu:155-161)
        kuu = tmax(fabs(rec[9]), tmax(fabs(rec[10]), fabs(rec[11])));
        kuv = tmax(fabs(rec[12]), tmax(fabs(rec[13]), fabs(rec[14])));
        kvv = tmax(fabs(rec[15]), tmax(fabs(rec[16]), fabs(rec[17])));
      } else {
        T P[3];
        eval_point(s, spanu, Nu, spanv, Nv, P);
        out.x = P[0];
        out.y = P[1];
        out.z = P[2];
      }
      out.w = T(0);
      sr.samples[t] = out;
    }
    if (need_k) {
      // Max is exact and order-free: reduce within the warp when every lane
      // sits in the same region, otherwise per lane.
      const int r0 = __shfl_sync(kFull, r, 0);
      const bool uniform = __all_sync(kFull, (!live) || r == r0);
      if (uniform) {
        for (int o = 16; o > 0; o >>= 1) {
          kuu = tmax(kuu, __shfl_xor_sync(kFull, kuu, o));
          kuv = tmax(kuv, __shfl_xor_sync(kFull, kuv, o));
          kvv = tmax(kvv, __shfl_xor_sync(kFull, kvv, o));
        }
        if ((threadIdx.x & 31) == 0 && __any_sync(1u, true)) {
          atomic_max_bits(&sr.kmax[3 * r0 + 0], kuu);
          atomic_max_bits(&sr.kmax[3 * r0 + 1], kuv);
          atomic_max_bits(&sr.kmax[3 * r0 + 2], kvv);
        }
      } else if (live) {
        atomic_max_bits(&sr.kmax[3 * r + 0], kuu);
        atomic_max_bits(&sr.kmax[3 * r + 1], kuv);
        atomic_max_bits(&sr.kmax[3 * r + 2], kvv);
      }
    }
  }
}

// Curvature padding per region (common.cu:149-172, intersection.cu:187-205).
template <typename T>
__global__ void k_pad(SideRound<T> sr, int use_k, T span_u0, T span_v0) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= sr.nreg) return;
  T pad = T(0);
  if (use_k) {
    const T muu = from_ordered<T>(sr.kmax[3 * r + 0]);
    const T muv = from_ordered<T>(sr.kmax[3 * r + 1]);
    const T mvv = from_ordered<T>(sr.kmax[3 * r + 2]);
    const int n = sr.g.nuv;
    const int side = n > 1 ? n - 1 : 1;
    const T ss = static_cast<T>(side * side);
    const T raw = (muu / ss + T(2) * muv / ss + mvv / ss) / T(8);
    const RegionRec<T> reg = sr.regions[r];
    const T us = fabs(reg.u1 - reg.u0) / span_u0;
    const T vs = fabs(reg.v1 - reg.v0) / span_v0;
    const T ps = tmax(us, vs);
    pad = raw * ps * ps;
    if (!isfinite(pad) || pad < T(0)) pad = T(0);
  }
  sr.pad[r] = pad;
}

template <typename T>
__device__ __forceinline__ T pos_inf();
template <>
__device__ __forceinline__ float pos_inf<float>() {
  return __uint_as_float(0x7f800000u);
}
template <>
__device__ __forceinline__ double pos_inf<double>() {
  return __longlong_as_double(0x7ff0000000000000ll);
}

// Cell boxes from 4 corner samples, tile-major (distance_analysis.cu:45-86,
// intersection.cu:106-148), one warp per tile (<= 64 cells, 2 per lane); the
// same warp reduces the tile's centre range and largest half span.  Half spans
// are stored without the padding; the screen forms radius = half + pad exactly
// as the reference does.
template <typename T>
__global__ void k_cells(SideRound<T> sr, int intersect, long long qs) {
  sr = qsh(sr, qoff(qs));
  const Geom g = sr.g;
  const int lane = threadIdx.x & 31;
  const long long ntile_total = static_cast<long long>(nreg_of(sr)) * g.ntiles;
  const int te2 = g.te * g.te;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long t = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; t < ntile_total;
       t += nwarps) {
    const int r = static_cast<int>(t / g.ntiles);
    const int tile = static_cast<int>(t - static_cast<long long>(r) * g.ntiles);
    const int ty = tile / g.tw, tx = tile - (tile / g.tw) * g.tw;
    const int nv = min(g.te, g.W - ty * g.te), nu = min(g.te, g.W - tx * g.te);
    const Vec4<T> *S = sr.samples + static_cast<long long>(r) * g.nuv * g.nuv;
    T lo[3] = {pos_inf<T>(), pos_inf<T>(), pos_inf<T>()};
    T hi[3] = {-pos_inf<T>(), -pos_inf<T>(), -pos_inf<T>()};
    T hm[3] = {T(0), T(0), T(0)};
    for (int local = lane; local < te2; local += 32) {
      const int a = local / g.te, b = local - (local / g.te) * g.te;
      Vec4<T> cen{T(0), T(0), T(0), T(0)}, hal{T(0), T(0), T(0), T(0)};
      if (a < nv && b < nu) {
        const int iv = ty * g.te + a, iu = tx * g.te + b;
        const Vec4<T> p0 = S[iv * g.nuv + iu];
        const Vec4<T> p1 = S[iv * g.nuv + iu + 1];
        const Vec4<T> p2 = S[(iv + 1) * g.nuv + iu];
        const Vec4<T> p3 = S[(iv + 1) * g.nuv + iu + 1];
        const T lx = tmin(p0.x, tmin(p1.x, tmin(p2.x, p3.x)));
        const T ly = tmin(p0.y, tmin(p1.y, tmin(p2.y, p3.y)));
        const T lz = tmin(p0.z, tmin(p1.z, tmin(p2.z, p3.z)));
        const T hx = tmax(p0.x, tmax(p1.x, tmax(p2.x, p3.x)));
        const T hy = tmax(p0.y, tmax(p1.y, tmax(p2.y, p3.y)));
        const T hz = tmax(p0.z, tmax(p1.z, tmax(p2.z, p3.z)));
        if (intersect) {
          cen.x = (lx + hx) / T(2);
          cen.y = (ly + hy) / T(2);
          cen.z = (lz + hz) / T(2);
        } else {
          cen.x = (lx - T(0) + hx + T(0)) / T(2);
          cen.y = (ly - T(0) + hy + T(0)) / T(2);
          cen.z = (lz - T(0) + hz + T(0)) / T(2);
        }
        hal.x = (hx - lx) / T(2);
        hal.y = (hy - ly) / T(2);
        hal.z = (hz - lz) / T(2);
        lo[0] = tmin(lo[0], cen.x);
        lo[1] = tmin(lo[1], cen.y);
        lo[2] = tmin(lo[2], cen.z);
        hi[0] = tmax(hi[0], cen.x);
        hi[1] = tmax(hi[1], cen.y);
        hi[2] = tmax(hi[2], cen.z);
        hm[0] = tmax(hm[0], hal.x);
        hm[1] = tmax(hm[1], hal.y);
        hm[2] = tmax(hm[2], hal.z);
      }
      sr.center[t * te2 + local] = cen;
      if (intersect) sr.half[t * te2 + local] = hal;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = tmin(lo[c], __shfl_xor_sync(kFull, lo[c], o));
        hi[c] = tmax(hi[c], __shfl_xor_sync(kFull, hi[c], o));
        hm[c] = tmax(hm[c], __shfl_xor_sync(kFull, hm[c], o));
      }
    }
    if (lane == 0) {
      sr.tlo[t] = Vec4<T>{lo[0], lo[1], lo[2], T(0)};
      sr.thi[t] = Vec4<T>{hi[0], hi[1], hi[2], T(0)};
      if (sr.thmax) sr.thmax[t] = Vec4<T>{hm[0], hm[1], hm[2], T(0)};
    }
  }
}

// Intersection cells of small regions in one pass (refinement rounds, nuv <=
// kRegNuv): a block of kRegThreads threads takes rpb regions at a time (rpb =
// kRegThreads / nuv^2, at most kRegMaxRpb, so that the block's threads stay
// busy at nuv 4 and 8) and computes, in shared memory, the regions' knot spans
// and basis lines (as k_basis), samples and compute_K terms (as k_samples),
// paddings (as k_pad), and cells and tile ranges (as k_cells), with the same
// functions and operation order, so centres, half spans and paddings carry
// the same bits.  Tile ranges are folded with order-preserving integer
// atomics (exact minima / maxima).  Nothing but the cells, tile ranges and
// paddings goes to HBM.
constexpr int kRegThreads = 256;
constexpr int kRegMaxRpb = 16;

__host__ __device__ inline int region_cells_rpb(int nuv) {
  int r = kRegThreads / (nuv * nuv);
  if (r < 1) r = 1;
  if (r > kRegMaxRpb) r = kRegMaxRpb;
  return r;
}

__host__ __device__ inline size_t al16(size_t b) { return (b + 15) & ~static_cast<size_t>(15); }

// Shared-memory layout of one block: basis [rpb][2 nuv][3 p1], spans
// [rpb][2 nuv], samples [rpb][nuv^2], region maxima [rpb][3], tile folds
// [rpb][ntiles][9].
template <typename T>
__host__ __device__ inline size_t region_cells_smem(const Geom &g, int rpb, size_t *offs) {
  using U = typename OrdBits<T>::type;
  size_t o = 0;
  offs[0] = o;
  o = al16(o + sizeof(T) * rpb * 2 * g.nuv * 3 * g.p1max);
  offs[1] = o;
  o = al16(o + sizeof(int) * rpb * 2 * g.nuv);
  offs[2] = o;
  o = al16(o + sizeof(Vec4<T>) * rpb * g.nuv * g.nuv);
  offs[3] = o;
  o = al16(o + sizeof(unsigned long long) * rpb * 3);
  offs[4] = o;
  o = al16(o + sizeof(U) * rpb * g.ntiles * 9);
  return o;
}

// FP64: three blocks per SM (at most 85 registers a thread, a few words
// spilled) instead of the two that 126 registers gave; the kernel waits on
// block barriers and shared-memory loads, so more blocks in flight shorten it.
// FP32: four blocks (64 registers, no spills).
template <typename T>
__global__ void __launch_bounds__(kRegThreads, sizeof(T) == 8 ? 3 : 4) k_region_cells(SurfView<T> s, SideRound<T> sr, int need_k, T span_u0,
                                                              T span_v0, int cover) {
  using U = typename OrdBits<T>::type;
  extern __shared__ __align__(16) unsigned char rc_raw[];
  const Geom g = sr.g;
  const int nuv = g.nuv, p1 = g.p1max, te2 = g.te * g.te, nl = 2 * nuv, ns = nuv * nuv;
  const int ncell = g.ntiles * te2, rpb = region_cells_rpb(nuv), tid = threadIdx.x, nth = blockDim.x;
  size_t offs[5];
  region_cells_smem<T>(g, rpb, offs);
  T *sb = reinterpret_cast<T *>(rc_raw + offs[0]);
  int *ssp = reinterpret_cast<int *>(rc_raw + offs[1]);
  Vec4<T> *smp = reinterpret_cast<Vec4<T> *>(rc_raw + offs[2]);
  unsigned long long *skm = reinterpret_cast<unsigned long long *>(rc_raw + offs[3]);
  U *stl = reinterpret_cast<U *>(rc_raw + offs[4]);
  const U lo_id = ~U(0), hi_id = U(0), hm_id = ord_enc(T(0));
  for (int r0 = blockIdx.x * rpb; r0 < sr.nreg; r0 += gridDim.x * rpb) {
    const int nr = min(rpb, sr.nreg - r0);
    for (int t = tid; t < nr * 3; t += nth) skm[t] = 0ull;
    for (int t = tid; t < nr * g.ntiles; t += nth) {
      U *f = stl + static_cast<long long>(t) * 9;
      f[0] = f[1] = f[2] = lo_id;
      f[3] = f[4] = f[5] = hi_id;
      f[6] = f[7] = f[8] = hm_id;
    }
    // basis lines of every region: u lines 0..nuv-1, v lines nuv..2 nuv-1
    for (int t = tid; t < nr * nl; t += nth) {
      const int k = t / nl, line = t - k * nl;
      const RegionRec<T> reg = sr.regions[r0 + k];
      const int dir = line >= nuv, q = line - dir * nuv;
      const T lo = dir ? reg.v0 : reg.u0;
      const T hi = dir ? reg.v1 : reg.u1;
      const T step = cover ? (hi - lo) / static_cast<T>(nuv - 1) : (hi - lo) / static_cast<T>(nuv);
      const T x = (cover && q == nuv - 1) ? hi : step * static_cast<T>(q) + lo;
      const int p = dir ? s.degv : s.degu;
      T *out = sb + static_cast<long long>(t) * 3 * p1;
      for (int j = 0; j < 3 * p1; ++j) out[j] = T(0);
      if (s.zero) {
        ssp[t] = p;
      } else {
        const int span = find_span(dir ? s.nkv : s.nku, p, x, dir ? s.V : s.U);
        ssp[t] = span;
        basis_ders_any<T, kRegP1>(span, p, x, dir ? s.V : s.U, min(dir ? s.dv : s.du, 2), out, p1);
      }
    }
    __syncthreads();
    // samples and compute_K terms (max is exact and order-free)
    for (int t = tid; t < nr * ns; t += nth) {
      const int k = t / ns, qq = t - k * ns;
      const int idx = qq % nuv, idy = qq / nuv;
      const int lu = k * nl + idx, lv = k * nl + nuv + idy;
      const T *Nu = sb + static_cast<long long>(lu) * 3 * p1, *Nv = sb + static_cast<long long>(lv) * 3 * p1;
      Vec4<T> P;
      if (need_k) {
        T rec[18];
        eval_record(s, ssp[lu], Nu, ssp[lv], Nv, p1, rec);
        P = Vec4<T>{rec[0], rec[1], rec[2], T(0)};
        atomic_max_bits(&skm[3 * k + 0], tmax(fabs(rec[9]), tmax(fabs(rec[10]), fabs(rec[11]))));
        atomic_max_bits(&skm[3 * k + 1], tmax(fabs(rec[12]), tmax(fabs(rec[13]), fabs(rec[14]))));
        atomic_max_bits(&skm[3 * k + 2], tmax(fabs(rec[15]), tmax(fabs(rec[16]), fabs(rec[17]))));
      } else {
        T q3[3];
        eval_point(s, ssp[lu], Nu, ssp[lv], Nv, q3);
        P = Vec4<T>{q3[0], q3[1], q3[2], T(0)};
      }
      smp[t] = P;
    }
    __syncthreads();
    // paddings (k_pad)
    for (int k = tid; k < nr; k += nth) {
      const int r = r0 + k;
      T pad = T(0);
      if (need_k) {
        const T muu = from_ordered<T>(skm[3 * k]), muv = from_ordered<T>(skm[3 * k + 1]),
                mvv = from_ordered<T>(skm[3 * k + 2]);
        const int side = nuv > 1 ? nuv - 1 : 1;
        const T ss = static_cast<T>(side * side);
        const T raw = (muu / ss + T(2) * muv / ss + mvv / ss) / T(8);
        const RegionRec<T> reg = sr.regions[r];
        const T us = fabs(reg.u1 - reg.u0) / span_u0;
        const T vs = fabs(reg.v1 - reg.v0) / span_v0;
        const T ps = tmax(us, vs);
        pad = raw * ps * ps;
        if (!isfinite(pad) || pad < T(0)) pad = T(0);
        sr.kmax[3 * r + 0] = skm[3 * k];
        sr.kmax[3 * r + 1] = skm[3 * k + 1];
        sr.kmax[3 * r + 2] = skm[3 * k + 2];
      }
      sr.pad[r] = pad;
    }
    // cells, tile-major (k_cells), folded into the tile ranges
    for (int t = tid; t < nr * ncell; t += nth) {
      const int k = t / ncell, c = t - k * ncell;
      const int tile = c / te2, local = c - tile * te2;
      const int ty = tile / g.tw, tx = tile - ty * g.tw;
      const int a = local / g.te, b = local - (local / g.te) * g.te;
      const int nv = min(g.te, g.W - ty * g.te), nu = min(g.te, g.W - tx * g.te);
      Vec4<T> cen{T(0), T(0), T(0), T(0)}, hal{T(0), T(0), T(0), T(0)};
      if (a < nv && b < nu) {
        const int iv = ty * g.te + a, iu = tx * g.te + b;
        const Vec4<T> *S = smp + static_cast<long long>(k) * ns;
        const Vec4<T> p0 = S[iv * nuv + iu], q1 = S[iv * nuv + iu + 1];
        const Vec4<T> p2 = S[(iv + 1) * nuv + iu], p3 = S[(iv + 1) * nuv + iu + 1];
        const T lx = tmin(p0.x, tmin(q1.x, tmin(p2.x, p3.x)));
        const T ly = tmin(p0.y, tmin(q1.y, tmin(p2.y, p3.y)));
        const T lz = tmin(p0.z, tmin(q1.z, tmin(p2.z, p3.z)));
        const T hx = tmax(p0.x, tmax(q1.x, tmax(p2.x, p3.x)));
        const T hy = tmax(p0.y, tmax(q1.y, tmax(p2.y, p3.y)));
        const T hz = tmax(p0.z, tmax(q1.z, tmax(p2.z, p3.z)));
        cen.x = (lx + hx) / T(2);
        cen.y = (ly + hy) / T(2);
        cen.z = (lz + hz) / T(2);
        hal.x = (hx - lx) / T(2);
        hal.y = (hy - ly) / T(2);
        hal.z = (hz - lz) / T(2);
        U *f = stl + (static_cast<long long>(k) * g.ntiles + tile) * 9;
        atomicMin(f + 0, ord_enc(cen.x));
        atomicMin(f + 1, ord_enc(cen.y));
        atomicMin(f + 2, ord_enc(cen.z));
        atomicMax(f + 3, ord_enc(cen.x));
        atomicMax(f + 4, ord_enc(cen.y));
        atomicMax(f + 5, ord_enc(cen.z));
        atomicMax(f + 6, ord_enc(hal.x));
        atomicMax(f + 7, ord_enc(hal.y));
        atomicMax(f + 8, ord_enc(hal.z));
      }
      const long long o = static_cast<long long>(r0 + k) * g.cpr + c;
      sr.center[o] = cen;
      sr.half[o] = hal;
    }
    __syncthreads();
    for (int t = tid; t < nr * g.ntiles; t += nth) {
      const U *f = stl + static_cast<long long>(t) * 9;
      const long long o = static_cast<long long>(r0) * g.ntiles + t;
      sr.tlo[o] = Vec4<T>{ord_dec(f[0]), ord_dec(f[1]), ord_dec(f[2]), T(0)};
      sr.thi[o] = Vec4<T>{ord_dec(f[3]), ord_dec(f[4]), ord_dec(f[5]), T(0)};
      sr.thmax[o] = Vec4<T>{ord_dec(f[6]), ord_dec(f[7]), ord_dec(f[8]), T(0)};
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void k_records(SurfView<T> s, T ustep, T vstep, T ustart, T vstart, int nuv, T *out) {
  // Full-record grid for the evalWithCuda entry point; basis per sample.
  const long long total = static_cast<long long>(nuv) * nuv;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int idx = static_cast<int>(t % nuv), idy = static_cast<int>(t / nuv);
    const T u = ustep * static_cast<T>(idx) + ustart;
    const T v = vstep * static_cast<T>(idy) + vstart;
    T Nu[3 * kMaxDeg], Nv[3 * kMaxDeg];
    T rec[18];
    int spanu = s.degu, spanv = s.degv;
    if (!s.zero) {
      spanu = find_span(s.nku, s.degu, u, s.U);
      basis_ders_any<T, kMaxDeg>(spanu, s.degu, u, s.U, s.du, Nu, kMaxDeg);
      spanv = find_span(s.nkv, s.degv, v, s.V);
      basis_ders_any<T, kMaxDeg>(spanv, s.degv, v, s.V, s.dv, Nv, kMaxDeg);
    }
    eval_record(s, spanu, Nu, spanv, Nv, kMaxDeg, rec);
    T *o = out + t * 18;
    for (int q = 0; q < 18; ++q) o[q] = rec[q];
  }
}

// ---------------------------------------------------------------------------
// Screening helpers
// ---------------------------------------------------------------------------

// Squared centre distance, distance_analysis.cu:202-207.
template <typename T>
__device__ __forceinline__ T center_d2(const Vec4<T> &a, const Vec4<T> &b) {
  const T dx = a.x - b.x;
  const T dy = a.y - b.y;
  const T dz = a.z - b.z;
  return dx * dx + dy * dy + dz * dz;
}

// Gap between two centre ranges on one axis; rounding is monotone, so the
// rounded gap never exceeds the rounded |c1 - c2| of any member pair.
template <typename T>
__device__ __forceinline__ T axis_gap(T lo1, T hi1, T lo2, T hi2) {
  const T g1 = lo2 - hi1;
  const T g2 = lo1 - hi2;
  return tmax(tmax(g1, g2), T(0));
}

// Lower bound of every rounded d2 between members of two tiles.
template <typename T>
__device__ __forceinline__ T tile_lb(const Vec4<T> &lo1, const Vec4<T> &hi1, const Vec4<T> &lo2, const Vec4<T> &hi2) {
  const T gx = axis_gap(lo1.x, hi1.x, lo2.x, hi2.x);
  const T gy = axis_gap(lo1.y, hi1.y, lo2.y, hi2.y);
  const T gz = axis_gap(lo1.z, hi1.z, lo2.z, hi2.z);
  return gx * gx + gy * gy + gz * gz;
}


// Bitonic sort of n (power of two) unsigned keys in shared memory, ascending.
__device__ void bitonic_u32(unsigned *a, int n) {
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const unsigned x = a[i], y = a[j];
          if ((x > y) == up) {
            a[i] = y;
            a[j] = x;
          }
        }
      }
    }
  }
  __syncthreads();
}

// Block-wide: k-th smallest of the per-thread minima (distinct pairs), as a
// valid upper bound of the k-th smallest d2 over all pairs, folded into tau.
__device__ void fold_tau(unsigned my_bits, int k, unsigned *tau, unsigned *sh) {
  const int n = blockDim.x;  // power of two
  sh[threadIdx.x] = my_bits;
  bitonic_u32(sh, n);
  if (threadIdx.x == 0 && k <= n) {
    const unsigned b = sh[k - 1];
    if (b != 0x7f800000u) atomicMin(tau, b);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Distance screening
// ---------------------------------------------------------------------------

// Representative cell of a tile: its middle cell (always valid).
__device__ __forceinline__ int tile_rep(int t, const Geom &g) {
  const int ty = t / g.tw, tx = t - (t / g.tw) * g.tw;
  const int nv = min(g.te, g.W - ty * g.te), nu = min(g.te, g.W - tx * g.te);
  return (nv / 2) * g.te + nu / 2;
}

// Lower bound as float bits, rounded down (ordering key of the survivors).
__device__ __forceinline__ unsigned lb_bits_down(float x) { return __float_as_uint(x); }
__device__ __forceinline__ unsigned lb_bits_down(double x) { return __float_as_uint(__double2float_rd(x)); }

// ---- FP32-screen thresholds ----------------------------------------------
// In the FP32-screen form every cell centre c32 differs from the FP64 form's
// c64 by at most a per-coordinate bound; e bounds the Euclidean norm of the
// summed bounds of both sides (computed on the host, rounded up).  With
// D = exact distance of two centres and 5u the relative error of a computed
// squared distance in either precision (2^-20 covers both):
//   d2_64 <= tau64  =>  d2_32 <= screen_widen(tau64, e)
//   d2_32 <= v      =>  d2_64 <= screen_ub(v, e)
// All operations round upward.
__device__ __forceinline__ float screen_widen(float tau64, float e) {
  if (!(tau64 < __uint_as_float(0x7f800000u))) return tau64;
  float sq = __fsqrt_ru(__fmul_ru(tau64, 1.0f + 0x1p-20f));
  sq = __fadd_ru(sq, e);
  return __fmul_ru(__fmul_ru(sq, sq), 1.0f + 0x1p-20f);
}
__device__ __forceinline__ unsigned screen_ub_bits(float v32, float e) {
  if (!(v32 < __uint_as_float(0x7f800000u))) return 0x7f800000u;
  float sq = __fsqrt_ru(__fmul_ru(v32, 1.0f + 0x1p-20f));
  sq = __fadd_ru(sq, e);
  return __float_as_uint(__fmul_ru(__fmul_ru(sq, sq), 1.0f + 0x1p-20f));
}

// Squared distance of two centres: the reference's operation order (exact
// forms), or FMA-contracted for the FP32 screen (error covered above).
template <typename T, bool S>
__device__ __forceinline__ T pair_d2(const Vec4<T> &a, const Vec4<T> &b) {
  if constexpr (S) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
  } else {
    return center_d2(a, b);
  }
}

// Threshold value (in the FP64 domain for the screen) of a pair distance.
template <typename T, bool S>
__device__ __forceinline__ unsigned thr_bits(T d2, float e) {
  if constexpr (S) {
    return screen_ub_bits(d2, e);
  } else {
    return tau_bits_up(d2);
  }
}

// Compare value (in the FP32 domain for the screen) of the shared threshold.
template <typename T, bool S>
__device__ __forceinline__ T thr_compare(unsigned tau_bits, float e) {
  if constexpr (S) {
    return screen_widen(__uint_as_float(tau_bits), e);
  } else {
    return tau_value<T>(tau_bits);
  }
}

// Ascending bitonic sort of one value per lane; returns the value of lane q.
__device__ __forceinline__ unsigned warp_sorted_at(unsigned v, int q) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const unsigned o = __shfl_xor_sync(kFull, v, stride);
      const bool asc = (lane & size) == 0 || size == 32;
      const bool low = (lane & stride) == 0;
      v = (low == asc) ? min(v, o) : max(v, o);
    }
  }
  return __shfl_sync(kFull, v, q);
}

// Threshold seed: the representative cell pair (middle cells) of every tile
// pair.  Rows (slot, t1) are spread over blocks, t2 over threads; each block
// folds the k-th smallest of its per-thread minima into tau.
template <typename T, bool S>
__global__ void __launch_bounds__(256) k_dist_tau(SideRound<T> a, SideRound<T> b, const int *map1,
                                                  const int *map2, int nslots, int k, ScreenStats *stats, float e,
                                                  long long qs) {
  __shared__ unsigned sh[256];
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  nslots = nslots_of(nslots, stats);
  const Geom g1 = a.g, g2 = b.g;
  const int n1 = g1.te * g1.te, n2 = g2.te * g2.te;
  const int nrows = nslots * g1.ntiles;
  T best = pos_inf<T>();  // smallest pair d2; thr_bits is monotone, so it is applied once per fold
  for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
    const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
    const Vec4<T> c1 = a.center[(static_cast<long long>(map1[slot]) * g1.ntiles + t1) * n1 + tile_rep(t1, g1)];
    const long long base2 = static_cast<long long>(map2[slot]) * g2.ntiles;
    for (int t2 = threadIdx.x; t2 < g2.ntiles; t2 += blockDim.x) {
      const Vec4<T> c2 = b.center[(base2 + t2) * n2 + tile_rep(t2, g2)];
      best = tmin(best, pair_d2<T, S>(c1, c2));
    }
  }
  fold_tau(thr_bits<T, S>(best, e), k, &stats->tau_bits, sh);
}

// Tile pairs whose box-gap bound does not exceed tau survive, with the bound
// (float, rounded down) as the key the leaf is ordered by.
template <typename T, bool S>
__global__ void k_dist_cull(SideRound<T> a, SideRound<T> b, const int *map1, const int *map2, int nslots,
                            unsigned long long *surv, unsigned *surv_lb, unsigned long long surv_cap,
                            ScreenStats *stats, float e, long long qs) {
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  surv = qsh(surv, qo);
  surv_lb = qsh(surv_lb, qo);
  nslots = nslots_of(nslots, stats);
  const Geom g1 = a.g, g2 = b.g;
  const int nrows = nslots * g1.ntiles;
  const T tau = thr_compare<T, S>(stats->tau_bits, e);
  for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
    const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
    const long long i1 = static_cast<long long>(map1[slot]) * g1.ntiles + t1;
    const Vec4<T> lo1 = a.tlo[i1], hi1 = a.thi[i1];
    const long long base2 = static_cast<long long>(map2[slot]) * g2.ntiles;
    for (int t0 = 0; t0 < g2.ntiles; t0 += blockDim.x) {
      const int t2 = t0 + threadIdx.x;
      bool keep = false;
      T lb = T(0);
      if (t2 < g2.ntiles) {
        lb = tile_lb(lo1, hi1, b.tlo[base2 + t2], b.thi[base2 + t2]);
        // The screen's pair distances are FMA-contracted: shave the rounded
        // bound by 2^-19 (more than the 12u they can differ by).
        if constexpr (S) lb = __fmul_rd(lb, 1.0f - 0x1p-19f);
        keep = lb <= tau;
      }
      const long long pos = warp_append(keep, &stats->survivors);
      if (pos >= 0 && static_cast<unsigned long long>(pos) < surv_cap) {
        surv[pos] = pack_tile_pair(static_cast<unsigned>(row), static_cast<unsigned>(t2));
        if (surv_lb) surv_lb[pos] = lb_bits_down(lb);
      }
    }
  }
  if (threadIdx.x == 0 && blockIdx.x == 0)
    atomicAdd(&stats->tile_pairs, static_cast<unsigned long long>(nrows) * g2.ntiles);
}

// All cell pairs of the surviving tile pairs, one warp per tile pair taken
// from a work counter: the tile-2 centres sit in registers (cells lane and
// lane+32), the tile-1 centres are broadcast row by row.  A pair with
// d2 <= tau is a candidate.  With surv sorted by its lower bound, a warp that
// meets a bound above tau stops: every later tile pair has a larger bound and
// tau never grows.  Warps tighten tau with the k-th smallest of their lanes'
// minima (k <= 32); blocks do the same at exit for larger k.
template <typename T>
__device__ __forceinline__ Vec4<T> shfl_vec(const Vec4<T> &v, int src) {
  Vec4<T> r;
  r.x = __shfl_sync(kFull, v.x, src);
  r.y = __shfl_sync(kFull, v.y, src);
  r.z = __shfl_sync(kFull, v.z, src);
  r.w = T(0);
  return r;
}

template <typename T, bool S>
__global__ void __launch_bounds__(256) k_dist_leaf(SideRound<T> a, SideRound<T> b, const int *map1, const int *map2,
                                                   const unsigned long long *surv, const unsigned *surv_lb,
                                                   unsigned long long nsurv, unsigned long long surv_cap,
                                                   int sorted, int k, int collect, DistCand<T> *cand,
                                                   unsigned long long cand_cap, ScreenStats *stats, float e,
                                                   long long qs) {
  __shared__ unsigned sh[256];
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  surv = qsh(surv, qo);
  surv_lb = qsh(surv_lb, qo);
  cand = qsh(cand, qo);
  nsurv = count_of(nsurv, stats->survivors, surv_cap);
  const Geom g1 = a.g, g2 = b.g;
  const int te1 = g1.te, te2 = g2.te;
  const int n1 = te1 * te1, n2 = te2 * te2;
  const int lane = threadIdx.x & 31;
  unsigned long long tests = 0;
  T best = pos_inf<T>();
  const Vec4<T> far4{pos_inf<T>(), pos_inf<T>(), pos_inf<T>(), T(0)};
  // Sorted lists are taken in order from a work counter (a bound above tau
  // ends the warp); unsorted lists are split statically and skip such pairs.
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  // Unsorted lists are split statically: warp i owns entries i, i + nwarps,
  // ... and scans 32 of them at once (one bound per lane, a ballot of those
  // under tau), then works through the passing ones.
  unsigned long long chunk = (blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x) >> 5;
  unsigned pending = 0;
  for (;;) {
    unsigned long long w = 0;
    if (sorted) {
      if (lane == 0) w = atomicAdd(&stats->work, 1ull);
      w = __shfl_sync(kFull, w, 0);
    } else {
      while (pending == 0 && chunk < nsurv) {
        const unsigned long long x = chunk + lane * nwarps;
        const unsigned tb = *reinterpret_cast<volatile unsigned *>(&stats->tau_bits);
        const bool pass = x < nsurv && (!surv_lb || __uint_as_float(surv_lb[x]) <=
                                                        static_cast<float>(thr_compare<float, S>(tb, e)));
        pending = __ballot_sync(kFull, pass);
        if (pending == 0) chunk += nwarps * 32;
      }
      if (pending == 0) break;
      w = chunk + static_cast<unsigned long long>(__ffs(pending) - 1) * nwarps;
      pending &= pending - 1;
      if (pending == 0) chunk += nwarps * 32;
    }
    if (w >= nsurv) break;
    const unsigned taub = *reinterpret_cast<volatile unsigned *>(&stats->tau_bits);
    const T tau = thr_compare<T, S>(taub, e);
    if (surv_lb && __uint_as_float(surv_lb[w]) > static_cast<float>(thr_compare<float, S>(taub, e))) {
      if (sorted) break;
      continue;
    }
    const unsigned long long q = surv[w];
    const int row = static_cast<int>(q >> 32), t2 = static_cast<int>(q & 0xffffffffull);
    const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
    const long long base1 = (static_cast<long long>(map1[slot]) * g1.ntiles + t1) * n1;
    const long long base2 = (static_cast<long long>(map2[slot]) * g2.ntiles + t2) * n2;
    const int ty1 = t1 / g1.tw, tx1 = t1 - ty1 * g1.tw, ty2 = t2 / g2.tw, tx2 = t2 - ty2 * g2.tw;
    const int nv1 = min(te1, g1.W - ty1 * te1), nu1 = min(te1, g1.W - tx1 * te1);
    const int nv2 = min(te2, g2.W - ty2 * te2), nu2 = min(te2, g2.W - tx2 * te2);
    const int ja = lane, jb = lane + 32;
    const int ja_v = ja / te2, ja_u = ja - ja_v * te2, jb_v = jb / te2, jb_u = jb - jb_v * te2;
    const bool va = ja < n2 && ja_v < nv2 && ja_u < nu2;
    const bool vb = jb < n2 && jb_v < nv2 && jb_u < nu2;
    const Vec4<T> c2a = va ? b.center[base2 + ja] : far4;
    const Vec4<T> c2b = vb ? b.center[base2 + jb] : far4;
    // Tile-1 centres: two per lane, broadcast row by row through shuffles.
    const Vec4<T> c1a = ja < n1 ? a.center[base1 + ja] : far4;
    const Vec4<T> c1b = jb < n1 ? a.center[base1 + jb] : far4;
    const int cja = (ty2 * te2 + ja_v) * g2.W + tx2 * te2 + ja_u;
    const int cjb = (ty2 * te2 + jb_v) * g2.W + tx2 * te2 + jb_u;
    for (int a1 = 0; a1 < nv1; ++a1) {
      for (int b1 = 0; b1 < nu1; ++b1) {
        const int l1 = a1 * te1 + b1;
        const Vec4<T> c1 = shfl_vec(l1 < 32 ? c1a : c1b, l1 & 31);
        const T da = pair_d2<T, S>(c1, c2a);
        const T db = pair_d2<T, S>(c1, c2b);
        best = tmin(best, tmin(da, db));
        if (collect) {
          // tau is +inf until k pairs are known: padding lanes (d2 = +inf) must not pass.
          const bool ha = va && da <= tau, hb = vb && db <= tau;
          if (__any_sync(kFull, ha || hb)) {
            const int ci = (ty1 * te1 + a1) * g1.W + tx1 * te1 + b1;
            long long pos = warp_append(ha, &stats->candidates);
            if (pos >= 0 && static_cast<unsigned long long>(pos) < cand_cap)
              cand[pos] = DistCand<T>{da, slot, ci, cja};
            pos = warp_append(hb, &stats->candidates);
            if (pos >= 0 && static_cast<unsigned long long>(pos) < cand_cap)
              cand[pos] = DistCand<T>{db, slot, ci, cjb};
          }
        }
      }
    }
    if (lane == 0) tests += static_cast<unsigned long long>(nv1 * nu1) * (nv2 * nu2);
    if (k <= 32) {
      const unsigned mine = thr_bits<T, S>(best, e);
      if (__popc(__ballot_sync(kFull, mine < taub)) >= k) {
        const unsigned kth = warp_sorted_at(mine, k - 1);
        if (lane == 0) atomicMin(&stats->tau_bits, kth);
      }
    }
  }
  if (collect && lane == 0) atomicAdd(&stats->pair_tests, tests);
  if (k > 32) fold_tau(thr_bits<T, S>(best, e), k, &stats->tau_bits, sh);
}

// Threshold pass over the first nhead tile pairs (the ones with the smallest
// bounds when surv is sorted): one warp per tile pair, each lane keeps the KL
// smallest d2 of its own pairs in a sorted register list, and the warp merges
// the 32 lists to the exact k-th smallest d2 of the tile pair (k <= KL), which
// is a valid upper bound of the global k-th and is folded into tau.  Only d2
// <= tau (the threshold when the tile pair starts) enter the lists: with k
// such values the k-th among them is the tile pair's k-th, and with fewer the
// tile pair's k-th exceeds tau and its fold would change nothing.
template <typename T, int KL, bool S>
__global__ void __launch_bounds__(256) k_dist_head(SideRound<T> a, SideRound<T> b, const int *map1,
                                                   const int *map2, const unsigned long long *surv,
                                                   unsigned long long nhead, int k, ScreenStats *stats, float e,
                                                   long long qs) {
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  surv = qsh(surv, qo);
  nhead = count_of(nhead, stats->nhead, stats->nhead);
  const Geom g1 = a.g, g2 = b.g;
  const int te1 = g1.te, te2 = g2.te;
  const int n1 = te1 * te1, n2 = te2 * te2;
  const int lane = threadIdx.x & 31;
  const Vec4<T> far4{pos_inf<T>(), pos_inf<T>(), pos_inf<T>(), T(0)};
  const unsigned long long nwarps = (static_cast<unsigned long long>(gridDim.x) * blockDim.x) >> 5;
  for (unsigned long long w = (blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x) >> 5;
       w < nhead; w += nwarps) {
    const unsigned long long q = surv[w];
    const int row = static_cast<int>(q >> 32), t2 = static_cast<int>(q & 0xffffffffull);
    const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
    const long long base1 = (static_cast<long long>(map1[slot]) * g1.ntiles + t1) * n1;
    const long long base2 = (static_cast<long long>(map2[slot]) * g2.ntiles + t2) * n2;
    const int ty1 = t1 / g1.tw, tx1 = t1 - ty1 * g1.tw, ty2 = t2 / g2.tw, tx2 = t2 - ty2 * g2.tw;
    const int nv1 = min(te1, g1.W - ty1 * te1), nu1 = min(te1, g1.W - tx1 * te1);
    const int nv2 = min(te2, g2.W - ty2 * te2), nu2 = min(te2, g2.W - tx2 * te2);
    const int ja = lane, jb = lane + 32;
    const int ja_v = ja / te2, ja_u = ja - ja_v * te2, jb_v = jb / te2, jb_u = jb - jb_v * te2;
    const bool va = ja < n2 && ja_v < nv2 && ja_u < nu2;
    const bool vb = jb < n2 && jb_v < nv2 && jb_u < nu2;
    const Vec4<T> c2a = va ? b.center[base2 + ja] : far4;
    const Vec4<T> c2b = vb ? b.center[base2 + jb] : far4;
    const Vec4<T> c1a = ja < n1 ? a.center[base1 + ja] : far4;
    const Vec4<T> c1b = jb < n1 ? a.center[base1 + jb] : far4;
    const unsigned taub = *reinterpret_cast<volatile unsigned *>(&stats->tau_bits);
    const T tau = thr_compare<T, S>(taub, e);
    T L[KL];
#pragma unroll
    for (int q2 = 0; q2 < KL; ++q2) L[q2] = pos_inf<T>();
    for (int a1 = 0; a1 < nv1; ++a1) {
      for (int b1 = 0; b1 < nu1; ++b1) {
        const int l1 = a1 * te1 + b1;
        const Vec4<T> c1 = shfl_vec(l1 < 32 ? c1a : c1b, l1 & 31);
        const T d[2] = {pair_d2<T, S>(c1, c2a), pair_d2<T, S>(c1, c2b)};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const T x = d[h];
          if (x < L[KL - 1] && x <= tau) {
#pragma unroll
            for (int q2 = KL - 1; q2 >= 1; --q2) L[q2] = (x < L[q2 - 1]) ? L[q2 - 1] : ((x < L[q2]) ? x : L[q2]);
            L[0] = (x < L[0]) ? x : L[0];
          }
        }
      }
    }
    // k rounds of warp minimum over the list heads; the owner pops its head.
    T kth = pos_inf<T>();
    for (int r = 0; r < k; ++r) {
      T m = L[0];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = tmin(m, __shfl_xor_sync(kFull, m, o));
      const unsigned owner = __ballot_sync(kFull, L[0] == m);
      if (lane == __ffs(owner) - 1) {
#pragma unroll
        for (int q2 = 0; q2 < KL - 1; ++q2) L[q2] = L[q2 + 1];
        L[KL - 1] = pos_inf<T>();
      }
      kth = m;
    }
    if (lane == 0 && kth != pos_inf<T>()) atomicMin(&stats->tau_bits, thr_bits<T, S>(kth, e));
  }
}

// ---- supertile level ------------------------------------------------------

// Bounds of every supertile (8 x 8 tiles): one warp reduces its <= 64 tiles.
template <typename T>
__global__ void k_supertiles(SideRound<T> sr, long long qs) {
  sr = qsh(sr, qoff(qs));
  const Geom g = sr.g;
  const int lane = threadIdx.x & 31;
  const long long total = static_cast<long long>(nreg_of(sr)) * g.nst;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long w = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; w < total; w += nwarps) {
    const int r = static_cast<int>(w / g.nst), st = static_cast<int>(w - static_cast<long long>(r) * g.nst);
    const int sy = st / g.stw, sx = st - (st / g.stw) * g.stw;
    T lo[3] = {pos_inf<T>(), pos_inf<T>(), pos_inf<T>()};
    T hi[3] = {-pos_inf<T>(), -pos_inf<T>(), -pos_inf<T>()};
    for (int l = lane; l < kMaxTile * kMaxTile; l += 32) {
      const int ty = sy * kMaxTile + l / kMaxTile, tx = sx * kMaxTile + l % kMaxTile;
      if (ty < g.tw && tx < g.tw) {
        const long long t = static_cast<long long>(r) * g.ntiles + ty * g.tw + tx;
        const Vec4<T> a = sr.tlo[t], b = sr.thi[t];
        lo[0] = tmin(lo[0], a.x);
        lo[1] = tmin(lo[1], a.y);
        lo[2] = tmin(lo[2], a.z);
        hi[0] = tmax(hi[0], b.x);
        hi[1] = tmax(hi[1], b.y);
        hi[2] = tmax(hi[2], b.z);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = tmin(lo[c], __shfl_xor_sync(kFull, lo[c], o));
        hi[c] = tmax(hi[c], __shfl_xor_sync(kFull, hi[c], o));
      }
    }
    if (lane == 0) {
      sr.stlo[w] = Vec4<T>{lo[0], lo[1], lo[2], T(0)};
      sr.sthi[w] = Vec4<T>{hi[0], hi[1], hi[2], T(0)};
    }
  }
}

// Representative cell of a supertile: the representative of its middle tile.
__device__ __forceinline__ long long super_rep(int r, int st, const Geom &g) {
  const int sy = st / g.stw, sx = st - (st / g.stw) * g.stw;
  const int nty = min(kMaxTile, g.tw - sy * kMaxTile), ntx = min(kMaxTile, g.tw - sx * kMaxTile);
  const int t = (sy * kMaxTile + nty / 2) * g.tw + sx * kMaxTile + ntx / 2;
  return (static_cast<long long>(r) * g.ntiles + t) * (g.te * g.te) + tile_rep(t, g);
}

// The warp's 32 values sorted ascending across the lanes (bitonic network):
// lane i receives the i-th smallest.
template <typename T>
__device__ __forceinline__ T warp_sort_asc(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const T o = __shfl_xor_sync(kFull, v, stride);
      const bool asc = (lane & size) == 0 || size == 32;
      const bool low = (lane & stride) == 0;
      v = (low == asc) ? (o < v ? o : v) : (o < v ? v : o);
    }
  }
  return v;
}

// Representative cell of a supertile's tile (ry, rx) of an R x R grid of
// representatives, R clamped to the supertile's own tile counts so that the
// representatives are distinct tiles (ragged supertiles at the grid's edge).
__device__ __forceinline__ long long super_rep_at(int r, int st, const Geom &g, int R, int ry, int rx, bool &valid) {
  const int sy = st / g.stw, sx = st - (st / g.stw) * g.stw;
  const int nty = min(kMaxTile, g.tw - sy * kMaxTile), ntx = min(kMaxTile, g.tw - sx * kMaxTile);
  const int Ry = min(R, nty), Rx = min(R, ntx);
  valid = ry < Ry && rx < Rx;
  const int ty = (2 * ry + 1) * nty / (2 * Ry), tx = (2 * rx + 1) * ntx / (2 * Rx);
  const int t = (sy * kMaxTile + min(ty, nty - 1)) * g.tw + sx * kMaxTile + min(tx, ntx - 1);
  return (static_cast<long long>(r) * g.ntiles + t) * (g.te * g.te) + tile_rep(t, g);
}

// Threshold seed of the two-level screen.  k <= kStKL: each supertile
// contributes an R x R grid of representative cells (R = kStR), and each
// lane keeps the k smallest representative-pair d2 it computes in a sorted
// register list; every warp folds the exact k-th of its lanes' lists (k
// distinct cell pairs) into tau.  Larger k: one representative per
// supertile and the block k-th of thread minima.
constexpr int kStR = 2;
constexpr int kStKL = 8;

template <typename T, bool S>
__global__ void __launch_bounds__(256) k_dist_tau_st(SideRound<T> a, SideRound<T> b, const int *map1,
                                                     const int *map2, int nslots, int k, ScreenStats *stats, float e,
                                                     long long qs) {
  __shared__ unsigned sh[256];
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  nslots = nslots_of(nslots, stats);
  const Geom g1 = a.g, g2 = b.g;
  const int nrows = nslots * g1.nst;
  if (k > kStKL) {
    T best = pos_inf<T>();  // smallest pair d2; thr_bits is monotone, so it is applied once per fold
    for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
      const int slot = row / g1.nst, s1 = row - slot * g1.nst;
      const Vec4<T> c1 = a.center[super_rep(map1[slot], s1, g1)];
      for (int s2 = threadIdx.x; s2 < g2.nst; s2 += blockDim.x) {
        const Vec4<T> c2 = b.center[super_rep(map2[slot], s2, g2)];
        best = tmin(best, pair_d2<T, S>(c1, c2));
      }
    }
    fold_tau(thr_bits<T, S>(best, e), k, &stats->tau_bits, sh);
    return;
  }
  constexpr int R2 = kStR * kStR;
  const Vec4<T> far4{pos_inf<T>(), pos_inf<T>(), pos_inf<T>(), T(0)};
  T L[kStKL];
#pragma unroll
  for (int q = 0; q < kStKL; ++q) L[q] = pos_inf<T>();
  // Supertile pairs (row, s2) over every thread of the query's blocks.
  const long long npairs = static_cast<long long>(nrows) * g2.nst;
  for (long long pr = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; pr < npairs;
       pr += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int row = static_cast<int>(pr / g2.nst), s2 = static_cast<int>(pr - static_cast<long long>(row) * g2.nst);
    const int slot = row / g1.nst, s1 = row - slot * g1.nst;
    Vec4<T> c1[R2];
#pragma unroll
    for (int i = 0; i < R2; ++i) {
      bool v;
      const long long idx = super_rep_at(map1[slot], s1, g1, kStR, i / kStR, i % kStR, v);
      c1[i] = v ? a.center[idx] : far4;
    }
#pragma unroll
    for (int j = 0; j < R2; ++j) {
      bool v;
      const long long idx = super_rep_at(map2[slot], s2, g2, kStR, j / kStR, j % kStR, v);
      if (!v) continue;
      const Vec4<T> c2 = b.center[idx];
#pragma unroll
      for (int i = 0; i < R2; ++i) {
        const T x = pair_d2<T, S>(c1[i], c2);  // +inf for an absent representative
        if (x < L[kStKL - 1]) {
#pragma unroll
          for (int q = kStKL - 1; q >= 1; --q) L[q] = (x < L[q - 1]) ? L[q - 1] : ((x < L[q]) ? x : L[q]);
          L[0] = (x < L[0]) ? x : L[0];
        }
      }
    }
  }
  // Block merge: each warp pops its k smallest (k rounds of warp minimum
  // over the list heads) into shared memory; warp 0 takes the exact k-th of
  // the block's 8 x k values (two sorted halves of 32, then the k smallest
  // of their first 16 each) and folds it.
  __shared__ T s_top[8 * kStKL];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int r = 0; r < kStKL; ++r) {
    T m = L[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = tmin(m, __shfl_xor_sync(kFull, m, o));
    const unsigned owner = __ballot_sync(kFull, L[0] == m);
    if (lane == __ffs(owner) - 1) {
#pragma unroll
      for (int q = 0; q < kStKL - 1; ++q) L[q] = L[q + 1];
      L[kStKL - 1] = pos_inf<T>();
    }
    if (lane == 0) s_top[warp * kStKL + r] = r < k ? m : pos_inf<T>();
  }
  __syncthreads();
  if (warp == 0) {
    const T s0 = warp_sort_asc(s_top[lane]), s1 = warp_sort_asc(s_top[lane + 32]);
    const T y0 = __shfl_sync(kFull, s0, lane & 15), y1 = __shfl_sync(kFull, s1, lane & 15);
    const T kth = __shfl_sync(kFull, warp_sort_asc(lane < 16 ? y0 : y1), k - 1);
    if (lane == 0 && kth != pos_inf<T>()) atomicMin(&stats->tau_bits, thr_bits<T, S>(kth, e));
  }
}

template <typename T, bool S>
__global__ void k_dist_cull_st(SideRound<T> a, SideRound<T> b, const int *map1, const int *map2, int nslots,
                               unsigned long long *surv, unsigned long long cap, ScreenStats *stats, float e,
                               long long qs) {
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  surv = qsh(surv, qo);
  nslots = nslots_of(nslots, stats);
  const Geom g1 = a.g, g2 = b.g;
  const int nrows = nslots * g1.nst;
  const T tau = thr_compare<T, S>(stats->tau_bits, e);
  for (int row = blockIdx.x; row < nrows; row += gridDim.x) {
    const int slot = row / g1.nst, s1 = row - slot * g1.nst;
    const long long i1 = static_cast<long long>(map1[slot]) * g1.nst + s1;
    Vec4<T> lo1, hi1;
    st_bounds(a, i1, lo1, hi1);
    const long long base2 = static_cast<long long>(map2[slot]) * g2.nst;
    for (int s0 = 0; s0 < g2.nst; s0 += blockDim.x) {
      const int s2 = s0 + threadIdx.x;
      bool keep = false;
      if (s2 < g2.nst) {
        Vec4<T> lo2, hi2;
        st_bounds(b, base2 + s2, lo2, hi2);
        T lb = tile_lb(lo1, hi1, lo2, hi2);
        if constexpr (S) lb = __fmul_rd(lb, 1.0f - 0x1p-19f);
        keep = lb <= tau;
      }
      const long long pos = warp_append(keep, &stats->st_survivors);
      if (pos >= 0 && static_cast<unsigned long long>(pos) < cap)
        surv[pos] = pack_tile_pair(static_cast<unsigned>(row), static_cast<unsigned>(s2));
    }
  }
}

// Surviving supertile pairs expanded into their <= 64 x 64 child tile pairs,
// one warp per supertile pair.  Each side's child tiles are first tested
// against the other supertile's box: a tile box lies inside its supertile's
// box and the rounded gap is monotone, so lb(t1, t2) >= lb(t1, S2) and a tile
// that fails against the box fails against every tile inside it.  Only the
// surviving children are crossed.
// cull = 0: fold the representative distances into tau (each warp folds the
// k-th of its lanes' minima after every supertile pair, so the pre-filter of
// the next one already uses the tighter value); cull = 1: append the tile
// pairs whose bound passes tau, with the bound as sort key (the same format
// k_dist_cull writes).
template <typename T, bool S>
__device__ __forceinline__ T shaved_lb(const Vec4<T> &lo1, const Vec4<T> &hi1, const Vec4<T> &lo2, const Vec4<T> &hi2) {
  T lb = tile_lb(lo1, hi1, lo2, hi2);
  // The screen's pair distances are FMA-contracted: shave the rounded bound
  // by 2^-19 (more than the 12u they can differ by).
  if constexpr (S) lb = __fmul_rd(lb, 1.0f - 0x1p-19f);
  return lb;
}

template <typename T, bool S>
__global__ void __launch_bounds__(128) k_dist_expand(SideRound<T> a, SideRound<T> b, const int *map1,
                                                     const int *map2, const unsigned long long *st_surv,
                                                     unsigned long long nst_surv, unsigned long long st_cap, int k,
                                                     int cull, unsigned long long *surv, unsigned *surv_lb,
                                                     unsigned long long cap, ScreenStats *stats, float e,
                                                     long long qs) {
  // One warp per supertile pair, warp-synchronous throughout (no block
  // barrier inside the loop), so a block keeps four pairs in flight.  The
  // surviving children of each side, with the data the crossing needs (the
  // representative centre, or the tile box), sit in the warp's shared lists.
  constexpr int kW = 4, kC = kMaxTile * kMaxTile;
  __shared__ unsigned sh[256];
  __shared__ int s_t[kW][2][kC];
  __shared__ Vec4<T> s_p[kW][2][kC];  // representative centre (cull = 0) or tile lo (cull = 1)
  __shared__ Vec4<T> s_q[kW][2][kC];  // tile hi (cull = 1)
  const long long qo = qoff(qs);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  stats = qsh(stats, qo);
  st_surv = qsh(st_surv, qo);
  surv = qsh(surv, qo);
  surv_lb = qsh(surv_lb, qo);
  nst_surv = count_of(nst_surv, stats->st_survivors, st_cap);
  const Geom g1 = a.g, g2 = b.g;
  const int n1 = g1.te * g1.te, n2 = g2.te * g2.te;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  T best = pos_inf<T>();  // smallest pair d2; thr_bits is monotone, so it is applied once per fold
  for (unsigned long long w = static_cast<unsigned long long>(blockIdx.x) * kW + warp; w < nst_surv;
       w += static_cast<unsigned long long>(gridDim.x) * kW) {
    const unsigned long long q = st_surv[w];
    const int row = static_cast<int>(q >> 32), s2 = static_cast<int>(q & 0xffffffffull);
    const int slot = row / g1.nst, s1 = row - slot * g1.nst;
    const int r1 = map1[slot], r2 = map2[slot];
    const unsigned taub = *reinterpret_cast<volatile unsigned *>(&stats->tau_bits);
    const T tau = thr_compare<T, S>(taub, e);
    Vec4<T> slo1, shi1, slo2, shi2;
    st_bounds(a, static_cast<long long>(r1) * g1.nst + s1, slo1, shi1);
    st_bounds(b, static_cast<long long>(r2) * g2.nst + s2, slo2, shi2);
    // Children of each side tested against the other supertile's box,
    // compacted in lane order.
    int m[2];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const SideRound<T> &X = side ? b : a;
      const Geom &g = side ? g2 : g1;
      const int sidx = side ? s2 : s1, r = side ? r2 : r1;
      const int sy = sidx / g.stw, sx = sidx - sy * g.stw;
      int base = 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int l = lane + 32 * h;
        const int ty = sy * kMaxTile + (l >> 3), tx = sx * kMaxTile + (l & 7);
        const bool valid = ty < g.tw && tx < g.tw;
        const int t = valid ? ty * g.tw + tx : 0;
        const long long i = static_cast<long long>(r) * g.ntiles + t;
        Vec4<T> lo{}, hi{};
        bool ok = false;
        if (valid) {
          lo = X.tlo[i];
          hi = X.thi[i];
          ok = (side ? shaved_lb<T, S>(slo1, shi1, lo, hi) : shaved_lb<T, S>(lo, hi, slo2, shi2)) <= tau;
        }
        const unsigned mask = __ballot_sync(kFull, ok);
        if (ok) {
          const int pos = base + __popc(mask & lt);
          s_t[warp][side][pos] = t;
          if (!cull) {
            s_p[warp][side][pos] = X.center[i * (side ? n2 : n1) + tile_rep(t, g)];
          } else {
            s_p[warp][side][pos] = lo;
            s_q[warp][side][pos] = hi;
          }
        }
        base += __popc(mask);
      }
      m[side] = base;
    }
    __syncwarp();
    const int m1 = m[0], m2 = m[1], total = m1 * m2;
    // c -> (c / m2, c % m2) through a float reciprocal: c < 2^12 and m2 <= 64
    // keep the rounded quotient within 2^-10 of the true one, whose fraction
    // lies in [1/128, 1 - 1/128], so the truncation is exact.
    const float inv = total > 0 ? 1.0f / static_cast<float>(m2) : 0.0f;
    for (int c0 = 0; c0 < total; c0 += 32) {
      const int c = c0 + lane;
      bool keep = false;
      T lb = T(0);
      int i1 = 0, i2 = 0;
      if (c < total) {
        i1 = __float2int_rz((static_cast<float>(c) + 0.5f) * inv);
        i2 = c - i1 * m2;
        if (!cull) {
          best = tmin(best, pair_d2<T, S>(s_p[warp][0][i1], s_p[warp][1][i2]));
        } else {
          lb = shaved_lb<T, S>(s_p[warp][0][i1], s_q[warp][0][i1], s_p[warp][1][i2], s_q[warp][1][i2]);
          keep = lb <= tau;
        }
      }
      if (cull) {
        const long long pos = warp_append(keep, &stats->survivors);
        if (pos >= 0 && static_cast<unsigned long long>(pos) < cap) {
          surv[pos] = pack_tile_pair(static_cast<unsigned>(slot * g1.ntiles + s_t[warp][0][i1]),
                                     static_cast<unsigned>(s_t[warp][1][i2]));
          surv_lb[pos] = lb_bits_down(lb);
        }
      }
    }
    if (lane == 0 && total > 0) atomicAdd(&stats->tile_pairs, static_cast<unsigned long long>(total));
    if (!cull && k <= 32) {
      const unsigned mine = thr_bits<T, S>(best, e);
      if (__popc(__ballot_sync(kFull, mine < taub)) >= k) {
        const unsigned kth = warp_sorted_at(mine, k - 1);
        if (lane == 0) atomicMin(&stats->tau_bits, kth);
      }
    }
    __syncwarp();
  }
  if (!cull && k > 32) fold_tau(thr_bits<T, S>(best, e), k, &stats->tau_bits, sh);
}

// Total order of the top-k (distance_analysis.cu:226-231).
template <typename T>
__device__ __forceinline__ bool cand_less(const DistCand<T> &x, const DistCand<T> &y) {
  if (x.d2 != y.d2) return x.d2 < y.d2;
  if (x.slot != y.slot) return x.slot < y.slot;
  if (x.i != y.i) return x.i < y.i;
  return x.j < y.j;
}

// Exact k smallest candidates under the total order, one block of 1024.
template <typename T>
__global__ void __launch_bounds__(1024) k_dist_select(const DistCand<T> *cand, unsigned long long cand_cap, int k,
                                                      DistCand<T> *out, ScreenStats *stats, long long qs) {
  extern __shared__ unsigned char smem_raw[];
  const long long qo = qoff(qs);
  cand = qsh(cand, qo);
  out = qsh(out, qo);
  stats = qsh(stats, qo);
  DistCand<T> *buf = reinterpret_cast<DistCand<T> *>(smem_raw);
  __shared__ unsigned hist[256];
  __shared__ unsigned long long s_prefix, s_mask;
  __shared__ int s_need, s_count;
  const unsigned long long total = stats->candidates;
  if (total > cand_cap) {
    if (threadIdx.x == 0) stats->status = -4;
    return;
  }
  const int m = static_cast<int>(total);
  // Every pair with d2 <= (true k-th d2) was appended, and the final tau is
  // >= the true k-th d2: entries above tau can be dropped first.
  const T tau = tau_value<T>(stats->tau_bits);
  const unsigned long long tau_b = ordered_bits(tau);
  constexpr int kBits = sizeof(T) * 8;
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    const DistCand<T> c = cand[e];
    if (ordered_bits(c.d2) <= tau_b) {
      const int pos = atomicAdd(&s_count, 1);
      if (pos < kSelectCap) buf[pos] = c;
    }
  }
  __syncthreads();
  int cnt = s_count;
  if (cnt > kSelectCap) {
    // MSD radix select of the k-th smallest d2 among the entries <= tau
    // (non-negative values: the bits are ordered), then keep entries <= it.
    if (threadIdx.x == 0) {
      s_prefix = 0;
      s_mask = 0;
      s_need = k;
    }
    for (int shift = kBits - 8; shift >= 0; shift -= 8) {
      for (int q = threadIdx.x; q < 256; q += blockDim.x) hist[q] = 0;
      __syncthreads();
      const unsigned long long prefix = s_prefix, mask = s_mask;
      for (int e = threadIdx.x; e < m; e += blockDim.x) {
        const unsigned long long bits = ordered_bits(cand[e].d2);
        if (bits <= tau_b && (bits & mask) == prefix) atomicAdd(&hist[(bits >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int need = s_need;
        int dgt = 0;
        for (; dgt < 256; ++dgt) {
          if (static_cast<int>(hist[dgt]) >= need) break;
          need -= hist[dgt];
        }
        s_need = need;
        s_prefix = prefix | (static_cast<unsigned long long>(dgt) << shift);
        s_mask = mask | (255ull << shift);
      }
      __syncthreads();
    }
    const unsigned long long kth_bits = s_prefix;
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < m; e += blockDim.x) {
      const DistCand<T> c = cand[e];
      if (ordered_bits(c.d2) <= kth_bits) {
        const int pos = atomicAdd(&s_count, 1);
        if (pos < kSelectCap) buf[pos] = c;
      }
    }
    __syncthreads();
    cnt = s_count;
    if (cnt > kSelectCap) {
      // Too many exact ties at the k-th d2: among the tied entries, radix
      // select the needed number by the (slot, i, j) key, most significant
      // byte first, so the kept set is exactly the first k of the order.
      if (threadIdx.x == 0) s_count = 0;
      __syncthreads();
      for (int e = threadIdx.x; e < m; e += blockDim.x)
        if (ordered_bits(cand[e].d2) < kth_bits) atomicAdd(&s_count, 1);
      __syncthreads();
      const int below = s_count;
      __shared__ unsigned s_key[3], s_kmask[3];
      if (threadIdx.x == 0) {
        s_need = k - below;
        for (int w = 0; w < 3; ++w) s_key[w] = s_kmask[w] = 0u;
      }
      __syncthreads();
      for (int byte = 11; byte >= 0; --byte) {
        const int word = 2 - byte / 4, shift = (byte % 4) * 8;  // word 0 = slot, 1 = i, 2 = j
        for (int q = threadIdx.x; q < 256; q += blockDim.x) hist[q] = 0;
        __syncthreads();
        const unsigned k0 = s_key[0], k1 = s_key[1], k2 = s_key[2];
        const unsigned m0 = s_kmask[0], m1 = s_kmask[1], m2 = s_kmask[2];
        for (int e = threadIdx.x; e < m; e += blockDim.x) {
          const DistCand<T> c = cand[e];
          if (ordered_bits(c.d2) != kth_bits) continue;
          const unsigned w0 = static_cast<unsigned>(c.slot), w1 = static_cast<unsigned>(c.i),
                         w2 = static_cast<unsigned>(c.j);
          if ((w0 & m0) != k0 || (w1 & m1) != k1 || (w2 & m2) != k2) continue;
          const unsigned wv = word == 0 ? w0 : (word == 1 ? w1 : w2);
          atomicAdd(&hist[(wv >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          int need = s_need, dgt = 0;
          for (; dgt < 256; ++dgt) {
            if (static_cast<int>(hist[dgt]) >= need) break;
            need -= hist[dgt];
          }
          s_need = need;
          s_key[word] |= static_cast<unsigned>(dgt) << shift;
          s_kmask[word] |= 255u << shift;
        }
        __syncthreads();
      }
      const unsigned K0 = s_key[0], K1 = s_key[1], K2 = s_key[2];
      if (threadIdx.x == 0) s_count = 0;
      __syncthreads();
      for (int e = threadIdx.x; e < m; e += blockDim.x) {
        const DistCand<T> c = cand[e];
        const unsigned long long b = ordered_bits(c.d2);
        bool take = b < kth_bits;
        if (b == kth_bits) {
          const unsigned w0 = static_cast<unsigned>(c.slot), w1 = static_cast<unsigned>(c.i),
                         w2 = static_cast<unsigned>(c.j);
          take = w0 < K0 || (w0 == K0 && (w1 < K1 || (w1 == K1 && w2 <= K2)));
        }
        if (take) {
          const int pos = atomicAdd(&s_count, 1);
          if (pos < kSelectCap) buf[pos] = c;
        }
      }
      __syncthreads();
      cnt = s_count;
      if (cnt > kSelectCap) {
        if (threadIdx.x == 0) stats->status = -4;
        return;
      }
    }
  }
  int n2 = 1;
  while (n2 < cnt) n2 <<= 1;
  for (int e = cnt + threadIdx.x; e < n2; e += blockDim.x) {
    DistCand<T> c;
    c.d2 = pos_inf<T>();
    c.slot = INT_MAX;
    c.i = INT_MAX;
    c.j = INT_MAX;
    buf[e] = c;
  }
  for (int size = 2; size <= n2; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const DistCand<T> x = buf[i], y = buf[j];
          if (cand_less(y, x) == up) {
            buf[i] = y;
            buf[j] = x;
          }
        }
      }
    }
  }
  __syncthreads();
  const int keep = cnt < k ? cnt : k;
  for (int e = threadIdx.x; e < keep; e += blockDim.x) out[e] = buf[e];
  if (threadIdx.x == 0) stats->nsel = keep;
}

// Child rectangle of cell bbox of a region sampled at nuv_parent:
// make_dist_refine_task / make_intersect_refine_task
// (distance_analysis.cu:340-354, intersection.cu:311-325).
template <typename T>
__device__ __forceinline__ RegionRec<T> child_rect(const RegionRec<T> &p, int nuv_parent, int bbox) {
  const T ustep = (p.u1 - p.u0) / static_cast<T>(nuv_parent);
  const T vstep = (p.v1 - p.v0) / static_cast<T>(nuv_parent);
  const int w = nuv_parent - 1;
  const int x = bbox % w, y = bbox / w;
  RegionRec<T> c;
  c.u0 = p.u0 + ustep * static_cast<T>(x);
  c.u1 = c.u0 + ustep;
  c.v0 = p.v0 + vstep * static_cast<T>(y);
  c.v1 = c.v0 + vstep;
  return c;
}

// Child rectangle of a cell on the covering grid (bounds mode): exactly the
// parameters its corner samples were taken at (k_basis, cover = 1).
template <typename T>
__device__ __forceinline__ RegionRec<T> child_rect_cover(const RegionRec<T> &p, int nuv_parent, int bbox) {
  const T ustep = (p.u1 - p.u0) / static_cast<T>(nuv_parent - 1);
  const T vstep = (p.v1 - p.v0) / static_cast<T>(nuv_parent - 1);
  const int w = nuv_parent - 1;
  const int x = bbox % w, y = bbox / w;
  RegionRec<T> c;
  c.u0 = ustep * static_cast<T>(x) + p.u0;
  c.u1 = x + 1 == w ? p.u1 : ustep * static_cast<T>(x + 1) + p.u0;
  c.v0 = vstep * static_cast<T>(y) + p.v0;
  c.v1 = y + 1 == w ? p.v1 : vstep * static_cast<T>(y + 1) + p.v0;
  return c;
}

// Pair-preserving refinement jobs with (slot, cell) dedup per side
// (distance_analysis.cu:399-491): one block.
template <typename T>
__global__ void __launch_bounds__(1024) k_dist_next(const DistCand<T> *top, ScreenStats *stats, SideRound<T> a,
                                                    SideRound<T> b, const int *map1, const int *map2, int nuv_next,
                                                    RegionRec<T> *next1, RegionRec<T> *next2, int *nmap1, int *nmap2,
                                                    long long qs) {
  __shared__ int first1[kMaxK], first2[kMaxK];
  __shared__ int uid1[kMaxK], uid2[kMaxK];
  const long long qo = qoff(qs);
  top = qsh(top, qo);
  stats = qsh(stats, qo);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  next1 = qsh(next1, qo);
  next2 = qsh(next2, qo);
  nmap1 = qsh(nmap1, qo);
  nmap2 = qsh(nmap2, qo);
  const int n = stats->nsel;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const DistCand<T> c = top[e];
    int f1 = 1, f2 = 1;
    for (int q = 0; q < e; ++q) {
      const DistCand<T> o = top[q];
      if (o.slot == c.slot && o.i == c.i) f1 = 0;
      if (o.slot == c.slot && o.j == c.j) f2 = 0;
    }
    first1[e] = f1;
    first2[e] = f2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int c1 = 0, c2 = 0;
    for (int e = 0; e < n; ++e) {
      uid1[e] = first1[e] ? c1++ : -1;
      uid2[e] = first2[e] ? c2++ : -1;
    }
    stats->nreg1 = c1;
    stats->nreg2 = c2;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const DistCand<T> c = top[e];
    int u1 = uid1[e], u2 = uid2[e];
    if (u1 < 0) {
      for (int q = 0; q < e; ++q)
        if (top[q].slot == c.slot && top[q].i == c.i) {
          u1 = uid1[q];
          break;
        }
    } else {
      next1[u1] = child_rect(a.regions[map1[c.slot]], a.g.nuv, c.i);
    }
    if (u2 < 0) {
      for (int q = 0; q < e; ++q)
        if (top[q].slot == c.slot && top[q].j == c.j) {
          u2 = uid2[q];
          break;
        }
    } else {
      next2[u2] = child_rect(b.regions[map2[c.slot]], b.g.nuv, c.j);
    }
    nmap1[e] = u1;
    nmap2[e] = u2;
  }
  (void)nuv_next;
}

// ---- batched distance: round bookkeeping and the threshold-pass list -------

// End of a batched round, one warp per query: the round's counters, status
// and kept pairs go to the query's record; the kept count becomes the next
// round's slot count (0 after a failure, which idles the query's later
// rounds); the counters restart unless this was the last round.
template <typename TP>
__global__ void k_dist_close(ScreenStats *stats, const DistCand<TP> *top, DistRecord<TP> *rec, int round,
                             unsigned long long surv_cap, unsigned long long cand_cap, int last, long long qs) {
  const long long qo = qoff(qs);
  stats = qsh(stats, qo);
  top = qsh(top, qo);
  rec = qsh(rec, qo);
  const int t = threadIdx.x;
  int st = stats->status;
  if (st == 0 && (stats->survivors > surv_cap || stats->candidates > cand_cap)) st = kStatusCapacity;
  const int n = st == 0 ? stats->nsel : 0;
  if (t < n && t < kBatchK) rec->top[round][t] = top[t];
  const unsigned long long tests = stats->pair_tests, cands = stats->candidates, surv = stats->survivors;
  const unsigned long long examined = stats->tile_pairs, st_kept = stats->st_survivors;
  __syncwarp();
  if (t == 0) {
    rec->tests[round] = static_cast<long long>(tests);
    rec->cands[round] = static_cast<long long>(cands);
    rec->survivors[round] = surv;
    rec->examined[round] = examined;
    rec->st_kept[round] = st_kept;
    rec->npairs[round] = n;
    rec->status[round] = st;
    stats->nslots = n;
    if (!last) {
      stats->tile_pairs = 0;
      stats->survivors = 0;
      stats->pair_tests = 0;
      stats->candidates = 0;
      stats->tau_bits = 0x7f800000u;
      stats->status = 0;
      stats->nsel = 0;
      stats->work = 0;
      stats->st_survivors = 0;
      stats->nhead = 0;
    }
  }
}

// ---- batched distance: every refinement round of a query in one block -------
//
// One block of kRefineThreads per query runs rounds first..last back to back
// (a round needs only the query's own previous round).  Per round:
//  * the regions of both sides (at most kBatchK each) are evaluated: basis
//    and span of each sample row and column as k_basis computes them (values
//    only) and every sample by eval_point (the factored cell kernels produce
//    the same bits) in shared memory, every cell centre from its four
//    corners as k_cells_fused forms it into the round's centre arrays in the
//    query's slab (L1 / L2-resident), and the centre range of each 4 x 4
//    tile;
//  * the exact k smallest pairs under the order (d2, slot, i, j) over every
//    slot's cell pairs: each lane keeps its own kBatchK smallest in sorted
//    registers (the k smallest overall are among the kBatchK smallest of the
//    lane that examined them).  Every tile pair gets its box-gap bound; each
//    slot's tile pair with the smallest bound is examined first (a warp per
//    slot) and they are merged to their exact k-th, tau; a tile pair whose
//    bound exceeds tau
//    holds no pair of the k smallest (every pair's d2 is at least its tile
//    pair's rounded gap), the others are examined, and a final merge gives
//    the k smallest.  Tiles of 4 x 4 cells keep the examined pairs near the
//    pairs that matter when the two patches run nearly parallel;
//  * the next round's regions with (slot, cell) dedup per side, as
//    k_dist_next, and the round's record and counters, as k_dist_close
//    (tests = cell pairs examined, cands = lane-list entries, survivors =
//    tile pairs examined, examined = tile pairs bounded).
constexpr int kRefCells = (kRefineNuv - 1) * (kRefineNuv - 1);
constexpr int kRefRegs = 2 * kBatchK;
constexpr int kRefTe = 4;                                   // tile edge (cells)
constexpr int kRefTw = (kRefineNuv - 1 + kRefTe - 1) / kRefTe;
constexpr int kRefTiles = kRefTw * kRefTw;
constexpr int kRefPairs = kBatchK * kRefTiles * kRefTiles;  // tile pairs of a round at most
constexpr int kRefineWarps = kRefineThreads / 32;
constexpr int kRefMerge = kRefineWarps * kBatchK;
constexpr int kRefRows = 6;  // control-net rows a sample column's u sums hold in registers
static_assert(kRefCells <= 256 && kBatchK <= 256, "cell and slot indices are packed in 8 bits each");
static_assert(kRefineNuv * kRefineNuv <= kRefineThreads, "one basis line per thread");
static_assert(kRefTe * kRefTe == 16, "a half warp per tile");
static_assert(kRefineWarps >= kBatchK, "a warp per slot picks the slot's first tile pair");

template <typename T, int MAXP>
struct RefineSmem {
  T tb[kRefRegs * kRefTiles][6];    // tile centre ranges: lo xyz, hi xyz
  T smp[3][kBatchK * kRefineNuv * kRefineNuv];  // one side's samples
  T nb[kBatchK][2][kRefineNuv][MAXP];            // basis values of sample columns (0) and rows (1)
  T tplb[kRefPairs];                // box-gap bound of each tile pair
  unsigned short tpl[kRefPairs];    // tile pairs left to examine after the head
  unsigned headmask[kRefPairs / 32];
  unsigned long long mob[kRefMerge];
  int mkey[kRefMerge];
  unsigned long long tob[kBatchK];  // the k smallest: ordered d2 bits and packed (slot, i, j)
  int tkey[kBatchK];
  int head[kRefineWarps];
  int sp[kBatchK][2][kRefineNuv];
  int map1[kBatchK], map2[kBatchK];
  unsigned long long tests, cands, surv;
  int n, ntpl;
};

template <typename T, int MAXP>
constexpr size_t refine_smem() {
  return sizeof(RefineSmem<T, MAXP>);
}

constexpr unsigned long long kRefPadOb = ~0ull;
constexpr int kRefPadKey = INT_MAX;

__device__ __forceinline__ bool ref_less(unsigned long long ao, int ak, unsigned long long bo, int bk) {
  return ao < bo || (ao == bo && ak < bk);
}

// Sorted insert into a lane's list of the kBatchK smallest entries.
__device__ __forceinline__ void ref_insert(unsigned long long (&lo)[kBatchK], int (&lk)[kBatchK],
                                           unsigned long long o, int key) {
  if (!ref_less(o, key, lo[kBatchK - 1], lk[kBatchK - 1])) return;
  lo[kBatchK - 1] = o;
  lk[kBatchK - 1] = key;
#pragma unroll
  for (int j = kBatchK - 1; j > 0; --j) {
    if (ref_less(lo[j], lk[j], lo[j - 1], lk[j - 1])) {
      const unsigned long long to = lo[j];
      lo[j] = lo[j - 1];
      lo[j - 1] = to;
      const int tk = lk[j];
      lk[j] = lk[j - 1];
      lk[j - 1] = tk;
    }
  }
}

// The k smallest entries of all lane lists of the block into sm.tob / tkey
// and their count into sm.n (every thread calls it; the lists are kept).
template <typename SM>
__device__ void ref_merge(SM &sm, const unsigned long long (&lo)[kBatchK], const int (&lk)[kBatchK], int k) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  unsigned long long co[kBatchK];
  int ck[kBatchK];
#pragma unroll
  for (int j = 0; j < kBatchK; ++j) {
    co[j] = lo[j];
    ck[j] = lk[j];
  }
  // Each warp's k smallest, one per step: the lane holding the warp's
  // smallest head drops it.
  for (int it = 0; it < kBatchK; ++it) {
    unsigned long long bo = co[0];
    int bk = ck[0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long oo = __shfl_xor_sync(kFull, bo, o);
      const int ok = __shfl_xor_sync(kFull, bk, o);
      if (ref_less(oo, ok, bo, bk)) {
        bo = oo;
        bk = ok;
      }
    }
    if (lane == 0) {
      sm.mob[w * kBatchK + it] = it < k ? bo : kRefPadOb;
      sm.mkey[w * kBatchK + it] = it < k ? bk : kRefPadKey;
    }
    // The lane holding the warp's smallest drops it (entries are unique;
    // lanes whose head is padding equal to it drop padding).
    if (co[0] == bo && ck[0] == bk) {
#pragma unroll
      for (int j = 0; j < kBatchK - 1; ++j) {
        co[j] = co[j + 1];
        ck[j] = ck[j + 1];
      }
      co[kBatchK - 1] = kRefPadOb;
      ck[kBatchK - 1] = kRefPadKey;
    }
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < kRefMerge) {
    const unsigned long long o = sm.mob[t];
    const int kk = sm.mkey[t];
    if (!(o == kRefPadOb && kk == kRefPadKey)) {
      int rank = 0;
      for (int e = 0; e < kRefMerge; ++e) rank += ref_less(sm.mob[e], sm.mkey[e], o, kk) ? 1 : 0;
      if (rank < k) {
        sm.tob[rank] = o;
        sm.tkey[rank] = kk;
      }
    }
  }
  if (t == 0) {
    int cnt = 0;
    for (int e = 0; e < kRefMerge; ++e) cnt += (sm.mob[e] == kRefPadOb && sm.mkey[e] == kRefPadKey) ? 0 : 1;
    sm.n = cnt < k ? cnt : k;
  }
  __syncthreads();
}


// Every region of one side into shared-memory slots off..off + nreg - 1, in
// four block-wide phases (basis rows, samples, cell centres, tile ranges),
// each spread over all threads.  Every thread calls it.
template <typename T, int MAXP, typename SM>
__device__ void ref_side(SM &sm, const SurfView<T> &s, const RegionRec<T> *regs, int nreg, int nuv, int off,
                         Vec4<T> *cen) {
  const int t = threadIdx.x, W = nuv - 1, tw = (W + kRefTe - 1) / kRefTe, nt = tw * tw;
  const int nl = 2 * nuv, ns = nuv * nuv, nc = W * W;
  for (int idx = t; idx < nreg * nl; idx += kRefineThreads) {
    // u = ((ustop - ustart) / nuv) * idx + ustart, as k_basis (no cover)
    const int r = idx / nl, rem = idx - r * nl, dir = rem >= nuv ? 1 : 0, q = dir ? rem - nuv : rem;
    const RegionRec<T> reg = regs[r];
    const T lo = dir ? reg.v0 : reg.u0, hi = dir ? reg.v1 : reg.u1;
    const T step = (hi - lo) / static_cast<T>(nuv);
    const T x = step * static_cast<T>(q) + lo;
    const int p = dir ? s.degv : s.degu;
    T *out = sm.nb[r][dir][q];
    if (s.zero) {
      sm.sp[r][dir][q] = p;
      for (int j = 0; j < MAXP; ++j) out[j] = T(0);
    } else {
      // the basis routine also zeroes two derivative rows (stride MAXP)
      T tmp[3 * MAXP];
      const int span = find_span(dir ? s.nkv : s.nku, p, x, dir ? s.V : s.U);
      sm.sp[r][dir][q] = span;
      basis_ders_any<T, MAXP>(span, p, x, dir ? s.V : s.U, 0, tmp, MAXP);
      for (int j = 0; j <= p; ++j) out[j] = tmp[j];
    }
  }
  __syncthreads();
  // Samples, a thread per (region, sample column, part of its rows): the u
  // sums of the control-net rows those samples need, in registers, then
  // each sample's v combination.  Every u sum and v accumulation is the operation
  // sequence of eval_point (contract3 / contract4 and the quotient), so the
  // samples carry its bits; a column needing more than kRefRows net rows
  // evaluates its samples one by one.
  // A column's sample rows are split over `split` threads so that every
  // thread has work (each forms the u sums its own rows need).
  const int ncol = max(nreg * nuv, 1);
  const int split = max(1, min(nuv, kRefineThreads / ncol)), rows_per = (nuv + split - 1) / split;
  for (int idx = t; idx < ncol * split && nreg > 0; idx += kRefineThreads) {
    const int col = idx / split, part = idx - col * split;
    const int r = col / nuv, b = col - r * nuv;
    const int a_begin = part * rows_per, a_end = min(nuv, a_begin + rows_per);
    if (a_begin >= a_end) continue;
    int rmin = sm.sp[r][1][a_begin], rmax = rmin;
    for (int a = a_begin + 1; a < a_end; ++a) {
      rmin = min(rmin, sm.sp[r][1][a]);
      rmax = max(rmax, sm.sp[r][1][a]);
    }
    rmin -= s.degv;
    const int nrows = rmax - rmin + 1;
    if (s.zero || nrows > kRefRows) {
      for (int a = a_begin; a < a_end; ++a) {
        T P[3];
        eval_point(s, sm.sp[r][0][b], sm.nb[r][0][b], sm.sp[r][1][a], sm.nb[r][1][a], P);
        sm.smp[0][r * ns + a * nuv + b] = P[0];
        sm.smp[1][r * ns + a * nuv + b] = P[1];
        sm.smp[2][r * ns + a * nuv + b] = P[2];
      }
      continue;
    }
    const T *Nu = sm.nb[r][0][b];
    const int cu0 = sm.sp[r][0][b] - s.degu;
    T rs[kRefRows][4];
#pragma unroll
    for (int R = 0; R < kRefRows; ++R) {
      T r0 = T(0), r1 = T(0), r2 = T(0), r3 = T(0);
      if (R < nrows) {
        const Vec4<T> *cp = s.cpw + static_cast<long long>(s.ncpu) * (rmin + R) + cu0;
        if (!s.rat) {
          for (int c = 0; c <= s.degu; ++c) {
            const Vec4<T> q = cp[c];
            const T n = Nu[c];
            r0 += n * q.x;
            r1 += n * q.y;
            r2 += n * q.z;
          }
        } else {
          for (int c = 0; c <= s.degu; ++c) {
            const Vec4<T> q = cp[c];
            const T nw = Nu[c] * q.w;
            r0 += nw * q.x;
            r1 += nw * q.y;
            r2 += nw * q.z;
            r3 += nw;
          }
        }
      }
      rs[R][0] = r0;
      rs[R][1] = r1;
      rs[R][2] = r2;
      rs[R][3] = r3;
    }
    for (int a = a_begin; a < a_end; ++a) {
      const T *Nv = sm.nb[r][1][a];
      const int R0 = sm.sp[r][1][a] - s.degv - rmin;
      T a0 = T(0), a1 = T(0), a2 = T(0), a3 = T(0);
#pragma unroll
      for (int R = 0; R < kRefRows; ++R) {
        const int rr = R - R0;
        if (rr >= 0 && rr <= s.degv) {
          const T m = Nv[rr];
          a0 += m * rs[R][0];
          a1 += m * rs[R][1];
          a2 += m * rs[R][2];
          a3 += m * rs[R][3];
        }
      }
      if (s.rat) {
        const T inv = T(1) / a3;
        a0 = a0 * inv;
        a1 = a1 * inv;
        a2 = a2 * inv;
      }
      sm.smp[0][r * ns + a * nuv + b] = a0;
      sm.smp[1][r * ns + a * nuv + b] = a1;
      sm.smp[2][r * ns + a * nuv + b] = a2;
    }
  }
  __syncthreads();
  for (int idx = t; idx < nreg * nc; idx += kRefineThreads) {
    const int r = idx / nc, l = idx - r * nc, a = l / W, b = l - (l / W) * W;
    const int i0 = r * ns + a * nuv + b, i1 = i0 + 1, i2 = i0 + nuv, i3 = i2 + 1;
    T m[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T *S = sm.smp[c];
      const T lo = fmn(S[i0], fmn(S[i1], fmn(S[i2], S[i3])));
      const T hi = fmx(S[i0], fmx(S[i1], fmx(S[i2], S[i3])));
      m[c] = (lo - T(0) + hi + T(0)) / T(2);
    }
    cen[r * nc + l] = Vec4<T>{m[0], m[1], m[2], T(0)};
  }
  __syncthreads();
  // Tile ranges: a half warp per 4 x 4 tile, one cell per lane.
  const int lane = t & 31, half = lane >> 4, hl = lane & 15;
  for (int base = 2 * (t >> 5); base < nreg * nt; base += 2 * kRefineWarps) {
    const int tt = base + half;
    const bool ok = tt < nreg * nt;
    const int r = ok ? tt / nt : 0, tile = ok ? tt - r * nt : 0, ty = tile / tw, tx = tile - (tile / tw) * tw;
    const int a = ty * kRefTe + (hl >> 2), b = tx * kRefTe + (hl & 3);
    T lo[3] = {pos_inf<T>(), pos_inf<T>(), pos_inf<T>()};
    T hi[3] = {-pos_inf<T>(), -pos_inf<T>(), -pos_inf<T>()};
    if (ok && a < W && b < W) {
      const Vec4<T> v = cen[r * nc + a * W + b];
      lo[0] = hi[0] = v.x;
      lo[1] = hi[1] = v.y;
      lo[2] = hi[2] = v.z;
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = fmn(lo[c], __shfl_xor_sync(kFull, lo[c], o));
        hi[c] = fmx(hi[c], __shfl_xor_sync(kFull, hi[c], o));
      }
    }
    if (ok && hl == 0) {
      T *d = sm.tb[(off + r) * kRefTiles + tile];
      d[0] = lo[0];
      d[1] = lo[1];
      d[2] = lo[2];
      d[3] = hi[0];
      d[4] = hi[1];
      d[5] = hi[2];
    }
  }
}

// All cell pairs of tile pair tp (slot-major, then tile 1, then tile 2),
// one warp: lane l takes tile-2 cell l % 16 against tile-1 cells
// 8 (l / 16) .. 8 (l / 16) + 7.  Pairs with ordered d2 above tau_ob are not
// entered.
template <typename T, typename SM>
__device__ __forceinline__ void ref_tile_pair(const SM &sm, const Vec4<T> *cen1, const Vec4<T> *cen2, int tp, int W,
                                              unsigned long long tau_ob, unsigned long long (&lo)[kBatchK],
                                              int (&lk)[kBatchK], unsigned long long &tests,
                                              unsigned long long &ins) {
  const int lane = threadIdx.x & 31, tw = (W + kRefTe - 1) / kRefTe, nt = tw * tw;
  const int slot = tp / (nt * nt), rem = tp - slot * nt * nt, t1 = rem / nt, t2 = rem - (rem / nt) * nt;
  const Vec4<T> *C1 = cen1 + sm.map1[slot] * W * W, *C2 = cen2 + sm.map2[slot] * W * W;
  const int ty1 = t1 / tw, tx1 = t1 - ty1 * tw, ty2 = t2 / tw, tx2 = t2 - ty2 * tw;
  const int l2 = lane & 15, a2 = ty2 * kRefTe + (l2 >> 2), b2 = tx2 * kRefTe + (l2 & 3);
  if (a2 >= W || b2 >= W) return;
  const int ci2 = a2 * W + b2;
  const Vec4<T> c2 = C2[ci2];
  unsigned long long n = 0;
#pragma unroll 4
  for (int q = 0; q < 8; ++q) {
    const int l1 = 8 * (lane >> 4) + q, a1 = ty1 * kRefTe + (l1 >> 2), b1 = tx1 * kRefTe + (l1 & 3);
    if (a1 >= W || b1 >= W) continue;
    const int ci1 = a1 * W + b1;
    const unsigned long long ob = ordered_bits(center_d2(C1[ci1], c2));
    ++n;
    if (ob <= tau_ob) {
      const int key = (slot << 16) | (ci1 << 8) | ci2;
      if (ref_less(ob, key, lo[kBatchK - 1], lk[kBatchK - 1])) {
        ref_insert(lo, lk, ob, key);
        ++ins;
      }
    }
  }
  tests += n;
}

template <typename T, int MAXP>
__global__ void __launch_bounds__(kRefineThreads) k_dist_refine(SurfView<T> sa, SurfView<T> sb, const SurfView<T> *va,
                                                                 const SurfView<T> *vb, ScreenStats *stats,
                                                                 DistRecord<T> *rec, RefineArgs<T> args,
                                                                 long long qs) {
  extern __shared__ __align__(16) unsigned char refine_raw[];
  RefineSmem<T, MAXP> &sm = *reinterpret_cast<RefineSmem<T, MAXP> *>(refine_raw);
  const long long qo = qoff(qs);
  if (va) sa = *qsh(va, qo);
  if (vb) sb = *qsh(vb, qo);
  stats = qsh(stats, qo);
  rec = qsh(rec, qo);
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int nuv = args.nuv, W = nuv - 1, tw = (W + kRefTe - 1) / kRefTe, nt = tw * tw, k = args.k;
  for (int round = args.first; round <= args.last; ++round) {
    const RefineRound<T> R = args.r[round - 1];
    const RegionRec<T> *reg1 = qsh(R.reg1, qo), *reg2 = qsh(R.reg2, qo);
    const int *map1 = qsh(R.map1, qo), *map2 = qsh(R.map2, qo);
    Vec4<T> *cen1 = qsh(R.cen1, qo), *cen2 = qsh(R.cen2, qo);
    const int last = round == args.last;
    // Counts from the previous round (its close and next).
    const int st = stats->status;
    const int nslots = st == 0 ? min(stats->nslots, kBatchK) : 0;
    const int nreg1 = nslots > 0 ? min(stats->nreg1, kBatchK) : 0;
    const int nreg2 = nslots > 0 ? min(stats->nreg2, kBatchK) : 0;
    if (t == 0) {
      sm.tests = 0;
      sm.cands = 0;
      sm.surv = 0;
    }
    if (t < kBatchK) {
      // region indices of the slots, kept inside the evaluated regions
      sm.map1[t] = t < nslots ? min(max(map1[t], 0), max(nreg1 - 1, 0)) : 0;
      sm.map2[t] = t < nslots ? min(max(map2[t], 0), max(nreg2 - 1, 0)) : 0;
    }
    ref_side<T, MAXP>(sm, sa, reg1, nreg1, nuv, 0, cen1);
    __syncthreads();
    ref_side<T, MAXP>(sm, sb, reg2, nreg2, nuv, kBatchK, cen2);
    __syncthreads();
    // Warp w bounds slot w's tile pairs and examines the one with the
    // smallest bound (ties by index); the k-th of those pairs is tau.
    const int npairs = nslots * nt * nt, per = nt * nt;
    unsigned long long lo[kBatchK];
    int lk[kBatchK];
#pragma unroll
    for (int j = 0; j < kBatchK; ++j) {
      lo[j] = kRefPadOb;
      lk[j] = kRefPadKey;
    }
    if (t < kRefPairs / 32) sm.headmask[t] = 0u;
    if (t == 0) sm.ntpl = 0;
    __syncthreads();
    unsigned long long tests = 0, ins = 0, surv = 0;
    if (w < nslots) {
      unsigned long long bo = kRefPadOb;
      int bk = kRefPadKey;
      const T *tb1 = sm.tb[sm.map1[w] * kRefTiles];
      const T *tb2 = sm.tb[(kBatchK + sm.map2[w]) * kRefTiles];
      for (int q = lane; q < per; q += 32) {
        const int t1 = q / nt, t2 = q - (q / nt) * nt, tp = w * per + q;
        const T *b1 = tb1 + 6 * t1, *b2 = tb2 + 6 * t2;
        const T lb = tile_lb(Vec4<T>{b1[0], b1[1], b1[2], T(0)}, Vec4<T>{b1[3], b1[4], b1[5], T(0)},
                             Vec4<T>{b2[0], b2[1], b2[2], T(0)}, Vec4<T>{b2[3], b2[4], b2[5], T(0)});
        sm.tplb[tp] = lb;
        const unsigned long long ob = ordered_bits(lb);
        if (ref_less(ob, tp, bo, bk)) {
          bo = ob;
          bk = tp;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long oo = __shfl_xor_sync(kFull, bo, o);
        const int ok = __shfl_xor_sync(kFull, bk, o);
        if (ref_less(oo, ok, bo, bk)) {
          bo = oo;
          bk = ok;
        }
      }
      if (lane == 0) atomicOr(&sm.headmask[bk >> 5], 1u << (bk & 31));
      ref_tile_pair<T>(sm, cen1, cen2, bk, W, kRefPadOb, lo, lk, tests, ins);
      ++surv;
    }
    ref_merge(sm, lo, lk, k);
    const unsigned long long tau_ob = sm.n == k ? sm.tob[k - 1] : kRefPadOb;
    // The other tile pairs whose bound is at most tau, compacted, then one
    // per warp.
    for (int tp = t; tp < npairs; tp += kRefineThreads) {
      if ((sm.headmask[tp >> 5] >> (tp & 31)) & 1u) continue;
      if (ordered_bits(sm.tplb[tp]) > tau_ob) continue;
      const int pos = atomicAdd(&sm.ntpl, 1);
      sm.tpl[pos] = static_cast<unsigned short>(tp);
    }
    __syncthreads();
    const int ntpl = sm.ntpl;
    for (int e = w; e < ntpl; e += kRefineWarps) {
      ref_tile_pair<T>(sm, cen1, cen2, sm.tpl[e], W, tau_ob, lo, lk, tests, ins);
      ++surv;
    }
    // tests / ins are per lane, surv per warp
    if (lane == 0) atomicAdd(&sm.surv, surv);
    atomicAdd(&sm.tests, tests);
    atomicAdd(&sm.cands, ins);
    ref_merge(sm, lo, lk, k);
    const int n = sm.n;
    DistCand<T> *top = qsh(R.top, qo);
    if (t < n) {
      const int key = sm.tkey[t];
      const DistCand<T> c{from_ordered<T>(sm.tob[t]), key >> 16, (key >> 8) & 255, key & 255};
      top[t] = c;
      rec->top[round - 1][t] = c;
    }
    if (t == 0) {
      if (R.next1 && n > 0) {
        // Pair-preserving jobs with (slot, cell) dedup per side, in the
        // order of the kept pairs (k_dist_next).
        RegionRec<T> *next1 = qsh(R.next1, qo), *next2 = qsh(R.next2, qo);
        int *nmap1 = qsh(R.nmap1, qo), *nmap2 = qsh(R.nmap2, qo);
        int c1 = 0, c2 = 0;
        int m1[kBatchK], m2[kBatchK];  // this round's maps, kept on chip while they are built
        for (int e = 0; e < n; ++e) {
          const int ke = sm.tkey[e], se = ke >> 16, ie = (ke >> 8) & 255, je = ke & 255;
          int u1 = -1, u2 = -1;
          for (int q = 0; q < e; ++q) {
            const int kq = sm.tkey[q], sq = kq >> 16;
            if (u1 < 0 && sq == se && ((kq >> 8) & 255) == ie) u1 = m1[q];
            if (u2 < 0 && sq == se && (kq & 255) == je) u2 = m2[q];
          }
          if (u1 < 0) {
            u1 = c1++;
            next1[u1] = child_rect(reg1[sm.map1[se]], nuv, ie);
          }
          if (u2 < 0) {
            u2 = c2++;
            next2[u2] = child_rect(reg2[sm.map2[se]], nuv, je);
          }
          m1[e] = u1;
          m2[e] = u2;
          nmap1[e] = u1;
          nmap2[e] = u2;
        }
        stats->nreg1 = c1;
        stats->nreg2 = c2;
      }
      rec->tests[round - 1] = static_cast<long long>(sm.tests);
      rec->cands[round - 1] = static_cast<long long>(sm.cands);
      rec->survivors[round - 1] = sm.surv;
      rec->examined[round - 1] = static_cast<unsigned long long>(npairs);
      rec->st_kept[round - 1] = 0;
      rec->npairs[round - 1] = n;
      rec->status[round - 1] = st;
      stats->nsel = n;
      stats->nslots = n;
      stats->tile_pairs = static_cast<unsigned long long>(npairs);
      stats->survivors = sm.surv;
      stats->pair_tests = sm.tests;
      stats->candidates = sm.cands;
      if (!last) {
        stats->status = 0;
        stats->tau_bits = 0x7f800000u;
      }
    }
    __syncthreads();
  }
}

// Block-wide search over 4096 counts for the bin where the running total
// reaches want: *bin and the count still needed inside it (1024 threads).
__device__ void find_crossing(const unsigned *hist, unsigned want, unsigned *s_warp, int *s_bin, unsigned *s_need) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const unsigned h0 = hist[4 * t], h1 = hist[4 * t + 1], h2 = hist[4 * t + 2], h3 = hist[4 * t + 3];
  const unsigned sum = h0 + h1 + h2 + h3;
  unsigned inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned v = __shfl_up_sync(kFull, inc, o);
    if (lane >= o) inc += v;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    unsigned w = s_warp[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(kFull, w, o);
      if (lane >= o) w += v;
    }
    s_warp[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  const unsigned before = (warp ? s_warp[warp - 1] : 0u) + inc - sum;
  if (before < want && before + sum >= want) {
    unsigned c = before;
    int b = 4 * t;
    if (c + h0 < want) {
      c += h0;
      ++b;
      if (c + h1 < want) {
        c += h1;
        ++b;
        if (c + h2 < want) {
          c += h2;
          ++b;
        }
      }
    }
    *s_bin = b;
    *s_need = want - c;
  }
  __syncthreads();
}

// Threshold-pass list of a batched round, one block of 1024 per query: all
// surviving tile pairs when at most `want` survive, else about `want` of them
// (at most head_cap) with the smallest bounds (two-level radix select on the
// bound bits), so the exact per-tile-pair k-th comes from the closest tile
// pairs and the collecting pass meets a tight threshold.
__global__ void __launch_bounds__(1024) k_dist_pick(const unsigned long long *surv, const unsigned *surv_lb,
                                                    unsigned long long surv_cap, unsigned long long *head,
                                                    unsigned long long head_cap, unsigned want, ScreenStats *stats,
                                                    long long qs) {
  __shared__ unsigned hist[4096];
  __shared__ unsigned s_warp[32], s_need, s_cnt;
  __shared__ int s_bin;
  const long long qo = qoff(qs);
  surv = qsh(surv, qo);
  surv_lb = qsh(surv_lb, qo);
  head = qsh(head, qo);
  stats = qsh(stats, qo);
  const unsigned long long n = count_of(kFromDevice, stats->survivors, surv_cap);
  if (n <= want) {
    for (unsigned long long e = threadIdx.x; e < n; e += blockDim.x) head[e] = surv[e];
    if (threadIdx.x == 0) stats->nhead = n;
    return;
  }
  for (int b = threadIdx.x; b < 4096; b += blockDim.x) hist[b] = 0;
  if (threadIdx.x == 0) {
    s_bin = 4095;
    s_need = want;
  }
  __syncthreads();
  for (unsigned long long e = threadIdx.x; e < n; e += blockDim.x) atomicAdd(&hist[surv_lb[e] >> 20], 1u);
  __syncthreads();
  find_crossing(hist, want, s_warp, &s_bin, &s_need);
  const unsigned b1 = static_cast<unsigned>(s_bin), need = s_need;
  for (int b = threadIdx.x; b < 4096; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  for (unsigned long long e = threadIdx.x; e < n; e += blockDim.x) {
    const unsigned key = surv_lb[e];
    if ((key >> 20) == b1) atomicAdd(&hist[(key >> 8) & 4095u], 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) s_bin = 4095;
  __syncthreads();
  find_crossing(hist, need, s_warp, &s_bin, &s_need);
  const unsigned thr = (b1 << 12) | static_cast<unsigned>(s_bin);
  if (threadIdx.x == 0) s_cnt = 0;
  __syncthreads();
  for (unsigned long long e = threadIdx.x; e < n; e += blockDim.x) {
    if ((surv_lb[e] >> 8) <= thr) {
      const unsigned pos = atomicAdd(&s_cnt, 1u);
      if (pos < head_cap) head[pos] = surv[e];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) stats->nhead = s_cnt < head_cap ? s_cnt : head_cap;
}

// ---------------------------------------------------------------------------
// Intersection screening
// ---------------------------------------------------------------------------

// FP32-screen widening of one region pair, per axis: the FP64 paddings of
// both regions (rounded up through a relative margin of 2^-20) plus the
// host's bound w of the samples' FP32 error and every rounding on either
// side; see inter_screen_widen in the host code.
__device__ __forceinline__ float iscreen_q(double p1, double p2, float w) {
  return __double2float_ru((p1 + p2) * (1.0 + 0x1p-20) + static_cast<double>(w));
}

// A tile pair is skipped only when, on some axis, the rounded gap between the
// centre ranges reaches the rounded sum of the largest padded radii: then no
// member pair passes the strict test of intersection.cu:60-62.  S (the FP32
// screen, T = float): the radii sum is (h1 + h2) + Q with Q from
// iscreen_q, and pad64a / pad64b hold the FP64 paddings.
template <typename T, bool S>
__global__ void k_inter_cull(SideRound<T> a, SideRound<T> b, const int *map1, const int *map2, int nslots,
                             unsigned long long *surv, unsigned long long surv_cap, ScreenStats *stats,
                             Vec4<float> wq, const double *pad64a, const double *pad64b) {
  const Geom g1 = a.g, g2 = b.g;
  const long long nrows = static_cast<long long>(nslots) * g1.ntiles;
  const int lanes = blockDim.x;
  // Rows (slot, t1) x t2 flattened so that small tile counts still fill warps.
  const long long total = nrows * g2.ntiles;
  for (long long base = blockIdx.x * static_cast<long long>(lanes); base < total;
       base += static_cast<long long>(gridDim.x) * lanes) {
    const long long e = base + threadIdx.x;
    bool keep = false;
    int row = 0, t2 = 0;
    if (e < total) {
      row = static_cast<int>(e / g2.ntiles);
      t2 = static_cast<int>(e - static_cast<long long>(row) * g2.ntiles);
      const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
      const int r1 = map1[slot], r2 = map2[slot];
      const long long i1 = static_cast<long long>(r1) * g1.ntiles + t1;
      const long long i2 = static_cast<long long>(r2) * g2.ntiles + t2;
      const Vec4<T> lo1 = a.tlo[i1], hi1 = a.thi[i1], h1 = a.thmax[i1];
      const Vec4<T> lo2 = b.tlo[i2], hi2 = b.thi[i2], h2 = b.thmax[i2];
      bool sx, sy, sz;
      if constexpr (S) {
        const double q1 = pad64a[r1], q2 = pad64b[r2];
        sx = axis_gap(lo1.x, hi1.x, lo2.x, hi2.x) >= (h1.x + h2.x) + iscreen_q(q1, q2, wq.x);
        sy = axis_gap(lo1.y, hi1.y, lo2.y, hi2.y) >= (h1.y + h2.y) + iscreen_q(q1, q2, wq.y);
        sz = axis_gap(lo1.z, hi1.z, lo2.z, hi2.z) >= (h1.z + h2.z) + iscreen_q(q1, q2, wq.z);
      } else {
        const T p1 = a.pad[r1], p2 = b.pad[r2];
        sx = axis_gap(lo1.x, hi1.x, lo2.x, hi2.x) >= (h1.x + p1) + (h2.x + p2);
        sy = axis_gap(lo1.y, hi1.y, lo2.y, hi2.y) >= (h1.y + p1) + (h2.y + p2);
        sz = axis_gap(lo1.z, hi1.z, lo2.z, hi2.z) >= (h1.z + p1) + (h2.z + p2);
      }
      keep = !(sx || sy || sz);
    }
    const long long pos = warp_append(keep, &stats->survivors);
    if (pos >= 0 && static_cast<unsigned long long>(pos) < surv_cap)
      surv[pos] = pack_tile_pair(static_cast<unsigned>(row), static_cast<unsigned>(t2));
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(&stats->tile_pairs, static_cast<unsigned long long>(total));
}

// Strict per-axis overlap of every cell pair of the surviving tile pairs
// (intersection.cu:46-63), one warp per tile pair: tile-2 centres and padded
// radii in registers, tile-1 cells broadcast row by row; hits are appended as
// (slot, i, j) sort keys.  S (FP32 screen): |c1 - c2| < (h1 + h2) + Q per
// axis, a superset of the FP64 form's pairs.
template <typename T, bool S>
__global__ void __launch_bounds__(256) k_inter_leaf(SideRound<T> a, SideRound<T> b, const int *map1,
                                                    const int *map2, const unsigned long long *surv,
                                                    unsigned long long nsurv, int ij_bits, unsigned long long *keys,
                                                    unsigned long long key_cap, ScreenStats *stats, Vec4<float> wq,
                                                    const double *pad64a, const double *pad64b) {
  const Geom g1 = a.g, g2 = b.g;
  const int te1 = g1.te, te2 = g2.te;
  const int n1 = te1 * te1, n2 = te2 * te2;
  const int lane = threadIdx.x & 31;
  unsigned long long tests = 0;
  const Vec4<T> zero4{T(0), T(0), T(0), T(0)};
  const Vec4<T> neg4{-pos_inf<T>(), -pos_inf<T>(), -pos_inf<T>(), T(0)};
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(&stats->work, 1ull);
    w = __shfl_sync(kFull, w, 0);
    if (w >= nsurv) break;
    const unsigned long long q = surv[w];
    const int row = static_cast<int>(q >> 32), t2 = static_cast<int>(q & 0xffffffffull);
    const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
    const int r1 = map1[slot], r2 = map2[slot];
    const long long base1 = (static_cast<long long>(r1) * g1.ntiles + t1) * n1;
    const long long base2 = (static_cast<long long>(r2) * g2.ntiles + t2) * n2;
    // Per-cell radius terms: FP64 form, p1 on side 1 and p2 on side 2; FP32
    // screen, the pair's widening Q per axis (from the kernel argument wq,
    // which stays unchanged across tile pairs).
    T p1 = T(0), p2 = T(0);
    Vec4<float> Q{0.0f, 0.0f, 0.0f, 0.0f};
    if constexpr (S) {
      const double q1 = pad64a[r1], q2 = pad64b[r2];
      Q = Vec4<float>{iscreen_q(q1, q2, wq.x), iscreen_q(q1, q2, wq.y), iscreen_q(q1, q2, wq.z), 0.0f};
    } else {
      p1 = a.pad[r1];
      p2 = b.pad[r2];
    }
    const int ty1 = t1 / g1.tw, tx1 = t1 - ty1 * g1.tw, ty2 = t2 / g2.tw, tx2 = t2 - ty2 * g2.tw;
    const int nv1 = min(te1, g1.W - ty1 * te1), nu1 = min(te1, g1.W - tx1 * te1);
    const int nv2 = min(te2, g2.W - ty2 * te2), nu2 = min(te2, g2.W - tx2 * te2);
    const int ja = lane, jb = lane + 32;
    const int ja_v = ja / te2, ja_u = ja - ja_v * te2, jb_v = jb / te2, jb_u = jb - jb_v * te2;
    const bool va = ja < n2 && ja_v < nv2 && ja_u < nu2;
    const bool vb = jb < n2 && jb_v < nv2 && jb_u < nu2;
    // Invalid lanes get a zero centre and a -inf radius: |dc| < -inf never holds.
    Vec4<T> c2a = va ? b.center[base2 + ja] : zero4, c2b = vb ? b.center[base2 + jb] : zero4;
    Vec4<T> r2a = neg4, r2b = neg4;
    if (va) {
      r2a = b.half[base2 + ja];
      if constexpr (!S) {
        r2a.x = r2a.x + p2;  // radius = x_span / 2 + curvature_padding
        r2a.y = r2a.y + p2;
        r2a.z = r2a.z + p2;
      }
    }
    if (vb) {
      r2b = b.half[base2 + jb];
      if constexpr (!S) {
        r2b.x = r2b.x + p2;
        r2b.y = r2b.y + p2;
        r2b.z = r2b.z + p2;
      }
    }
    const unsigned long long cja = static_cast<unsigned long long>((ty2 * te2 + ja_v) * g2.W + tx2 * te2 + ja_u);
    const unsigned long long cjb = static_cast<unsigned long long>((ty2 * te2 + jb_v) * g2.W + tx2 * te2 + jb_u);
    const unsigned long long slot_key = static_cast<unsigned long long>(slot) << (2 * ij_bits);
    for (int a1 = 0; a1 < nv1; ++a1) {
      for (int b1 = 0; b1 < nu1; ++b1) {
        const Vec4<T> c1 = a.center[base1 + a1 * te1 + b1];
        Vec4<T> r1 = a.half[base1 + a1 * te1 + b1];
        bool ha, hb;
        if constexpr (S) {
          ha = fabs(c1.x - c2a.x) < (r1.x + r2a.x) + Q.x && fabs(c1.y - c2a.y) < (r1.y + r2a.y) + Q.y &&
               fabs(c1.z - c2a.z) < (r1.z + r2a.z) + Q.z;
          hb = fabs(c1.x - c2b.x) < (r1.x + r2b.x) + Q.x && fabs(c1.y - c2b.y) < (r1.y + r2b.y) + Q.y &&
               fabs(c1.z - c2b.z) < (r1.z + r2b.z) + Q.z;
        } else {
          r1.x = r1.x + p1;
          r1.y = r1.y + p1;
          r1.z = r1.z + p1;
          ha = fabs(c1.x - c2a.x) < (r1.x + r2a.x) && fabs(c1.y - c2a.y) < (r1.y + r2a.y) &&
               fabs(c1.z - c2a.z) < (r1.z + r2a.z);
          hb = fabs(c1.x - c2b.x) < (r1.x + r2b.x) && fabs(c1.y - c2b.y) < (r1.y + r2b.y) &&
               fabs(c1.z - c2b.z) < (r1.z + r2b.z);
        }
        if (__any_sync(kFull, ha || hb)) {
          const unsigned long long ci =
              static_cast<unsigned long long>((ty1 * te1 + a1) * g1.W + tx1 * te1 + b1) << ij_bits;
          long long pos = warp_append(ha, &stats->candidates);
          if (pos >= 0 && static_cast<unsigned long long>(pos) < key_cap) keys[pos] = slot_key | ci | cja;
          pos = warp_append(hb, &stats->candidates);
          if (pos >= 0 && static_cast<unsigned long long>(pos) < key_cap) keys[pos] = slot_key | ci | cjb;
        }
      }
    }
    if (lane == 0) tests += static_cast<unsigned long long>(nv1 * nu1) * (nv2 * nu2);
  }
  if (lane == 0) atomicAdd(&stats->pair_tests, tests);
}

// ---- bounds mode (certified distance interval) ------------------------------

// Rigorous padding of a region's cells on the covering grid, per coordinate:
// over a cell, coordinate c of the surface is within
// (du^2 max|S_uu[c]| + dv^2 max|S_vv[c]|) / 8 of the bilinear interpolant of
// the four corners (tensor-product linear interpolation), and that
// interpolant lies in the corners' box.  du, dv are the region's sample
// spacings, inflated for the rounding of the sample parameters; m2u / m2v
// bound |S_uu| / |S_vv| per coordinate over the surface (the
// second-derivative nets, convex hull); eps covers the evaluation and the
// centre / half-span rounding.  pad4 holds a Vec4 per region.
__global__ void k_pad_bound(SideRound<double> sr, Vec4<double> *pad4, SurfView<double> v, const Vec4<double> *tab,
                            double eps) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= sr.nreg) return;
  const RegionRec<double> reg = sr.regions[r];
  const double n1 = static_cast<double>(sr.g.nuv - 1);
  const double slack = 1.0 + 0x1p-40;
  const double du = __dadd_ru(__dmul_ru(__ddiv_ru(fabs(reg.u1 - reg.u0), n1), slack),
                              0x1p-50 * (fabs(reg.u0) + fabs(reg.u1)));
  const double dv = __dadd_ru(__dmul_ru(__ddiv_ru(fabs(reg.v1 - reg.v0), n1), slack),
                              0x1p-50 * (fabs(reg.v0) + fabs(reg.v1)));
  const double du2 = __dmul_ru(du, du), dv2 = __dmul_ru(dv, dv);
  // The largest span bounds over every knot span the region touches.  The
  // upper end is looked up just below itself: a region that ends on a knot
  // lies in the closed span before it, where that span's polynomial bound
  // holds.
  const int p = v.degu, q = v.degv, nsu = v.ncpu - p;
  const double ulo = fmin(reg.u0, reg.u1), uhi = fmax(reg.u0, reg.u1);
  const double vlo = fmin(reg.v0, reg.v1), vhi = fmax(reg.v0, reg.v1);
  const int su0 = find_span(v.nku, p, ulo, v.U), su1 = find_span(v.nku, p, uhi > ulo ? nextafter(uhi, ulo) : uhi, v.U);
  const int sv0 = find_span(v.nkv, q, vlo, v.V), sv1 = find_span(v.nkv, q, vhi > vlo ? nextafter(vhi, vlo) : vhi, v.V);
  Vec4<double> mu{0, 0, 0, 0}, mv{0, 0, 0, 0};
  for (int sv = sv0; sv <= sv1; ++sv)
    for (int su = su0; su <= su1; ++su) {
      const Vec4<double> a = tab[2 * ((sv - q) * nsu + (su - p))], b = tab[2 * ((sv - q) * nsu + (su - p)) + 1];
      mu = Vec4<double>{fmax(mu.x, a.x), fmax(mu.y, a.y), fmax(mu.z, a.z), 0.0};
      mv = Vec4<double>{fmax(mv.x, b.x), fmax(mv.y, b.y), fmax(mv.z, b.z), 0.0};
    }
  auto one = [&](double m_u, double m_v) {
    const double e = __dadd_ru(__dmul_ru(du2, m_u), __dmul_ru(dv2, m_v));
    return __dadd_ru(__dmul_ru(__dmul_ru(e, 0.125), slack), eps);
  };
  pad4[r] = Vec4<double>{one(mu.x, mv.x), one(mu.y, mv.y), one(mu.z, mv.z), 0.0};
}

// Lower bound of the gap between [c1 - r1, c1 + r1] and [c2 - r2, c2 + r2].
__device__ __forceinline__ double axis_gap_rd(double c1, double r1, double c2, double r2) {
  const double d = c1 >= c2 ? __dsub_rd(c1, c2) : __dsub_rd(c2, c1);
  const double g = __dsub_rd(d, __dadd_ru(r1, r2));
  return g > 0.0 ? g : 0.0;
}

__device__ __forceinline__ double gap2_rd(double gx, double gy, double gz) {
  return __dadd_rd(__dadd_rd(__dmul_rd(gx, gx), __dmul_rd(gy, gy)), __dmul_rd(gz, gz));
}

// Lower bound of the distance between two cell patches from their corner
// samples: each patch lies in the convex hull of its four corners widened by
// its per-coordinate pads, and projecting onto a unit direction never
// lengthens a distance, so with d the centre-to-centre direction
//   gap >= (min_j d.q_j - max_i d.p_i - sum_c |d_c| (pad1_c + pad2_c)) / |d|.
// Near the closest approach d is close to the common normal and the hulls are
// thin along it, so this bound is second-order in the cell size where the
// axis-aligned gap is first-order.  The dot products' rounding is covered by
// subtracting 8 u |d| (max |p| + max |q|) (u = 2^-53) from the numerator.
__device__ __forceinline__ double proj_gap_rd(const Vec4<double> P[4], const Vec4<double> Q[4], const Vec4<double> &c1,
                                              const Vec4<double> &c2, const Vec4<double> &p1,
                                              const Vec4<double> &p2) {
  const double dx = c2.x - c1.x, dy = c2.y - c1.y, dz = c2.z - c1.z;
  const double dn = sqrt(dx * dx + dy * dy + dz * dz);
  if (!(dn > 0.0)) return 0.0;
  double pmax = -pos_inf<double>(), qmin = pos_inf<double>(), mag = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    pmax = fmax(pmax, dx * P[i].x + dy * P[i].y + dz * P[i].z);
    qmin = fmin(qmin, dx * Q[i].x + dy * Q[i].y + dz * Q[i].z);
    mag = fmax(mag, fmax(fabs(P[i].x) + fabs(P[i].y) + fabs(P[i].z), fabs(Q[i].x) + fabs(Q[i].y) + fabs(Q[i].z)));
  }
  const double spread = __dadd_ru(__dadd_ru(__dmul_ru(fabs(dx), __dadd_ru(p1.x, p2.x)),
                                            __dmul_ru(fabs(dy), __dadd_ru(p1.y, p2.y))),
                                  __dmul_ru(fabs(dz), __dadd_ru(p1.z, p2.z)));
  const double slop = __dmul_ru(__dmul_ru(0x1p-50, __dadd_ru(fabs(dx), __dadd_ru(fabs(dy), fabs(dz)))), 2.0 * mag);
  const double num = __dsub_rd(__dsub_rd(__dsub_rd(qmin, pmax), spread), slop);
  if (!(num > 0.0)) return 0.0;
  return __ddiv_rd(num, __dmul_ru(dn, 1.0 + 0x1p-50));
}

// Squared distance of two points, rounded up.
__device__ __forceinline__ double dist2_ru(const Vec4<double> &p, const Vec4<double> &q) {
  const double dx = p.x >= q.x ? __dsub_ru(p.x, q.x) : __dsub_ru(q.x, p.x);
  const double dy = p.y >= q.y ? __dsub_ru(p.y, q.y) : __dsub_ru(q.y, p.y);
  const double dz = p.z >= q.z ? __dsub_ru(p.z, q.z) : __dsub_ru(q.z, p.z);
  return __dadd_ru(__dadd_ru(__dmul_ru(dx, dx), __dmul_ru(dy, dy)), __dmul_ru(dz, dz));
}

// Tile pairs whose box gap (centre ranges widened by the largest padded half
// spans) can be <= ub.
__global__ void k_bound_cull(SideRound<double> a, SideRound<double> b, const int *map1, const int *map2, int nslots,
                             double ub2, unsigned long long *surv, unsigned long long surv_cap, ScreenStats *stats) {
  const Geom g1 = a.g, g2 = b.g;
  const long long total = static_cast<long long>(nslots) * g1.ntiles * g2.ntiles;
  for (long long base = blockIdx.x * static_cast<long long>(blockDim.x); base < total;
       base += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long e = base + threadIdx.x;
    bool keep = false;
    int row = 0, t2 = 0;
    if (e < total) {
      row = static_cast<int>(e / g2.ntiles);
      t2 = static_cast<int>(e - static_cast<long long>(row) * g2.ntiles);
      const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
      const int r1 = map1[slot], r2 = map2[slot];
      const long long i1 = static_cast<long long>(r1) * g1.ntiles + t1;
      const long long i2 = static_cast<long long>(r2) * g2.ntiles + t2;
      const Vec4<double> lo1 = a.tlo[i1], hi1 = a.thi[i1], h1 = a.thmax[i1];
      const Vec4<double> lo2 = b.tlo[i2], hi2 = b.thi[i2], h2 = b.thmax[i2];
      const Vec4<double> p1 = reinterpret_cast<const Vec4<double> *>(a.pad)[r1];
      const Vec4<double> p2 = reinterpret_cast<const Vec4<double> *>(b.pad)[r2];
      double gg[3];
      const double L1[3] = {lo1.x, lo1.y, lo1.z}, H1[3] = {hi1.x, hi1.y, hi1.z}, R1[3] = {h1.x, h1.y, h1.z};
      const double L2[3] = {lo2.x, lo2.y, lo2.z}, H2[3] = {hi2.x, hi2.y, hi2.z}, R2[3] = {h2.x, h2.y, h2.z};
      const double P1[3] = {p1.x, p1.y, p1.z}, P2[3] = {p2.x, p2.y, p2.z};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double gap = fmax(fmax(__dsub_rd(L2[c], H1[c]), __dsub_rd(L1[c], H2[c])), 0.0);
        const double reach = __dadd_ru(__dadd_ru(R1[c], P1[c]), __dadd_ru(R2[c], P2[c]));
        const double g = __dsub_rd(gap, reach);
        gg[c] = g > 0.0 ? g : 0.0;
      }
      keep = gap2_rd(gg[0], gg[1], gg[2]) <= ub2;
    }
    const long long pos = warp_append(keep, &stats->survivors);
    if (pos >= 0 && static_cast<unsigned long long>(pos) < surv_cap)
      surv[pos] = pack_tile_pair(static_cast<unsigned>(row), static_cast<unsigned>(t2));
  }
  if (threadIdx.x == 0 && blockIdx.x == 0) atomicAdd(&stats->tile_pairs, static_cast<unsigned long long>(total));
}

// Cell pairs of the surviving tile pairs whose padded boxes can be within ub,
// one warp per tile pair (the layout of k_inter_leaf); each warp folds the
// smallest kept squared gap of its tile pair into lb_bits, and the smallest
// squared distance (rounded up) between the kept pairs' first corner
// samples, which are surface points, into ub_bits.
__global__ void __launch_bounds__(256) k_bound_leaf(SideRound<double> a, SideRound<double> b, const int *map1,
                                                    const int *map2, const unsigned long long *surv,
                                                    unsigned long long nsurv, int ij_bits, double ub2,
                                                    unsigned long long *keys, unsigned long long key_cap,
                                                    ScreenStats *stats) {
  const Geom g1 = a.g, g2 = b.g;
  const int te1 = g1.te, te2 = g2.te;
  const int n1 = te1 * te1, n2 = te2 * te2;
  const int lane = threadIdx.x & 31;
  unsigned long long tests = 0;
  const Vec4<double> zero4{0.0, 0.0, 0.0, 0.0};
  for (;;) {
    unsigned long long w = 0;
    if (lane == 0) w = atomicAdd(&stats->work, 1ull);
    w = __shfl_sync(kFull, w, 0);
    if (w >= nsurv) break;
    const unsigned long long q = surv[w];
    const int row = static_cast<int>(q >> 32), t2 = static_cast<int>(q & 0xffffffffull);
    const int slot = row / g1.ntiles, t1 = row - slot * g1.ntiles;
    const int r1 = map1[slot], r2 = map2[slot];
    const long long base1 = (static_cast<long long>(r1) * g1.ntiles + t1) * n1;
    const long long base2 = (static_cast<long long>(r2) * g2.ntiles + t2) * n2;
    const Vec4<double> p1 = reinterpret_cast<const Vec4<double> *>(a.pad)[r1];
    const Vec4<double> p2 = reinterpret_cast<const Vec4<double> *>(b.pad)[r2];
    const int ty1 = t1 / g1.tw, tx1 = t1 - ty1 * g1.tw, ty2 = t2 / g2.tw, tx2 = t2 - ty2 * g2.tw;
    const int nv1 = min(te1, g1.W - ty1 * te1), nu1 = min(te1, g1.W - tx1 * te1);
    const int nv2 = min(te2, g2.W - ty2 * te2), nu2 = min(te2, g2.W - tx2 * te2);
    const int ja = lane, jb = lane + 32;
    const int ja_v = ja / te2, ja_u = ja - ja_v * te2, jb_v = jb / te2, jb_u = jb - jb_v * te2;
    const bool va = ja < n2 && ja_v < nv2 && ja_u < nu2;
    const bool vb = jb < n2 && jb_v < nv2 && jb_u < nu2;
    const Vec4<double> c2a = va ? b.center[base2 + ja] : zero4, c2b = vb ? b.center[base2 + jb] : zero4;
    Vec4<double> r2a = zero4, r2b = zero4;
    if (va) {
      r2a = b.half[base2 + ja];
      r2a.x = __dadd_ru(r2a.x, p2.x);
      r2a.y = __dadd_ru(r2a.y, p2.y);
      r2a.z = __dadd_ru(r2a.z, p2.z);
    }
    if (vb) {
      r2b = b.half[base2 + jb];
      r2b.x = __dadd_ru(r2b.x, p2.x);
      r2b.y = __dadd_ru(r2b.y, p2.y);
      r2b.z = __dadd_ru(r2b.z, p2.z);
    }
    const unsigned long long cja = static_cast<unsigned long long>((ty2 * te2 + ja_v) * g2.W + tx2 * te2 + ja_u);
    const unsigned long long cjb = static_cast<unsigned long long>((ty2 * te2 + jb_v) * g2.W + tx2 * te2 + jb_u);
    const unsigned long long slot_key = static_cast<unsigned long long>(slot) << (2 * ij_bits);
    // First corner samples of the lane's side-2 cells.
    const Vec4<double> *S1 = a.samples + static_cast<long long>(r1) * g1.nuv * g1.nuv;
    const Vec4<double> *S2 = b.samples + static_cast<long long>(r2) * g2.nuv * g2.nuv;
    // Corner samples (surface points) of the lane's side-2 cells.
    Vec4<double> Qa[4], Qb[4];
#pragma unroll
    for (int cn = 0; cn < 4; ++cn) {
      const int dv = cn >> 1, du = cn & 1;
      Qa[cn] = va ? S2[(ty2 * te2 + ja_v + dv) * g2.nuv + tx2 * te2 + ja_u + du] : zero4;
      Qb[cn] = vb ? S2[(ty2 * te2 + jb_v + dv) * g2.nuv + tx2 * te2 + jb_u + du] : zero4;
    }
    const Vec4<double> &q2a = Qa[0], &q2b = Qb[0];
    double mine = pos_inf<double>(), close = pos_inf<double>();
    for (int a1 = 0; a1 < nv1; ++a1) {
      for (int b1 = 0; b1 < nu1; ++b1) {
        const Vec4<double> c1 = a.center[base1 + a1 * te1 + b1];
        Vec4<double> r1v = a.half[base1 + a1 * te1 + b1];
        r1v.x = __dadd_ru(r1v.x, p1.x);
        r1v.y = __dadd_ru(r1v.y, p1.y);
        r1v.z = __dadd_ru(r1v.z, p1.z);
        const double ga = gap2_rd(axis_gap_rd(c1.x, r1v.x, c2a.x, r2a.x), axis_gap_rd(c1.y, r1v.y, c2a.y, r2a.y),
                                  axis_gap_rd(c1.z, r1v.z, c2a.z, r2a.z));
        const double gb = gap2_rd(axis_gap_rd(c1.x, r1v.x, c2b.x, r2b.x), axis_gap_rd(c1.y, r1v.y, c2b.y, r2b.y),
                                  axis_gap_rd(c1.z, r1v.z, c2b.z, r2b.z));
        bool ha = va && ga <= ub2, hb = vb && gb <= ub2;
        double ka = ga, kb = gb;
        if (ha || hb) {
          Vec4<double> P[4];
#pragma unroll
          for (int cn = 0; cn < 4; ++cn)
            P[cn] = S1[(ty1 * te1 + a1 + (cn >> 1)) * g1.nuv + tx1 * te1 + b1 + (cn & 1)];
          // Tighter second-order bound (both bounds are valid: keep the larger).
          if (ha) {
            const double pg = proj_gap_rd(P, Qa, c1, c2a, p1, p2);
            ka = fmax(ka, __dmul_rd(pg, pg));
            ha = ka <= ub2;
          }
          if (hb) {
            const double pg = proj_gap_rd(P, Qb, c1, c2b, p1, p2);
            kb = fmax(kb, __dmul_rd(pg, pg));
            hb = kb <= ub2;
          }
          if (ha) close = fmin(close, dist2_ru(P[0], q2a));
          if (hb) close = fmin(close, dist2_ru(P[0], q2b));
        }
        if (ha) mine = fmin(mine, ka);
        if (hb) mine = fmin(mine, kb);
        if (__any_sync(kFull, ha || hb)) {
          const unsigned long long ci =
              static_cast<unsigned long long>((ty1 * te1 + a1) * g1.W + tx1 * te1 + b1) << ij_bits;
          long long pos = warp_append(ha, &stats->candidates);
          if (pos >= 0 && static_cast<unsigned long long>(pos) < key_cap) keys[pos] = slot_key | ci | cja;
          pos = warp_append(hb, &stats->candidates);
          if (pos >= 0 && static_cast<unsigned long long>(pos) < key_cap) keys[pos] = slot_key | ci | cjb;
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mine = fmin(mine, __shfl_xor_sync(kFull, mine, o));
      close = fmin(close, __shfl_xor_sync(kFull, close, o));
    }
    if (lane == 0) {
      tests += static_cast<unsigned long long>(nv1 * nu1) * (nv2 * nu2);
      if (mine < pos_inf<double>()) atomicMin(&stats->lb_bits, static_cast<unsigned long long>(__double_as_longlong(mine)));
      if (close < pos_inf<double>())
        atomicMin(&stats->ub_bits, static_cast<unsigned long long>(__double_as_longlong(close)));
    }
  }
  if (lane == 0) atomicAdd(&stats->pair_tests, tests);
}

__global__ void k_inter_prep(const unsigned long long *keys, long long n, int ij_bits, unsigned long long *key2,
                             int *idx, unsigned *flag1) {
  const unsigned long long mij = (1ull << ij_bits) - 1ull;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const unsigned long long k = keys[q];
    const unsigned long long slot = k >> (2 * ij_bits);
    key2[q] = (slot << ij_bits) | (k & mij);
    idx[q] = static_cast<int>(q);
    flag1[q] = (q == 0 || (keys[q - 1] >> ij_bits) != (k >> ij_bits)) ? 1u : 0u;
  }
}

__global__ void k_flag_runs(const unsigned long long *sorted, long long n, unsigned *flags) {
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x)
    flags[q] = (q == 0 || sorted[q - 1] != sorted[q]) ? 1u : 0u;
}

// Side 1: pair q (sorted by (slot, i, j)) -> region id ex1[q] + flag1[q] - 1.
template <typename T>
__global__ void k_inter_side1(const unsigned long long *keys, long long n, int ij_bits, const unsigned *flag1,
                              const unsigned *ex1, SideRound<T> cur, const int *map1, RegionRec<T> *next,
                              int *nmap1, int cover) {
  const unsigned long long mij = (1ull << ij_bits) - 1ull;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int id = static_cast<int>(ex1[q] + flag1[q]) - 1;
    nmap1[q] = id;
    if (flag1[q]) {
      const unsigned long long k = keys[q];
      const int slot = static_cast<int>(k >> (2 * ij_bits));
      const int i = static_cast<int>((k >> ij_bits) & mij);
      next[id] = cover ? child_rect_cover(cur.regions[map1[slot]], cur.g.nuv, i)
                       : child_rect(cur.regions[map1[slot]], cur.g.nuv, i);
    }
  }
}

// Side 2: sorted (slot, j) keys with their pair index.
template <typename T>
__global__ void k_inter_side2(const unsigned long long *key2s, const int *idxs, long long n, int ij_bits,
                              const unsigned *flag2, const unsigned *ex2, SideRound<T> cur, const int *map2,
                              RegionRec<T> *next, int *nmap2, int cover) {
  const unsigned long long mij = (1ull << ij_bits) - 1ull;
  for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < n;
       p += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int id = static_cast<int>(ex2[p] + flag2[p]) - 1;
    nmap2[idxs[p]] = id;
    if (flag2[p]) {
      const unsigned long long k = key2s[p];
      const int slot = static_cast<int>(k >> ij_bits);
      const int j = static_cast<int>(k & mij);
      next[id] = cover ? child_rect_cover(cur.regions[map2[slot]], cur.g.nuv, j)
                       : child_rect(cur.regions[map2[slot]], cur.g.nuv, j);
    }
  }
}

// ---------------------------------------------------------------------------
// FP32-screen form: FP32 positions from FP64 basis tables, FP64 re-check
// ---------------------------------------------------------------------------

// P of one sample in FP32: the FP64 basis values (the same tables the FP64
// form uses) are rounded to FP32 and contracted with FMAs against the FP32
// control net; rational surfaces divide by the weight in FP64.  The host
// bounds |P32 - P64| per coordinate from the operation count.
__device__ __forceinline__ Vec4<float> screen_point(const SurfView<float> &s, int spanu, const double *Nu, int spanv,
                                                    const double *Nv) {
  Vec4<float> P{0.0f, 0.0f, 0.0f, 0.0f};
  if (s.zero) return P;
  const int cu0 = spanu - s.degu, cv0 = spanv - s.degv;
  float ax = 0.0f, ay = 0.0f, az = 0.0f, aw = 0.0f;
  for (int rr = 0; rr <= s.degv; ++rr) {
    const Vec4<float> *cp = s.cpw + static_cast<long long>(s.ncpu) * (cv0 + rr) + cu0;
    float rx = 0.0f, ry = 0.0f, rz = 0.0f, rw = 0.0f;
    for (int c = 0; c <= s.degu; ++c) {
      const Vec4<float> v = cp[c];
      float n = __double2float_rn(Nu[c]);
      if (s.rat) {
        n = __fmul_rn(n, v.w);
        rw = __fadd_rn(rw, n);
      }
      rx = __fmaf_rn(n, v.x, rx);
      ry = __fmaf_rn(n, v.y, ry);
      rz = __fmaf_rn(n, v.z, rz);
    }
    const float m = __double2float_rn(Nv[rr]);
    ax = __fmaf_rn(m, rx, ax);
    ay = __fmaf_rn(m, ry, ay);
    az = __fmaf_rn(m, rz, az);
    aw = __fmaf_rn(m, rw, aw);
  }
  if (s.rat) {
    const double w = static_cast<double>(aw);
    P.x = __double2float_rn(static_cast<double>(ax) / w);
    P.y = __double2float_rn(static_cast<double>(ay) / w);
    P.z = __double2float_rn(static_cast<double>(az) / w);
  } else {
    P.x = ax;
    P.y = ay;
    P.z = az;
  }
  return P;
}

__global__ void k_samples_screen(SurfView<float> s, const SurfView<float> *vdev, SideRound<double> basis_side,
                                 SideRound<float> out, long long qs) {
  const long long qo = qoff(qs);
  if (vdev) s = *qsh(vdev, qo);
  basis_side = qsh(basis_side, qo);
  out = qsh(out, qo);
  const Geom g = basis_side.g;
  const int nuv = g.nuv;
  const long long per = static_cast<long long>(nuv) * nuv;
  const long long total = per * nreg_of(basis_side);
  const int p1 = g.p1max;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(t / per);
    const int q = static_cast<int>(t - static_cast<long long>(r) * per);
    const int idx = q % nuv, idy = q / nuv;
    const long long lu = (static_cast<long long>(r) * 2 + 0) * nuv + idx;
    const long long lv = (static_cast<long long>(r) * 2 + 1) * nuv + idy;
    out.samples[t] = screen_point(s, basis_side.spans[lu], basis_side.basis + lu * 3 * p1, basis_side.spans[lv],
                                  basis_side.basis + lv * 3 * p1);
  }
}

// ---- FP32 screen of the intersection query ---------------------------------
//
// Samples, curvature terms, cell boxes and the overlap screen of a round in
// FP32; everything the FP64 form's decisions depend on is recovered exactly
// (see k_iscreen_samples, k_kmax_recheck, k_inter_verify_cells).

// |sum of a basis row| bound: sum_c |N_c| over the p+1 non-zero functions of
// one grid line, in double, for the per-sample error bounds.
__device__ __forceinline__ double abs_row_sum(const double *N, int p) {
  double s = 0.0;
  for (int c = 0; c <= p; ++c) s += fabs(N[c]);
  return s;
}

// FP32 samples of one side's regions from the FP64 basis tables (rounded to
// FP32 and contracted with FMAs against the FP32 control net, as
// screen_point does; rational sums are divided in FP64).  With need_k the
// curvature terms of compute_K (common.cu:155-161: max-abs component of Puu,
// Puv, Pvv) are formed from the same FP32 homogeneous sums, each with a
// rigorous bound d of its distance to the FP64 form's value:
//  * every homogeneous sum h_ab = sum_r sum_c N^(a)_c N^(b)_r (w P, w)_rc is
//    within g * S^(a)_u * S^(b)_v * max|w P| (max w for the weight channel) of
//    the FP64 form's sum, where S = sum |N| over a basis row and
//    g = gamma_n(u32) + gamma_n(u64), n = p + q + 6 roundings on either chain;
//  * rational surfaces propagate those bounds through the quotient rule
//    (S W = H, Su W = Hu - Wu S, Suu W = Huu - 2 Wu Su - Wuu S, Suv W = Huv -
//    Wu Sv - Wv Su - Wuv S) with every product of two perturbations kept and
//    W - eW in the denominators, times 1.01 for the FP64 rounding of both
//    quotients.
// khi[t] = (k + d) rounded up per term; klo[3 r + q] = max over the region of
// (k - d) rounded down (float bits; non-negative values order as unsigned).
// Samples whose bound cannot be formed (W - eW <= 0, non-finite sums) get an
// infinite khi, so k_kmax_recheck re-evaluates them.
struct IScreenConst {
  double g;         // gamma_n(u32) + gamma_n(u64), with margin
  double cmax[3];   // max |control point coordinate|
  double wcmax[3];  // max |w * coordinate| (rational; = cmax otherwise)
  double wmax;      // max weight (rational)
};

template <bool NEEDK>
__global__ void __launch_bounds__(128) k_iscreen_samples(SurfView<float> s, SideRound<double> bs,
                                                         SideRound<float> out, Vec4<float> *khi, unsigned *klo,
                                                         IScreenConst cst) {
  const Geom g = bs.g;
  const int nuv = g.nuv;
  const long long per = static_cast<long long>(nuv) * nuv;
  const long long total = per * bs.nreg;
  const int p1 = g.p1max;
  for (long long base = blockIdx.x * static_cast<long long>(blockDim.x); base < total;
       base += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long t = base + threadIdx.x;
    const bool live = t < total;
    int r = 0;
    float lo3[3] = {0.0f, 0.0f, 0.0f};
    if (live) {
      r = static_cast<int>(t / per);
      const int q = static_cast<int>(t - static_cast<long long>(r) * per);
      const int idx = q % nuv, idy = q / nuv;
      const long long lu = (static_cast<long long>(r) * 2 + 0) * nuv + idx;
      const long long lv = (static_cast<long long>(r) * 2 + 1) * nuv + idy;
      const double *Nu = bs.basis + lu * 3 * p1;
      const double *Nv = bs.basis + lv * 3 * p1;
      const int spanu = bs.spans[lu], spanv = bs.spans[lv];
      if (!NEEDK || s.zero) {
        out.samples[t] = screen_point(s, spanu, Nu, spanv, Nv);
        if (NEEDK) khi[t] = Vec4<float>{0.0f, 0.0f, 0.0f, 0.0f};
      } else {
        // Homogeneous FP32 sums of the six derivative combinations (P, Pu, Pv,
        // Puu, Puv, Pvv) x (x, y, z, w), u sums per control-net row shared by
        // the combinations of one u order.
        float h[6][4];
#pragma unroll
        for (int m = 0; m < 6; ++m) h[m][0] = h[m][1] = h[m][2] = h[m][3] = 0.0f;
        const int cu0 = spanu - s.degu, cv0 = spanv - s.degv;
        for (int rr = 0; rr <= s.degv; ++rr) {
          const Vec4<float> *cp = s.cpw + static_cast<long long>(s.ncpu) * (cv0 + rr) + cu0;
          float R[3][4];
#pragma unroll
          for (int a = 0; a < 3; ++a) R[a][0] = R[a][1] = R[a][2] = R[a][3] = 0.0f;
          for (int c = 0; c <= s.degu; ++c) {
            const Vec4<float> v = cp[c];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              if (a > s.du) break;
              float n = __double2float_rn(Nu[a * p1 + c]);
              if (s.rat) {
                n = __fmul_rn(n, v.w);
                R[a][3] = __fadd_rn(R[a][3], n);
              }
              R[a][0] = __fmaf_rn(n, v.x, R[a][0]);
              R[a][1] = __fmaf_rn(n, v.y, R[a][1]);
              R[a][2] = __fmaf_rn(n, v.z, R[a][2]);
            }
          }
          const float m0 = __double2float_rn(Nv[rr]);
          const float m1 = s.dv >= 1 ? __double2float_rn(Nv[p1 + rr]) : 0.0f;
          const float m2 = s.dv >= 2 ? __double2float_rn(Nv[2 * p1 + rr]) : 0.0f;
          // combination m: (u order, v order) = (0,0) (1,0) (0,1) (2,0) (1,1) (0,2)
#pragma unroll
          for (int ch = 0; ch < 4; ++ch) {
            h[0][ch] = __fmaf_rn(m0, R[0][ch], h[0][ch]);
            h[1][ch] = __fmaf_rn(m0, R[1][ch], h[1][ch]);
            h[2][ch] = __fmaf_rn(m1, R[0][ch], h[2][ch]);
            h[3][ch] = __fmaf_rn(m0, R[2][ch], h[3][ch]);
            h[4][ch] = __fmaf_rn(m1, R[1][ch], h[4][ch]);
            h[5][ch] = __fmaf_rn(m2, R[0][ch], h[5][ch]);
          }
        }
        // Derivative orders above the degree stay zero (evaluation.cu:283,315).
        const int ku[6] = {0, 1, 0, 2, 1, 0}, kv[6] = {0, 0, 1, 0, 1, 2};
        double Su[3], Sv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          Su[a] = a <= s.du ? abs_row_sum(Nu + a * p1, s.degu) * (1.0 + 1e-12) : 0.0;
          Sv[a] = a <= s.dv ? abs_row_sum(Nv + a * p1, s.degv) * (1.0 + 1e-12) : 0.0;
        }
        double eh[6][4];  // bounds of |h32 - h64|
#pragma unroll
        for (int m = 0; m < 6; ++m) {
          const double mag = cst.g * Su[ku[m]] * Sv[kv[m]];
          eh[m][0] = mag * cst.wcmax[0];
          eh[m][1] = mag * cst.wcmax[1];
          eh[m][2] = mag * cst.wcmax[2];
          eh[m][3] = mag * cst.wmax;
        }
        double S[6][3], e[6][3];
        bool ok = true;
        if (!s.rat) {
#pragma unroll
          for (int m = 0; m < 6; ++m)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              S[m][c] = static_cast<double>(h[m][c]);
              e[m][c] = eh[m][c];
            }
        } else {
          const double W = h[0][3], Wu = h[1][3], Wv = h[2][3], Wuu = h[3][3], Wuv = h[4][3], Wvv = h[5][3];
          const double eW = eh[0][3], eWu = eh[1][3], eWv = eh[2][3], eWuu = eh[3][3], eWuv = eh[4][3],
                       eWvv = eh[5][3];
          const double Wl = W - eW;
          ok = Wl > 0.0;
          const double inv = 1.0 / W;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const double F = h[0][c] * inv;
            const double Fu = (h[1][c] - Wu * F) * inv;
            const double Fv = (h[2][c] - Wv * F) * inv;
            const double Fuu = (h[3][c] - 2.0 * Wu * Fu - Wuu * F) * inv;
            const double Fuv = (h[4][c] - Wu * Fv - Wv * Fu - Wuv * F) * inv;
            const double Fvv = (h[5][c] - 2.0 * Wv * Fv - Wvv * F) * inv;
            S[0][c] = F, S[1][c] = Fu, S[2][c] = Fv, S[3][c] = Fuu, S[4][c] = Fuv, S[5][c] = Fvv;
            const double eF = (eh[0][c] + fabs(F) * eW) / Wl;
            const double eFu = (eh[1][c] + fabs(Wu) * eF + fabs(F) * eWu + eWu * eF + fabs(Fu) * eW) / Wl;
            const double eFv = (eh[2][c] + fabs(Wv) * eF + fabs(F) * eWv + eWv * eF + fabs(Fv) * eW) / Wl;
            const double eFuu = (eh[3][c] + 2.0 * (fabs(Wu) * eFu + fabs(Fu) * eWu + eWu * eFu) + fabs(Wuu) * eF +
                                 fabs(F) * eWuu + eWuu * eF + fabs(Fuu) * eW) / Wl;
            const double eFuv = (eh[4][c] + fabs(Wu) * eFv + fabs(Fv) * eWu + eWu * eFv + fabs(Wv) * eFu +
                                 fabs(Fu) * eWv + eWv * eFu + fabs(Wuv) * eF + fabs(F) * eWuv + eWuv * eF +
                                 fabs(Fuv) * eW) / Wl;
            const double eFvv = (eh[5][c] + 2.0 * (fabs(Wv) * eFv + fabs(Fv) * eWv + eWv * eFv) + fabs(Wvv) * eF +
                                 fabs(F) * eWvv + eWvv * eF + fabs(Fvv) * eW) / Wl;
            e[0][c] = eF, e[1][c] = eFu, e[2][c] = eFv, e[3][c] = eFuu, e[4][c] = eFuv, e[5][c] = eFvv;
          }
        }
        Vec4<float> P;
        if (s.rat) {
          // P as screen_point forms it: the FP32 sums divided in FP64.
          const double w = static_cast<double>(h[0][3]);
          P = Vec4<float>{__double2float_rn(static_cast<double>(h[0][0]) / w),
                          __double2float_rn(static_cast<double>(h[0][1]) / w),
                          __double2float_rn(static_cast<double>(h[0][2]) / w), 0.0f};
        } else {
          P = Vec4<float>{h[0][0], h[0][1], h[0][2], 0.0f};
        }
        out.samples[t] = P;
        float hi3[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const int m = 3 + q;
          double kv = 0.0, kd = 0.0;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            kv = fmax(kv, fabs(S[m][c]));
            kd = fmax(kd, e[m][c]);
          }
          kd *= 1.01;
          const bool fin = ok && isfinite(kv) && isfinite(kd);
          lo3[q] = fin ? fmaxf(__double2float_rd(kv - kd), 0.0f) : 0.0f;
          hi3[q] = fin ? __double2float_ru(kv + kd) : pos_inf<float>();
        }
        khi[t] = Vec4<float>{hi3[0], hi3[1], hi3[2], 0.0f};
      }
    }
    if (NEEDK) {
      // Region maxima of the lower bounds: warp maximum when every live lane
      // shares the region, else per lane.
      const int r0 = __shfl_sync(kFull, r, 0);
      const bool uniform = __all_sync(kFull, (!live) || r == r0);
      if (uniform) {
#pragma unroll
        for (int q = 0; q < 3; ++q)
          for (int o = 16; o > 0; o >>= 1) lo3[q] = fmaxf(lo3[q], __shfl_xor_sync(kFull, lo3[q], o));
        if ((threadIdx.x & 31) == 0)
#pragma unroll
          for (int q = 0; q < 3; ++q) atomicMax(&klo[3 * r0 + q], __float_as_uint(lo3[q]));
      } else if (live) {
#pragma unroll
        for (int q = 0; q < 3; ++q) atomicMax(&klo[3 * r + q], __float_as_uint(lo3[q]));
      }
    }
  }
}

// Exact compute_K maxima from the FP32 bounds: every sample's FP64 term lies
// in [lo, hi], so the FP64 maximum of a region is at least the largest lo
// and is reached only at samples with hi >= that.  Those samples are
// evaluated in FP64 with the FP64 form's code (eval_record), and their terms
// folded with the same atomic maximum: the result equals the FP64 form's
// bits.  count gets the number of samples re-evaluated.
__global__ void k_kmax_recheck(SurfView<double> s, SideRound<double> bs, const Vec4<float> *khi,
                               const unsigned *klo, unsigned long long *count) {
  const Geom g = bs.g;
  const int nuv = g.nuv;
  const long long per = static_cast<long long>(nuv) * nuv;
  const long long total = per * bs.nreg;
  const int p1 = g.p1max;
  unsigned long long mine = 0;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(t / per);
    const Vec4<float> hb = khi[t];
    const bool cand = hb.x >= __uint_as_float(klo[3 * r]) || hb.y >= __uint_as_float(klo[3 * r + 1]) ||
                      hb.z >= __uint_as_float(klo[3 * r + 2]);
    if (!cand) continue;
    ++mine;
    const int q = static_cast<int>(t - static_cast<long long>(r) * per);
    const int idx = q % nuv, idy = q / nuv;
    const long long lu = (static_cast<long long>(r) * 2 + 0) * nuv + idx;
    const long long lv = (static_cast<long long>(r) * 2 + 1) * nuv + idy;
    double rec[18];
    eval_record(s, bs.spans[lu], bs.basis + lu * 3 * p1, bs.spans[lv], bs.basis + lv * 3 * p1, p1, rec);
    // max-abs component of Puu, Puv, Pvv (common.cu:155-161), as k_samples
    atomic_max_bits(&bs.kmax[3 * r + 0], tmax(fabs(rec[9]), tmax(fabs(rec[10]), fabs(rec[11]))));
    atomic_max_bits(&bs.kmax[3 * r + 1], tmax(fabs(rec[12]), tmax(fabs(rec[13]), fabs(rec[14]))));
    atomic_max_bits(&bs.kmax[3 * r + 2], tmax(fabs(rec[15]), tmax(fabs(rec[16]), fabs(rec[17]))));
  }
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, mine);
}

// FP64 re-check from the FP64 cells of the round (the FP64 form's centres and
// half spans, from its position-only samples): the strict test of
// intersection.cu:60-62 in the FP64 leaf's operation order, per candidate key.
__global__ void __launch_bounds__(128) k_inter_verify_cells(SideRound<double> a, SideRound<double> b,
                                                            const int *map1, const int *map2,
                                                            const unsigned long long *keys, unsigned long long n,
                                                            int ij_bits, unsigned long long *out,
                                                            unsigned long long cap, ScreenStats *stats) {
  const unsigned long long mij = (1ull << ij_bits) - 1ull;
  auto at = [](const SideRound<double> &sr, int r, int cell) {
    const Geom &g = sr.g;
    const int iv = cell / g.W, iu = cell - (cell / g.W) * g.W;
    const int ty = iv / g.te, tx = iu / g.te;
    return (static_cast<long long>(r) * g.ntiles + ty * g.tw + tx) * (g.te * g.te) + (iv - ty * g.te) * g.te +
           (iu - tx * g.te);
  };
  for (unsigned long long base = blockIdx.x * static_cast<unsigned long long>(blockDim.x); base < n;
       base += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
    const unsigned long long q = base + threadIdx.x;
    bool keep = false;
    unsigned long long key = 0;
    if (q < n) {
      key = keys[q];
      const int slot = static_cast<int>(key >> (2 * ij_bits));
      const int i = static_cast<int>((key >> ij_bits) & mij), j = static_cast<int>(key & mij);
      const int r1 = map1[slot], r2 = map2[slot];
      const long long i1 = at(a, r1, i), i2 = at(b, r2, j);
      const Vec4<double> c1 = a.center[i1], c2 = b.center[i2];
      Vec4<double> r1v = a.half[i1], r2v = b.half[i2];
      const double p1 = a.pad[r1], p2 = b.pad[r2];
      r1v.x = r1v.x + p1;
      r1v.y = r1v.y + p1;
      r1v.z = r1v.z + p1;
      r2v.x = r2v.x + p2;
      r2v.y = r2v.y + p2;
      r2v.z = r2v.z + p2;
      keep = fabs(c1.x - c2.x) < (r1v.x + r2v.x) && fabs(c1.y - c2.y) < (r1v.y + r2v.y) &&
             fabs(c1.z - c2.z) < (r1v.z + r2v.z);
    }
    const long long pos = warp_append(keep, &stats->checked);
    if (pos >= 0 && static_cast<unsigned long long>(pos) < cap) out[pos] = key;
  }
}

// Distance cells without a sample grid in HBM: one warp per tile evaluates
// the tile's (te + 1)^2 corner samples into shared memory, then forms the
// tile's cell centres and centre range exactly as k_cells does.
// TB = precision of the basis tables, TC = of the samples and cells
// (TB = double, TC = float: the FP32 screen).
//
// The samples are evaluated in factored form: all samples of a tile column
// share the u span and u basis, so the u-direction sum of every control-net
// row the tile needs is formed once per (row, column) and then combined in v
// per sample.  Each of those sums and each v accumulation is the same
// operation sequence as in eval_point / screen_point, so the samples carry
// the same bits; tiles whose rows exceed the shared-memory table (or degrees
// above 8, MAXP > 9) take the per-sample path.
template <typename TB, typename TC, int MAXP>
__global__ void __launch_bounds__(128) k_cells_fused(SurfView<TC> s, const SurfView<TC> *vdev, SideRound<TB> bs,
                                                     SideRound<TC> out, long long qs) {
  constexpr int kE = kMaxTile + 1;       // samples per tile edge
  constexpr int kRows = 16;              // control-net rows of the row-sum table
  constexpr bool kFactor = MAXP <= 9;
  constexpr int kNB = kFactor ? MAXP : 1;
  constexpr int kNR = kFactor ? kRows : 1;
  using TN = TC;                         // basis values as the contraction uses them
  constexpr int kW = 4;                  // warps per block (one tile each)
  __shared__ Vec4<TC> smp[kW][kE * kE];
  __shared__ Vec4<TC> rsum[kW][kNR][kE];
  __shared__ TN snu[kW][kE][kNB], snv[kW][kE][kNB];
  __shared__ int ssu[kW][kE], ssv[kW][kE];
  const long long qo = qoff(qs);
  if (vdev) s = *qsh(vdev, qo);
  bs = qsh(bs, qo);
  out = qsh(out, qo);
  const Geom g = out.g;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int te2 = g.te * g.te;
  const int p1 = g.p1max;
  Vec4<TC> *S = smp[wib];
  const long long ntile_total = static_cast<long long>(nreg_of(bs)) * g.ntiles;
  const long long nwarps = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long t = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; t < ntile_total;
       t += nwarps) {
    const int r = static_cast<int>(t / g.ntiles);
    const int tile = static_cast<int>(t - static_cast<long long>(r) * g.ntiles);
    const int ty = tile / g.tw, tx = tile - (tile / g.tw) * g.tw;
    const int nv = min(g.te, g.W - ty * g.te), nu = min(g.te, g.W - tx * g.te);
    const int sw = nu + 1, ns = (nv + 1) * sw;
    const long long lu0 = (static_cast<long long>(r) * 2 + 0) * g.nuv + tx * g.te;
    const long long lv0 = (static_cast<long long>(r) * 2 + 1) * g.nuv + ty * g.te;
    bool factored = false;
    int rmin = 0;
    if constexpr (kFactor) {
      if (!s.zero) {
        // Spans and basis values of the tile's sample columns (lanes 0..nu)
        // and rows (lanes 16..16+nv), converted as the contraction uses them.
        if (lane <= nu) {
          ssu[wib][lane] = bs.spans[lu0 + lane];
          const TB *N = bs.basis + (lu0 + lane) * 3 * p1;
          for (int c = 0; c <= s.degu; ++c) {
            if constexpr (std::is_same<TB, TC>::value) snu[wib][lane][c] = N[c];
            else snu[wib][lane][c] = __double2float_rn(N[c]);
          }
        }
        if (lane >= 16 && lane - 16 <= nv) {
          const int a = lane - 16;
          ssv[wib][a] = bs.spans[lv0 + a];
          const TB *N = bs.basis + (lv0 + a) * 3 * p1;
          for (int c = 0; c <= s.degv; ++c) {
            if constexpr (std::is_same<TB, TC>::value) snv[wib][a][c] = N[c];
            else snv[wib][a][c] = __double2float_rn(N[c]);
          }
        }
        __syncwarp();
        int lo = INT_MAX, hi = INT_MIN;
        for (int a = 0; a <= nv; ++a) {
          lo = min(lo, ssv[wib][a]);
          hi = max(hi, ssv[wib][a]);
        }
        rmin = lo - s.degv;
        const int nrows = hi - rmin + 1;
        factored = nrows <= kRows;
        if (factored) {
          // u-direction sums of every needed control-net row and column.
          for (int it = lane; it < nrows * sw; it += 32) {
            const int R = it / sw, b = it - (it / sw) * sw;
            const Vec4<TC> *cp = s.cpw + static_cast<long long>(s.ncpu) * (rmin + R) + (ssu[wib][b] - s.degu);
            const TN *Nu = snu[wib][b];
            TC r0 = TC(0), r1 = TC(0), r2 = TC(0), r3 = TC(0);
            for (int c = 0; c <= s.degu; ++c) {
              const Vec4<TC> q = cp[c];
              if constexpr (std::is_same<TB, TC>::value) {
                if (!s.rat) {
                  const TC n = Nu[c];
                  r0 += n * q.x;
                  r1 += n * q.y;
                  r2 += n * q.z;
                } else {
                  const TC nw = Nu[c] * q.w;
                  r0 += nw * q.x;
                  r1 += nw * q.y;
                  r2 += nw * q.z;
                  r3 += nw;
                }
              } else {
                float n = Nu[c];
                if (s.rat) {
                  n = __fmul_rn(n, q.w);
                  r3 = __fadd_rn(r3, n);
                }
                r0 = __fmaf_rn(n, q.x, r0);
                r1 = __fmaf_rn(n, q.y, r1);
                r2 = __fmaf_rn(n, q.z, r2);
              }
            }
            rsum[wib][R][b] = Vec4<TC>{r0, r1, r2, r3};
          }
          __syncwarp();
          // v-direction combination per sample.
          for (int l = lane; l < ns; l += 32) {
            const int a = l / sw, b = l - (l / sw) * sw;
            const int R0 = ssv[wib][a] - s.degv - rmin;
            const TN *Nv = snv[wib][a];
            TC a0 = TC(0), a1 = TC(0), a2 = TC(0), a3 = TC(0);
            for (int rr = 0; rr <= s.degv; ++rr) {
              const Vec4<TC> row = rsum[wib][R0 + rr][b];
              const TC m = Nv[rr];
              if constexpr (std::is_same<TB, TC>::value) {
                a0 += m * row.x;
                a1 += m * row.y;
                a2 += m * row.z;
                a3 += m * row.w;
              } else {
                a0 = __fmaf_rn(m, row.x, a0);
                a1 = __fmaf_rn(m, row.y, a1);
                a2 = __fmaf_rn(m, row.z, a2);
                a3 = __fmaf_rn(m, row.w, a3);
              }
            }
            Vec4<TC> P{a0, a1, a2, TC(0)};
            if (s.rat) {
              if constexpr (std::is_same<TB, TC>::value) {
                const TC inv = TC(1) / a3;
                P.x = a0 * inv;
                P.y = a1 * inv;
                P.z = a2 * inv;
              } else {
                const double w = static_cast<double>(a3);
                P.x = __double2float_rn(static_cast<double>(a0) / w);
                P.y = __double2float_rn(static_cast<double>(a1) / w);
                P.z = __double2float_rn(static_cast<double>(a2) / w);
              }
            }
            S[l] = P;
          }
        }
      }
    }
    if (!factored) {
      for (int l = lane; l < ns; l += 32) {
        const int a = l / sw, b = l - (l / sw) * sw;
        const long long lu = lu0 + b, lv = lv0 + a;
        const TB *Nu = bs.basis + lu * 3 * p1;
        const TB *Nv = bs.basis + lv * 3 * p1;
        Vec4<TC> P;
        if constexpr (std::is_same<TB, TC>::value) {
          TC q[3];
          eval_point(s, bs.spans[lu], Nu, bs.spans[lv], Nv, q);
          P = Vec4<TC>{q[0], q[1], q[2], TC(0)};
        } else {
          P = screen_point(s, bs.spans[lu], Nu, bs.spans[lv], Nv);
        }
        S[l] = P;
      }
    }
    __syncwarp();
    TC lo[3] = {pos_inf<TC>(), pos_inf<TC>(), pos_inf<TC>()};
    TC hi[3] = {-pos_inf<TC>(), -pos_inf<TC>(), -pos_inf<TC>()};
    for (int local = lane; local < te2; local += 32) {
      const int a = local / g.te, b = local - (local / g.te) * g.te;
      Vec4<TC> cen{TC(0), TC(0), TC(0), TC(0)};
      if (a < nv && b < nu) {
        const Vec4<TC> p0 = S[a * sw + b];
        const Vec4<TC> p1v = S[a * sw + b + 1];
        const Vec4<TC> p2 = S[(a + 1) * sw + b];
        const Vec4<TC> p3 = S[(a + 1) * sw + b + 1];
        const TC lx = fmn(p0.x, fmn(p1v.x, fmn(p2.x, p3.x)));
        const TC ly = fmn(p0.y, fmn(p1v.y, fmn(p2.y, p3.y)));
        const TC lz = fmn(p0.z, fmn(p1v.z, fmn(p2.z, p3.z)));
        const TC hx = fmx(p0.x, fmx(p1v.x, fmx(p2.x, p3.x)));
        const TC hy = fmx(p0.y, fmx(p1v.y, fmx(p2.y, p3.y)));
        const TC hz = fmx(p0.z, fmx(p1v.z, fmx(p2.z, p3.z)));
        cen.x = (lx - TC(0) + hx + TC(0)) / TC(2);
        cen.y = (ly - TC(0) + hy + TC(0)) / TC(2);
        cen.z = (lz - TC(0) + hz + TC(0)) / TC(2);
        lo[0] = fmn(lo[0], cen.x);
        lo[1] = fmn(lo[1], cen.y);
        lo[2] = fmn(lo[2], cen.z);
        hi[0] = fmx(hi[0], cen.x);
        hi[1] = fmx(hi[1], cen.y);
        hi[2] = fmx(hi[2], cen.z);
      }
      out.center[t * te2 + local] = cen;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        lo[c] = fmn(lo[c], __shfl_xor_sync(kFull, lo[c], o));
        hi[c] = fmx(hi[c], __shfl_xor_sync(kFull, hi[c], o));
      }
    }
    if (lane == 0) {
      out.tlo[t] = Vec4<TC>{lo[0], lo[1], lo[2], TC(0)};
      out.thi[t] = Vec4<TC>{hi[0], hi[1], hi[2], TC(0)};
      if (out.stmin) fold_supertile(out, r, ty, tx, lo, hi);
    }
    __syncwarp();
  }
}

// Distance cells without a sample grid in HBM.  One block per (region, band
// of te cell rows, chunk of up to 32 tiles along u): the block evaluates the
// band's (te + 1) x (32 te + 1) corner samples into shared memory, then one
// warp per tile forms the tile's cell centres and centre range exactly as
// k_cells does.  TB = precision of the basis tables, TC = of the samples and
// cells (TB = double, TC = float: the FP32 screen).
//
// Samples are evaluated in factored form: a thread owns one sample column
// (its u span and u basis), forms the u-direction sum of every control-net
// row the band needs in registers, and combines them in v for each sample
// row.  Each u sum and each v accumulation is the same operation sequence as
// in eval_point / screen_point, so the samples carry the same bits.  The
// kernel is compiled for degrees <= D in both directions (loops of fixed trip
// count); bands needing more than D + 3 net rows (coarse grids) take the
// per-sample path.
constexpr int kBandTiles = 32;
constexpr int kBandCols = kBandTiles * kMaxTile + 1;
constexpr int kBandThreads = 288;  // one thread per sample column (257) in one pass
static_assert(kBandThreads == kBandTiles * kMaxTile + 32, "band cells: 8 warps of cell columns + 1 warp");
constexpr int kBandNetCols = 96;   // control-net columns a band's net tile holds
constexpr int kBandNetRows = 6;    // net rows of the tile (D + 3 for D = 3)

template <typename TC>
constexpr size_t band_smem() {
  return sizeof(Vec4<TC>) * ((kMaxTile + 1) * kBandCols + kBandNetRows * kBandNetCols);
}

// Arithmetic of the factored band evaluation, one helper per step, with the
// operation sequence of eval_point (TB == TC) or screen_point (TB = double,
// TC = float) for a net row's u sum, a sample's v accumulation and the
// rational quotient.
template <typename TB, typename TC, bool RAT>
__device__ __forceinline__ void band_row_sum(TC n, const Vec4<TC> &q, TC (&r)[4]) {
  if constexpr (std::is_same<TB, TC>::value) {
    if constexpr (!RAT) {
      r[0] += n * q.x;
      r[1] += n * q.y;
      r[2] += n * q.z;
    } else {
      const TC nw = n * q.w;
      r[0] += nw * q.x;
      r[1] += nw * q.y;
      r[2] += nw * q.z;
      r[3] += nw;
    }
  } else {
    float m = n;
    if constexpr (RAT) {
      m = __fmul_rn(m, q.w);
      r[3] = __fadd_rn(r[3], m);
    }
    r[0] = __fmaf_rn(m, q.x, r[0]);
    r[1] = __fmaf_rn(m, q.y, r[1]);
    r[2] = __fmaf_rn(m, q.z, r[2]);
  }
}

template <typename TB, typename TC, bool RAT>
__device__ __forceinline__ void band_v_acc(TC m, const TC (&rs)[4], TC (&a)[4]) {
  if constexpr (std::is_same<TB, TC>::value) {
    a[0] += m * rs[0];
    a[1] += m * rs[1];
    a[2] += m * rs[2];
    if constexpr (RAT) a[3] += m * rs[3];
  } else {
    a[0] = __fmaf_rn(m, rs[0], a[0]);
    a[1] = __fmaf_rn(m, rs[1], a[1]);
    a[2] = __fmaf_rn(m, rs[2], a[2]);
    if constexpr (RAT) a[3] = __fmaf_rn(m, rs[3], a[3]);
  }
}

template <typename TB, typename TC, bool RAT>
__device__ __forceinline__ Vec4<TC> band_point(const TC (&a)[4]) {
  Vec4<TC> P{a[0], a[1], a[2], TC(0)};
  if constexpr (RAT) {
    if constexpr (std::is_same<TB, TC>::value) {
      const TC inv = TC(1) / a[3];
      P.x = a[0] * inv;
      P.y = a[1] * inv;
      P.z = a[2] * inv;
    } else {
      const double w = static_cast<double>(a[3]);
      P.x = __double2float_rn(static_cast<double>(a[0]) / w);
      P.y = __double2float_rn(static_cast<double>(a[1]) / w);
      P.z = __double2float_rn(static_cast<double>(a[2]) / w);
    }
  }
  return P;
}

// One band unit of k_cells_band when both degrees equal D and the band's
// control-net tile (NR rows, rows past the band's own zero-filled) sits in
// shared memory.  Every predicate of the general loop is a compile-time
// constant here.
//
// Samples: threads 0..255 own sample columns 0..255 (all rows of the band);
// the last column (256) goes to warp 8, one lane per sample row, each lane
// forming the column's row sums itself (the same operations, so the same
// bits).  Cells: thread c owns cell column c of the chunk (tile c / 8,
// column c % 8 of it) and walks its te cell rows, carrying the previous
// sample row's pairwise min/max, so a cell costs two shared loads.  The
// tile range is an 8-lane reduction.  min/max are exact and, with fminf /
// fmaxf, independent of order (NaNs are skipped, and the sign of a zero
// extreme is erased by the centre's trailing + 0, which also keeps every
// centre off -0), so the centres and ranges carry the general loop's bits.
template <typename TB, typename TC, int D, int NR, bool RAT>
__device__ __forceinline__ void band_unit_fast(const SideRound<TC> &out, Vec4<TC> *S, const Vec4<TC> *NT,
                                               const TC (*coef)[8], int r, int ty, int tx0, int ntx, int nv,
                                               int ncols, int cu0, int su, const TC (&Nu)[D + 1]) {
  constexpr int kP = D + 1;
  constexpr int te = kMaxTile, te2 = kMaxTile * kMaxTile;
  constexpr int kCols = kBandTiles * kMaxTile;  // 256 cell columns, 257 sample columns
  const Geom g = out.g;
  const int tid = threadIdx.x;
  int col, a0, a1;
  if (tid < kCols) {
    col = tid;
    a0 = 0;
    a1 = nv;
  } else {
    col = kCols;
    a0 = a1 = tid - kCols;
    if (a0 > nv) col = ncols;  // idle lane
  }
  if (col < ncols) {
    TC rs[NR][4];
    const Vec4<TC> *cp = NT + (su - D - cu0);
#pragma unroll
    for (int R = 0; R < NR; ++R) {
      TC acc[4] = {TC(0), TC(0), TC(0), TC(0)};
#pragma unroll
      for (int c = 0; c < kP; ++c) band_row_sum<TB, TC, RAT>(Nu[c], cp[R * kBandNetCols + c], acc);
#pragma unroll
      for (int k = 0; k < 4; ++k) rs[R][k] = acc[k];
    }
    for (int a = a0; a <= a1; ++a) {
      TC m[NR];
      if constexpr (sizeof(TC) == 4) {
        const float4 v0 = *reinterpret_cast<const float4 *>(&coef[a][0]);
        m[0] = v0.x;
        m[1] = v0.y;
        m[2] = v0.z;
        m[3] = v0.w;
        if constexpr (NR > 4) {
          const float2 v1 = *reinterpret_cast<const float2 *>(&coef[a][4]);
          m[4] = v1.x;
          if constexpr (NR > 5) m[5] = v1.y;
        }
      } else {
#pragma unroll
        for (int R = 0; R < NR; ++R) m[R] = coef[a][R];
      }
      TC acc[4] = {TC(0), TC(0), TC(0), TC(0)};
#pragma unroll
      for (int R = 0; R < NR; ++R) band_v_acc<TB, TC, RAT>(m[R], rs[R], acc);
      S[a * kBandCols + col] = band_point<TB, TC, RAT>(acc);
    }
  }
  __syncthreads();
  if (tid >= kCols) return;  // warp 8: no cells (a whole warp, so the shuffles below stay converged)
  const int j = tid >> 3, b = tid & 7;
  const bool act = j < ntx;
  TC tlo[3] = {pos_inf<TC>(), pos_inf<TC>(), pos_inf<TC>()};
  TC thi[3] = {-pos_inf<TC>(), -pos_inf<TC>(), -pos_inf<TC>()};
  const int tx = tx0 + j;
  const long long t = static_cast<long long>(r) * g.ntiles + static_cast<long long>(ty) * g.tw + tx;
  if (act) {
    const bool colok = b < min(te, g.W - tx * te);
    Vec4<TC> p = S[tid], q = S[tid + 1];
    TC pmn[3] = {fmn(p.x, q.x), fmn(p.y, q.y), fmn(p.z, q.z)};
    TC pmx[3] = {fmx(p.x, q.x), fmx(p.y, q.y), fmx(p.z, q.z)};
    Vec4<TC> *dst = out.center + t * te2 + b;
#pragma unroll
    for (int a = 0; a < te; ++a) {
      p = S[(a + 1) * kBandCols + tid];
      q = S[(a + 1) * kBandCols + tid + 1];
      const TC nmn[3] = {fmn(p.x, q.x), fmn(p.y, q.y), fmn(p.z, q.z)};
      const TC nmx[3] = {fmx(p.x, q.x), fmx(p.y, q.y), fmx(p.z, q.z)};
      Vec4<TC> cen{TC(0), TC(0), TC(0), TC(0)};
      if (a < nv && colok) {
        TC c3[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const TC lo = fmn(pmn[k], nmn[k]), hi = fmx(pmx[k], nmx[k]);
          c3[k] = (lo - TC(0) + hi + TC(0)) * TC(0.5);  // = / 2 exactly
          tlo[k] = fmn(tlo[k], c3[k]);
          thi[k] = fmx(thi[k], c3[k]);
        }
        cen = Vec4<TC>{c3[0], c3[1], c3[2], TC(0)};
      }
      dst[a * te] = cen;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        pmn[k] = nmn[k];
        pmx[k] = nmx[k];
      }
    }
  }
#pragma unroll
  for (int o = 1; o < te; o <<= 1) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      tlo[k] = fmn(tlo[k], __shfl_xor_sync(kFull, tlo[k], o));
      thi[k] = fmx(thi[k], __shfl_xor_sync(kFull, thi[k], o));
    }
  }
  if (act && b == 0) {
    out.tlo[t] = Vec4<TC>{tlo[0], tlo[1], tlo[2], TC(0)};
    out.thi[t] = Vec4<TC>{thi[0], thi[1], thi[2], TC(0)};
    if (out.stmin) fold_supertile(out, r, ty, tx, tlo, thi);
  }
}

template <typename TB, typename TC, int D>
__global__ void __launch_bounds__(kBandThreads, sizeof(TC) == 8 ? 2 : 4) k_cells_band(SurfView<TC> s, const SurfView<TC> *vdev,
                                                              SideRound<TB> bs, SideRound<TC> out, long long qs) {
  constexpr int kE = kMaxTile + 1;
  constexpr int kP = D + 1;          // u basis values held per thread
  constexpr int kBandRows = D + 3;   // net rows held per thread
  static_assert(kBandRows <= kBandNetRows, "net tile rows");
  extern __shared__ __align__(16) unsigned char band_raw[];
  Vec4<TC> *S = reinterpret_cast<Vec4<TC> *>(band_raw);  // [kE][kBandCols]
  // The band's control-net tile: rows rmin.., columns cu0.. of the net.
  Vec4<TC> *NT = S + kE * kBandCols;                      // [kBandNetRows][kBandNetCols]
  // v coefficients of each sample row over the band's net rows, zero outside
  // the row's degv + 1 window: adding 0 * (finite row sum) to an accumulator
  // that starts at +0 (and so is never -0) leaves it unchanged, so the padded
  // sum has the bits of the windowed one.
  __shared__ __align__(16) TC coef[kE][8];
  const long long qo = qoff(qs);
  if (vdev) s = *qsh(vdev, qo);
  bs = qsh(bs, qo);
  out = qsh(out, qo);
  const Geom g = out.g;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // Large grids only (tw >= 16, so te = kMaxTile): the tile edge is a
  // compile-time constant and cell indices are shifts and masks.
  constexpr int te = kMaxTile, te2 = kMaxTile * kMaxTile;
  const int p1 = g.p1max;
  const int nch = (g.tw + kBandTiles - 1) / kBandTiles;
  // Units per side: regions x tw x nch, far below 2^31 (32-bit index
  // arithmetic; a 64-bit division per unit would cost every thread ~100
  // instructions).
  const int per_reg = g.tw * nch;
  const int nunits = nreg_of(bs) * per_reg;
  for (int unit = blockIdx.x; unit < nunits; unit += gridDim.x) {
    const int r = unit / per_reg;
    const int rest = unit - r * per_reg;
    const int ty = rest / nch, ch = rest - ty * nch;
    const int tx0 = ch * kBandTiles, ntx = min(kBandTiles, g.tw - tx0);
    const int nv = min(te, g.W - ty * te);
    const int nuc = min(ntx * te, g.W - tx0 * te);
    const int ncols = nuc + 1;
    const long long lu0 = (static_cast<long long>(r) * 2 + 0) * g.nuv + tx0 * te;
    const long long lv0 = (static_cast<long long>(r) * 2 + 1) * g.nuv + ty * te;
    const bool fit = !s.zero && s.degu <= D && s.degv <= D;
    int rmin = 0, nrows = kBandRows + 1, cu0 = 0, ncu = kBandNetCols + 1;
    if (fit) {
      // Spans are monotone along the band's sample rows and columns: the end
      // rows and columns give the net rows and columns the band reads.
      const int v0 = bs.spans[lv0], v1 = bs.spans[lv0 + nv];
      const int u0 = bs.spans[lu0], u1 = bs.spans[lu0 + ncols - 1];
      rmin = min(v0, v1) - s.degv;
      nrows = max(v0, v1) - rmin + 1;
      cu0 = min(u0, u1) - s.degu;
      ncu = max(u0, u1) + 1 - cu0;
    }
    const bool factored = fit && nrows <= kBandRows;
    const bool tiled = factored && ncu <= kBandNetCols;
    // Full-degree units take the fast path, over NR = D + 2 or D + 3 net
    // rows (rows past the band's own are zero-filled).
    const bool fast = tiled && s.degu == D && s.degv == D;
    const int nrf = nrows <= D + 2 ? D + 2 : D + 3;
    // The fast path's column inputs (span and u basis of this thread's
    // sample column; warp 8 shares column 256), loaded ahead of the barrier.
    const int fcol = tid < kBandCols - 1 ? tid : kBandCols - 1;
    int fsu = 0;
    TC fNu[D + 1];
    if (fast && fcol < ncols) {
      fsu = bs.spans[lu0 + fcol];
      const TB *Nb = bs.basis + (lu0 + fcol) * 3 * p1;
#pragma unroll
      for (int q = 0; q <= D; ++q) {
        if constexpr (std::is_same<TB, TC>::value) fNu[q] = Nb[q];
        else fNu[q] = __double2float_rn(Nb[q]);
      }
    }
    // v coefficients of the band's sample rows over its net rows.
    if (factored && tid < (nv + 1) * kBandRows) {
      const int a = tid / kBandRows, R = tid - a * kBandRows;
      const int q = R - (bs.spans[lv0 + a] - s.degv - rmin);
      TC m = TC(0);
      if (q >= 0 && q <= s.degv) {
        const TB x = bs.basis[(lv0 + a) * 3 * p1 + q];
        if constexpr (std::is_same<TB, TC>::value) m = x;
        else m = __double2float_rn(x);
      }
      coef[a][R] = m;
    }
    if (tiled) {
      const int nrs = fast ? nrf : nrows;
      for (int e = tid; e < nrs * ncu; e += blockDim.x) {
        const int R = e / ncu, cc = e - (e / ncu) * ncu;
        NT[R * kBandNetCols + cc] = R < nrows ? s.cpw[static_cast<long long>(s.ncpu) * (rmin + R) + cu0 + cc]
                                              : Vec4<TC>{TC(0), TC(0), TC(0), TC(0)};
      }
    }
    __syncthreads();
    if (fast) {
      if (s.rat) {
        if (nrf == D + 2)
          band_unit_fast<TB, TC, D, D + 2, true>(out, S, NT, coef, r, ty, tx0, ntx, nv, ncols, cu0, fsu, fNu);
        else
          band_unit_fast<TB, TC, D, D + 3, true>(out, S, NT, coef, r, ty, tx0, ntx, nv, ncols, cu0, fsu, fNu);
      } else {
        if (nrf == D + 2)
          band_unit_fast<TB, TC, D, D + 2, false>(out, S, NT, coef, r, ty, tx0, ntx, nv, ncols, cu0, fsu, fNu);
        else
          band_unit_fast<TB, TC, D, D + 3, false>(out, S, NT, coef, r, ty, tx0, ntx, nv, ncols, cu0, fsu, fNu);
      }
      __syncthreads();
      continue;
    }
    for (int col = tid; col < ncols; col += blockDim.x) {
      const long long lu = lu0 + col;
      if (factored) {
        const int su = bs.spans[lu];
        const TB *Nb = bs.basis + lu * 3 * p1;
        TC Nu[kP];
#pragma unroll
        for (int c = 0; c < kP; ++c) {
          if (c <= s.degu) {
            if constexpr (std::is_same<TB, TC>::value) Nu[c] = Nb[c];
            else Nu[c] = __double2float_rn(Nb[c]);
          }
        }
        TC rs[kBandRows][4];
#pragma unroll
        for (int R = 0; R < kBandRows; ++R) {
          TC r0 = TC(0), r1 = TC(0), r2 = TC(0), r3 = TC(0);
          if (R < nrows) {
            const Vec4<TC> *cp = tiled ? NT + R * kBandNetCols + (su - s.degu - cu0)
                                       : s.cpw + static_cast<long long>(s.ncpu) * (rmin + R) + (su - s.degu);
#pragma unroll
            for (int c = 0; c < kP; ++c) {
              if (c <= s.degu) {
                const Vec4<TC> q = cp[c];
                if constexpr (std::is_same<TB, TC>::value) {
                  if (!s.rat) {
                    const TC n = Nu[c];
                    r0 += n * q.x;
                    r1 += n * q.y;
                    r2 += n * q.z;
                  } else {
                    const TC nw = Nu[c] * q.w;
                    r0 += nw * q.x;
                    r1 += nw * q.y;
                    r2 += nw * q.z;
                    r3 += nw;
                  }
                } else {
                  float n = Nu[c];
                  if (s.rat) {
                    n = __fmul_rn(n, q.w);
                    r3 = __fadd_rn(r3, n);
                  }
                  r0 = __fmaf_rn(n, q.x, r0);
                  r1 = __fmaf_rn(n, q.y, r1);
                  r2 = __fmaf_rn(n, q.z, r2);
                }
              }
            }
          }
          rs[R][0] = r0;
          rs[R][1] = r1;
          rs[R][2] = r2;
          rs[R][3] = r3;
        }
        for (int a = 0; a <= nv; ++a) {
          TC a0 = TC(0), a1 = TC(0), a2 = TC(0), a3 = TC(0);
#pragma unroll
          for (int R = 0; R < kBandRows; ++R) {
            const TC m = coef[a][R];
            if constexpr (std::is_same<TB, TC>::value) {
              a0 += m * rs[R][0];
              a1 += m * rs[R][1];
              a2 += m * rs[R][2];
              if (s.rat) a3 += m * rs[R][3];
            } else {
              a0 = __fmaf_rn(m, rs[R][0], a0);
              a1 = __fmaf_rn(m, rs[R][1], a1);
              a2 = __fmaf_rn(m, rs[R][2], a2);
              if (s.rat) a3 = __fmaf_rn(m, rs[R][3], a3);
            }
          }
          Vec4<TC> P{a0, a1, a2, TC(0)};
          if (s.rat) {
            if constexpr (std::is_same<TB, TC>::value) {
              const TC inv = TC(1) / a3;
              P.x = a0 * inv;
              P.y = a1 * inv;
              P.z = a2 * inv;
            } else {
              const double w = static_cast<double>(a3);
              P.x = __double2float_rn(static_cast<double>(a0) / w);
              P.y = __double2float_rn(static_cast<double>(a1) / w);
              P.z = __double2float_rn(static_cast<double>(a2) / w);
            }
          }
          S[a * kBandCols + col] = P;
        }
      } else {
        for (int a = 0; a <= nv; ++a) {
          const long long lv = lv0 + a;
          const TB *Nu = bs.basis + lu * 3 * p1;
          const TB *Nv = bs.basis + lv * 3 * p1;
          Vec4<TC> P;
          if constexpr (std::is_same<TB, TC>::value) {
            TC q[3];
            eval_point(s, bs.spans[lu], Nu, bs.spans[lv], Nv, q);
            P = Vec4<TC>{q[0], q[1], q[2], TC(0)};
          } else {
            P = screen_point(s, bs.spans[lu], Nu, bs.spans[lv], Nv);
          }
          S[a * kBandCols + col] = P;
        }
      }
    }
    __syncthreads();
    // Cells, one warp per tile of the chunk (k_cells' arithmetic and layout).
    for (int j = warp; j < ntx; j += blockDim.x >> 5) {
      const int tx = tx0 + j;
      const int nu = min(te, g.W - tx * te);
      const long long t = static_cast<long long>(r) * g.ntiles + ty * g.tw + tx;
      TC lo[3] = {pos_inf<TC>(), pos_inf<TC>(), pos_inf<TC>()};
      TC hi[3] = {-pos_inf<TC>(), -pos_inf<TC>(), -pos_inf<TC>()};
      for (int local = lane; local < te2; local += 32) {
        const int a = local / te, b = local - (local / te) * te;
        Vec4<TC> cen{TC(0), TC(0), TC(0), TC(0)};
        if (a < nv && b < nu) {
          const int c0 = j * te + b;
          const Vec4<TC> p0 = S[a * kBandCols + c0];
          const Vec4<TC> p1v = S[a * kBandCols + c0 + 1];
          const Vec4<TC> p2 = S[(a + 1) * kBandCols + c0];
          const Vec4<TC> p3 = S[(a + 1) * kBandCols + c0 + 1];
          const TC lx = fmn(p0.x, fmn(p1v.x, fmn(p2.x, p3.x)));
          const TC ly = fmn(p0.y, fmn(p1v.y, fmn(p2.y, p3.y)));
          const TC lz = fmn(p0.z, fmn(p1v.z, fmn(p2.z, p3.z)));
          const TC hx = fmx(p0.x, fmx(p1v.x, fmx(p2.x, p3.x)));
          const TC hy = fmx(p0.y, fmx(p1v.y, fmx(p2.y, p3.y)));
          const TC hz = fmx(p0.z, fmx(p1v.z, fmx(p2.z, p3.z)));
          cen.x = (lx - TC(0) + hx + TC(0)) / TC(2);
          cen.y = (ly - TC(0) + hy + TC(0)) / TC(2);
          cen.z = (lz - TC(0) + hz + TC(0)) / TC(2);
          lo[0] = fmn(lo[0], cen.x);
          lo[1] = fmn(lo[1], cen.y);
          lo[2] = fmn(lo[2], cen.z);
          hi[0] = fmx(hi[0], cen.x);
          hi[1] = fmx(hi[1], cen.y);
          hi[2] = fmx(hi[2], cen.z);
        }
        out.center[t * te2 + local] = cen;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          lo[c] = fmn(lo[c], __shfl_xor_sync(kFull, lo[c], o));
          hi[c] = fmx(hi[c], __shfl_xor_sync(kFull, hi[c], o));
        }
      }
      if (lane == 0) {
        out.tlo[t] = Vec4<TC>{lo[0], lo[1], lo[2], TC(0)};
        out.thi[t] = Vec4<TC>{hi[0], hi[1], hi[2], TC(0)};
        if (out.stmin) fold_supertile(out, r, ty, tx, lo, hi);
      }
    }
    __syncthreads();
  }
}

// Distance cells of large grids, one warp per unit of 4 tiles (32 cell
// columns, 33 sample columns) of one band of 8 cell rows, every warp on its
// own: no block barrier anywhere.  The host picks this kernel when the
// degrees of the whole launch are known and equal (D = 2 or 3) and passes
// them, and the rational flag, as template arguments.
//
// Samples (factored, as in band_unit_fast): lane c owns sample column c
// (c < 32) and forms the u-direction sums of the band's NR net rows from its
// u span and basis (control points straight from L1), then every sample of
// its column in v; the last column (32) goes to lanes 0..nv, one sample
// row each, each lane forming the column's row sums itself (the same
// operations, so the same bits).  A unit whose band needs more than D + 3
// net rows evaluates its samples one by one (eval_point / screen_point,
// again the same bits).  Cells: as in band_unit_fast, lane c owns cell
// column c of the unit.
constexpr int kWT = 4;               // tiles per warp unit
constexpr int kWC = kWT * kMaxTile;  // cell columns per warp unit (one per lane)
constexpr int kWS = kWC + 1;         // sample columns per warp unit
constexpr int kWWarps = 8;           // warps per block

// A warp unit's samples as three coordinate planes (12 B per FP32 sample
// through shared memory instead of a padded 16 B vector).  The v coefficient
// rows come first and the struct is 16-byte aligned: bandw_column reads each
// row as a float4 + float2, so every row, in every warp's copy, starts on a
// 16-byte boundary.
template <typename TC>
struct alignas(16) BandWarpSmem {
  alignas(16) TC coef[kMaxTile + 1][8];
  TC Sx[kMaxTile + 1][kWS], Sy[kMaxTile + 1][kWS], Sz[kMaxTile + 1][kWS];
  __device__ __forceinline__ void put(int a, int col, const Vec4<TC> &P) {
    Sx[a][col] = P.x;
    Sy[a][col] = P.y;
    Sz[a][col] = P.z;
  }
  __device__ __forceinline__ Vec4<TC> get(int a, int col) const {
    return Vec4<TC>{Sx[a][col], Sy[a][col], Sz[a][col], TC(0)};
  }
};

static_assert(sizeof(BandWarpSmem<float>) % 16 == 0 && sizeof(BandWarpSmem<double>) % 16 == 0,
              "per-warp band staging must keep 16-byte row alignment");
static_assert((8 * sizeof(float)) % 16 == 0, "coefficient rows must be 16-byte multiples");

template <typename TC>
constexpr size_t bandw_smem() {
  return sizeof(BandWarpSmem<TC>) * kWWarps;
}

// Samples of sample column col, rows a0..a1 (factored).
template <typename TB, typename TC, int D, int NR, bool RAT>
__device__ __forceinline__ void bandw_column(BandWarpSmem<TC> &w, const SurfView<TC> &s, const SideRound<TB> &bs,
                                             long long lu0, int col, int a0, int a1, int rmin, int nrows, int p1) {
  constexpr int kP = D + 1;
  const long long lu = lu0 + col;
  const int su = bs.spans[lu];
  const TB *Nb = bs.basis + lu * 3 * p1;
  TC Nu[kP];
#pragma unroll
  for (int c = 0; c < kP; ++c) {
    if constexpr (std::is_same<TB, TC>::value) Nu[c] = Nb[c];
    else Nu[c] = __double2float_rn(Nb[c]);
  }
  TC rs[NR][4];
#pragma unroll
  for (int R = 0; R < NR; ++R) {
    TC acc[4] = {TC(0), TC(0), TC(0), TC(0)};
    if (R < nrows) {
      const Vec4<TC> *cp = s.cpw + static_cast<long long>(s.ncpu) * (rmin + R) + (su - D);
#pragma unroll
      for (int c = 0; c < kP; ++c) band_row_sum<TB, TC, RAT>(Nu[c], cp[c], acc);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) rs[R][k] = acc[k];
  }
  for (int a = a0; a <= a1; ++a) {
    TC m[NR];
    if constexpr (sizeof(TC) == 4) {
      const float4 v0 = *reinterpret_cast<const float4 *>(&w.coef[a][0]);
      m[0] = v0.x;
      m[1] = v0.y;
      m[2] = v0.z;
      m[3] = v0.w;
      if constexpr (NR > 4) {
        const float2 v1 = *reinterpret_cast<const float2 *>(&w.coef[a][4]);
        m[4] = v1.x;
        if constexpr (NR > 5) m[5] = v1.y;
      }
    } else {
#pragma unroll
      for (int R = 0; R < NR; ++R) m[R] = w.coef[a][R];
    }
    TC acc[4] = {TC(0), TC(0), TC(0), TC(0)};
#pragma unroll
    for (int R = 0; R < NR; ++R) band_v_acc<TB, TC, RAT>(m[R], rs[R], acc);
    w.put(a, col, band_point<TB, TC, RAT>(acc));
  }
}

template <typename TB, typename TC, int D, int NR, bool RAT>
__device__ __forceinline__ void bandw_samples(BandWarpSmem<TC> &w, const SurfView<TC> &s, const SideRound<TB> &bs,
                                              long long lu0, long long lv0, int nv, int ncols, int rmin, int nrows,
                                              int p1, int lane) {
  // v coefficients of the band's sample rows over its net rows, zero outside
  // each row's window (see k_cells_band).
  for (int idx = lane; idx < (nv + 1) * 8; idx += 32) {
    const int a = idx >> 3, R = idx & 7;
    TC m = TC(0);
    if (R < NR) {
      const int q = R - (bs.spans[lv0 + a] - D - rmin);
      if (q >= 0 && q <= D) {
        const TB x = bs.basis[(lv0 + a) * 3 * p1 + q];
        if constexpr (std::is_same<TB, TC>::value) m = x;
        else m = __double2float_rn(x);
      }
    }
    w.coef[a][R] = m;
  }
  __syncwarp();
  if (lane < ncols) bandw_column<TB, TC, D, NR, RAT>(w, s, bs, lu0, lane, 0, nv, rmin, nrows, p1);
  if (ncols > kWC && lane <= nv) bandw_column<TB, TC, D, NR, RAT>(w, s, bs, lu0, kWC, lane, lane, rmin, nrows, p1);
}

template <typename TB, typename TC, int D, bool RAT>
__global__ void __launch_bounds__(kWWarps * 32, sizeof(TC) == 8 ? 2 : 4)
    k_cells_bandw(SurfView<TC> s, const SurfView<TC> *vdev, SideRound<TB> bs, SideRound<TC> out, long long qs) {
  extern __shared__ __align__(16) unsigned char bandw_raw[];
  const long long qo = qoff(qs);
  if (vdev) s = *qsh(vdev, qo);
  bs = qsh(bs, qo);
  out = qsh(out, qo);
  const Geom g = out.g;
  constexpr int te = kMaxTile, te2 = kMaxTile * kMaxTile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  BandWarpSmem<TC> &w = reinterpret_cast<BandWarpSmem<TC> *>(bandw_raw)[warp];
  const int p1 = g.p1max;
  const int nwc = (g.tw + kWT - 1) / kWT;
  const int per_reg = g.tw * nwc;
  const int nunits = nreg_of(bs) * per_reg;
  for (int unit = blockIdx.x * kWWarps + warp; unit < nunits; unit += gridDim.x * kWWarps) {
    const int r = unit / per_reg;
    const int rest = unit - r * per_reg;
    const int ty = rest / nwc, wc = rest - ty * nwc;
    const int tx0 = wc * kWT, ntx = min(kWT, g.tw - tx0);
    const int nv = min(te, g.W - ty * te);
    const int ncols = min(kWC, g.W - tx0 * te) + 1;
    const long long lu0 = (2LL * r) * g.nuv + tx0 * te;
    const long long lv0 = (2LL * r + 1) * g.nuv + ty * te;
    // Spans are monotone along the band's sample rows: the end rows give the
    // net rows the band reads.
    const int v0 = bs.spans[lv0], v1 = bs.spans[lv0 + nv];
    const int rmin = min(v0, v1) - D;
    const int nrows = max(v0, v1) - rmin + 1;
    if (nrows <= D + 2) {
      bandw_samples<TB, TC, D, D + 2, RAT>(w, s, bs, lu0, lv0, nv, ncols, rmin, nrows, p1, lane);
    } else if (nrows <= D + 3) {
      bandw_samples<TB, TC, D, D + 3, RAT>(w, s, bs, lu0, lv0, nv, ncols, rmin, nrows, p1, lane);
    } else {
      for (int idx = lane; idx < (nv + 1) * ncols; idx += 32) {
        const int a = idx / ncols, col = idx - (idx / ncols) * ncols;
        const long long lu = lu0 + col, lv = lv0 + a;
        const TB *Nu = bs.basis + lu * 3 * p1;
        const TB *Nv = bs.basis + lv * 3 * p1;
        Vec4<TC> P;
        if constexpr (std::is_same<TB, TC>::value) {
          TC q[3];
          eval_point(s, bs.spans[lu], Nu, bs.spans[lv], Nv, q);
          P = Vec4<TC>{q[0], q[1], q[2], TC(0)};
        } else {
          P = screen_point(s, bs.spans[lu], Nu, bs.spans[lv], Nv);
        }
        w.put(a, col, P);
      }
    }
    __syncwarp();
    // Cells: lane c owns cell column c (tile c / 8, column c % 8 of it).
    const int j = lane >> 3, b = lane & 7;
    const bool act = j < ntx;
    TC tlo[3] = {pos_inf<TC>(), pos_inf<TC>(), pos_inf<TC>()};
    TC thi[3] = {-pos_inf<TC>(), -pos_inf<TC>(), -pos_inf<TC>()};
    const int tx = tx0 + j;
    const long long t = static_cast<long long>(r) * g.ntiles + static_cast<long long>(ty) * g.tw + tx;
    if (act) {
      const bool colok = b < min(te, g.W - tx * te);
      Vec4<TC> p = w.get(0, lane), q = w.get(0, lane + 1);
      TC pmn[3] = {fmn(p.x, q.x), fmn(p.y, q.y), fmn(p.z, q.z)};
      TC pmx[3] = {fmx(p.x, q.x), fmx(p.y, q.y), fmx(p.z, q.z)};
      Vec4<TC> *dst = out.center + t * te2 + b;
#pragma unroll
      for (int a = 0; a < te; ++a) {
        p = w.get(a + 1, lane);
        q = w.get(a + 1, lane + 1);
        const TC nmn[3] = {fmn(p.x, q.x), fmn(p.y, q.y), fmn(p.z, q.z)};
        const TC nmx[3] = {fmx(p.x, q.x), fmx(p.y, q.y), fmx(p.z, q.z)};
        Vec4<TC> cen{TC(0), TC(0), TC(0), TC(0)};
        if (a < nv && colok) {
          TC c3[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const TC lo = fmn(pmn[k], nmn[k]), hi = fmx(pmx[k], nmx[k]);
            c3[k] = (lo - TC(0) + hi + TC(0)) * TC(0.5);  // = / 2 exactly
            tlo[k] = fmn(tlo[k], c3[k]);
            thi[k] = fmx(thi[k], c3[k]);
          }
          cen = Vec4<TC>{c3[0], c3[1], c3[2], TC(0)};
        }
        dst[a * te] = cen;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          pmn[k] = nmn[k];
          pmx[k] = nmx[k];
        }
      }
    }
#pragma unroll
    for (int o = 1; o < te; o <<= 1) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        tlo[k] = fmn(tlo[k], __shfl_xor_sync(kFull, tlo[k], o));
        thi[k] = fmx(thi[k], __shfl_xor_sync(kFull, thi[k], o));
      }
    }
    if (act && b == 0) {
      out.tlo[t] = Vec4<TC>{tlo[0], tlo[1], tlo[2], TC(0)};
      out.thi[t] = Vec4<TC>{thi[0], thi[1], thi[2], TC(0)};
      if (out.stmin) fold_supertile(out, r, ty, tx, tlo, thi);
    }
    __syncwarp();
  }
}

// FP64 centre of one cell exactly as the FP64 form builds it: P at the four
// corners from the FP64 basis tables (eval_point), min/max, (lo - 0 + hi + 0)/2.
__device__ Vec4<double> cell_center64(const SurfView<double> &s, const SideRound<double> &sr, int region, int cell) {
  const Geom g = sr.g;
  const int iv = cell / g.W, iu = cell - (cell / g.W) * g.W;
  const int p1 = g.p1max;
  double P[4][3];
#pragma unroll
  for (int cnr = 0; cnr < 4; ++cnr) {
    const int idx = iu + (cnr & 1), idy = iv + (cnr >> 1);
    const long long lu = (static_cast<long long>(region) * 2 + 0) * g.nuv + idx;
    const long long lv = (static_cast<long long>(region) * 2 + 1) * g.nuv + idy;
    eval_point(s, sr.spans[lu], sr.basis + lu * 3 * p1, sr.spans[lv], sr.basis + lv * 3 * p1, P[cnr]);
  }
  Vec4<double> c;
  double lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = tmin(P[0][d], tmin(P[1][d], tmin(P[2][d], P[3][d])));
    hi[d] = tmax(P[0][d], tmax(P[1][d], tmax(P[2][d], P[3][d])));
  }
  c.x = (lo[0] - 0.0 + hi[0] + 0.0) / 2.0;
  c.y = (lo[1] - 0.0 + hi[1] + 0.0) / 2.0;
  c.z = (lo[2] - 0.0 + hi[2] + 0.0) / 2.0;
  c.w = 0.0;
  return c;
}

// Re-check of the screened candidates in FP64: the FP64 form's d2 of each.
__global__ void k_dist_verify(SurfView<double> sa, SurfView<double> sb, const SurfView<double> *va,
                              const SurfView<double> *vb, SideRound<double> a, SideRound<double> b, const int *map1,
                              const int *map2, const DistCand<float> *cand, long long n, unsigned long long cap,
                              const ScreenStats *stats, DistCand<double> *out, long long qs) {
  const long long qo = qoff(qs);
  if (va) sa = *qsh(va, qo);
  if (vb) sb = *qsh(vb, qo);
  a = qsh(a, qo);
  b = qsh(b, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  cand = qsh(cand, qo);
  out = qsh(out, qo);
  if (stats) n = static_cast<long long>(count_of(kFromDevice, qsh(stats, qo)->candidates, cap));
  for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const DistCand<float> c = cand[e];
    const Vec4<double> c1 = cell_center64(sa, a, map1[c.slot], c.i);
    const Vec4<double> c2 = cell_center64(sb, b, map2[c.slot], c.j);
    out[e] = DistCand<double>{center_d2(c1, c2), c.slot, c.i, c.j};
  }
}

// ---------------------------------------------------------------------------
// FP64 Newton refinement (closest points, intersection points)
// ---------------------------------------------------------------------------

// Full 18-value record at an arbitrary (u, v) in FP64.  MAXP bounds degree + 1
// (the kernels that call it are instantiated for degrees up to 8 and for any
// degree, so that the common case keeps a small stack frame).
template <int MAXP>
__device__ void point_record(const SurfView<double> &s, double u, double v, double rec[18]) {
  double Nu[3 * MAXP], Nv[3 * MAXP];
  int spanu = s.degu, spanv = s.degv;
  if (!s.zero) {
    spanu = find_span(s.nku, s.degu, u, s.U);
    basis_ders_any<double, MAXP>(spanu, s.degu, u, s.U, s.du, Nu, MAXP);
    spanv = find_span(s.nkv, s.degv, v, s.V);
    basis_ders_any<double, MAXP>(spanv, s.degv, v, s.V, s.dv, Nv, MAXP);
  }
  eval_record(s, spanu, Nu, spanv, Nv, MAXP, rec);
}

// The basis bound of a pair of surfaces' kernels: 9 for degrees up to 8.
inline int newton_maxp(const SurfView<double> &a, const SurfView<double> &b) {
  return (a.degu < 9 && a.degv < 9 && b.degu < 9 && b.degv < 9) ? 9 : kMaxDeg + 1;
}

// P, Pu, Pv of one point: the first 9 values of point_record, bit for bit
// (the same basis functions and first derivatives, which A2.3 forms
// independently of the higher orders; the same contractions; the first-order
// steps of the quotient rule), without the second-order work.  MAXP bounds
// degree + 1.
template <int MAXP>
__device__ void point_record1_impl(const SurfView<double> &s, double u, double v, double rec[9]) {
  double Nu[3 * MAXP], Nv[3 * MAXP];
#pragma unroll
  for (int q = 0; q < 9; ++q) rec[q] = 0.0;
  if (s.zero) return;
  const int spanu = find_span(s.nku, s.degu, u, s.U);
  basis_ders_any<double, MAXP>(spanu, s.degu, u, s.U, min(s.du, 1), Nu, MAXP);
  const int spanv = find_span(s.nkv, s.degv, v, s.V);
  basis_ders_any<double, MAXP>(spanv, s.degv, v, s.V, min(s.dv, 1), Nv, MAXP);
  const int cu0 = spanu - s.degu, cv0 = spanv - s.degv;
  const int ku[3] = {0, 1, 0}, lv[3] = {0, 0, 1};
  if (!s.rat) {
    for (int m = 0; m < 3; ++m) {
      if (ku[m] > s.du || lv[m] > s.dv) continue;
      double acc[3];
      contract3(s, cu0, cv0, Nu + ku[m] * MAXP, Nv + lv[m] * MAXP, acc);
      rec[3 * m] = acc[0];
      rec[3 * m + 1] = acc[1];
      rec[3 * m + 2] = acc[2];
    }
    return;
  }
  double h[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) h[q] = 0.0;
  for (int m = 0; m < 3; ++m) {
    if (ku[m] > s.du || lv[m] > s.dv) continue;
    double acc[4];
    contract4(s, cu0, cv0, Nu + ku[m] * MAXP, Nv + lv[m] * MAXP, acc);
    h[4 * m] = acc[0];
    h[4 * m + 1] = acc[1];
    h[4 * m + 2] = acc[2];
    h[4 * m + 3] = acc[3];
  }
  // quotient2's first-order part
  const double inv = 1.0 / h[3];
#pragma unroll
  for (int q = 0; q < 12; ++q) h[q] *= inv;
  const double ws = -h[7], wt = -h[11];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    h[4 + c] += ws * h[c];
    h[8 + c] += wt * h[c];
  }
  for (int m = 0; m < 3; ++m)
    for (int c = 0; c < 3; ++c) rec[3 * m + c] = h[4 * m + c];
}

template <int MAXP>
__device__ void point_record1(const SurfView<double> &s, double u, double v, double rec[9]) {
  point_record1_impl<MAXP>(s, u, v, rec);
}

__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__device__ __forceinline__ double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

// Solves the n x n system M x = r (n <= 4) by Gaussian elimination with
// partial pivoting; returns false when a pivot vanishes.
__device__ bool solve_small(double M[4][4], double r[4], int n) {
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int q = c + 1; q < n; ++q)
      if (fabs(M[q][c]) > fabs(M[piv][c])) piv = q;
    if (!(fabs(M[piv][c]) > 0.0)) return false;
    if (piv != c) {
      for (int q = 0; q < n; ++q) {
        const double t = M[c][q];
        M[c][q] = M[piv][q];
        M[piv][q] = t;
      }
      const double t = r[c];
      r[c] = r[piv];
      r[piv] = t;
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

// Levenberg-Marquardt on f(u, v, s, t) = |S1(u, v) - S2(s, t)|^2 from the
// centres of the candidate cells, inside the query rectangles.  Records are
// P, Pu, Pv, Puu, Puv, Pvv (3 each).  out: d, u, v, s, t, P1[3], P2[3].
template <int MAXP>
__device__ void newton_distance(const SurfView<double> &sa, const SurfView<double> &sb, const double dom[8],
                                double x[4], double out[11]) {
  double r1[18], r2[18];
  point_record<MAXP>(sa, x[0], x[1], r1);
  point_record<MAXP>(sb, x[2], x[3], r2);
  double D[3] = {r1[0] - r2[0], r1[1] - r2[1], r1[2] - r2[2]};
  double f = dot3(D, D);
  double lam = 1e-6;
  for (int it = 0; it < 60; ++it) {
    const double *S1u = r1 + 3, *S1v = r1 + 6, *S1uu = r1 + 9, *S1uv = r1 + 12, *S1vv = r1 + 15;
    const double *S2s = r2 + 3, *S2t = r2 + 6, *S2ss = r2 + 9, *S2st = r2 + 12, *S2tt = r2 + 15;
    double g[4] = {dot3(D, S1u), dot3(D, S1v), -dot3(D, S2s), -dot3(D, S2t)};
    double H[4][4];
    H[0][0] = dot3(S1u, S1u) + dot3(D, S1uu);
    H[0][1] = dot3(S1u, S1v) + dot3(D, S1uv);
    H[1][1] = dot3(S1v, S1v) + dot3(D, S1vv);
    H[0][2] = -dot3(S1u, S2s);
    H[0][3] = -dot3(S1u, S2t);
    H[1][2] = -dot3(S1v, S2s);
    H[1][3] = -dot3(S1v, S2t);
    H[2][2] = dot3(S2s, S2s) - dot3(D, S2ss);
    H[2][3] = dot3(S2s, S2t) - dot3(D, S2st);
    H[3][3] = dot3(S2t, S2t) - dot3(D, S2tt);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < a; ++b) H[a][b] = H[b][a];
    bool moved = false;
    while (lam < 1e16) {
      double M[4][4], step[4];
      for (int a = 0; a < 4; ++a) {
        for (int b = 0; b < 4; ++b) M[a][b] = H[a][b];
        M[a][a] += lam * (fabs(H[a][a]) + 1e-30);
        step[a] = -g[a];
      }
      if (!solve_small(M, step, 4)) {
        lam *= 10.0;
        continue;
      }
      double y[4];
      for (int a = 0; a < 4; ++a) y[a] = clampd(x[a] + step[a], dom[2 * a], dom[2 * a + 1]);
      double q1[18], q2[18];
      point_record<MAXP>(sa, y[0], y[1], q1);
      point_record<MAXP>(sb, y[2], y[3], q2);
      const double E[3] = {q1[0] - q2[0], q1[1] - q2[1], q1[2] - q2[2]};
      const double fy = dot3(E, E);
      if (fy < f) {
        double dmax = 0.0;
        for (int a = 0; a < 4; ++a) {
          dmax = fmax(dmax, fabs(y[a] - x[a]));
          x[a] = y[a];
        }
        for (int q = 0; q < 18; ++q) {
          r1[q] = q1[q];
          r2[q] = q2[q];
        }
        D[0] = E[0];
        D[1] = E[1];
        D[2] = E[2];
        f = fy;
        lam = fmax(lam * 0.1, 1e-12);
        moved = dmax > 1e-15;
        break;
      }
      lam *= 10.0;
    }
    if (!moved) break;
  }
  out[0] = sqrt(f);
  for (int a = 0; a < 4; ++a) out[1 + a] = x[a];
  for (int c = 0; c < 3; ++c) {
    out[5 + c] = r1[c];
    out[8 + c] = r2[c];
  }
}

// One thread per final candidate pair: cell centres as the starting point.
template <typename TP, int MAXP>
__global__ void k_newton_dist(SurfView<double> sa, SurfView<double> sb, const SurfView<double> *va,
                              const SurfView<double> *vb, const RegionRec<TP> *reg1, const RegionRec<TP> *reg2,
                              const int *map1, const int *map2, int nuv1, int nuv2, const DistCand<TP> *top, int n,
                              const ScreenStats *stats, const double *dom, double *out, long long qs) {
  const long long qo = qoff(qs);
  if (va) sa = *qsh(va, qo);
  if (vb) sb = *qsh(vb, qo);
  reg1 = qsh(reg1, qo);
  reg2 = qsh(reg2, qo);
  map1 = qsh(map1, qo);
  map2 = qsh(map2, qo);
  top = qsh(top, qo);
  dom = qsh(dom, qo);
  out = qsh(out, qo);
  if (stats) n = qsh(stats, qo)->nslots;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const DistCand<TP> c = top[e];
  const RegionRec<TP> R1 = reg1[map1[c.slot]], R2 = reg2[map2[c.slot]];
  const int w1 = nuv1 - 1, w2 = nuv2 - 1;
  const double du1 = (double(R1.u1) - double(R1.u0)) / nuv1, dv1 = (double(R1.v1) - double(R1.v0)) / nuv1;
  const double du2 = (double(R2.u1) - double(R2.u0)) / nuv2, dv2 = (double(R2.v1) - double(R2.v0)) / nuv2;
  double x[4] = {double(R1.u0) + du1 * ((c.i % w1) + 0.5), double(R1.v0) + dv1 * ((c.i / w1) + 0.5),
                 double(R2.u0) + du2 * ((c.j % w2) + 0.5), double(R2.v0) + dv2 * ((c.j / w2) + 0.5)};
  double d[8];
  for (int q = 0; q < 8; ++q) d[q] = dom[q];
  double o[11];
  newton_distance<MAXP>(sa, sb, d, x, o);
  for (int q = 0; q < 11; ++q) out[e * 11 + q] = o[q];
}

// Minimum-norm Gauss-Newton on S1(u, v) - S2(s, t) = 0 (3 equations, 4
// unknowns): step = -J^T (J J^T)^-1 D.  out: x, y, z, u, v, s, t, residual.
template <int MAXP>
__device__ void newton_point(const SurfView<double> &sa, const SurfView<double> &sb, const double dom[8], double x[4],
                             double out[8]) {
  double r1[9], r2[9], D[3];
  double prev = INFINITY;
  for (int it = 0; it < 40; ++it) {
    point_record1<MAXP>(sa, x[0], x[1], r1);
    point_record1<MAXP>(sb, x[2], x[3], r2);
    for (int c = 0; c < 3; ++c) D[c] = r1[c] - r2[c];
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
    if (!solve_small(M, y, 3)) break;
    double dmax = 0.0;
    for (int q = 0; q < 4; ++q) {
      const double step = -(J[0][q] * y[0] + J[1][q] * y[1] + J[2][q] * y[2]);
      const double nx = clampd(x[q] + step, dom[2 * q], dom[2 * q + 1]);
      dmax = fmax(dmax, fabs(nx - x[q]));
      x[q] = nx;
    }
    // converged, or the steps stopped shrinking at rounding level
    if (dmax <= 1e-15 || (dmax <= 1e-12 && dmax > 0.5 * prev)) break;
    prev = dmax;
  }
  point_record1<MAXP>(sa, x[0], x[1], r1);
  point_record1<MAXP>(sb, x[2], x[3], r2);
  for (int c = 0; c < 3; ++c) {
    D[c] = r1[c] - r2[c];
    out[c] = 0.5 * (r1[c] + r2[c]);
  }
  for (int q = 0; q < 4; ++q) out[3 + q] = x[q];
  out[7] = sqrt(dot3(D, D));
}

// 64-thread blocks, 8 per SM (at most 128 registers a thread, no spills):
// the iteration is a chain of dependent FP64 steps, so warps in flight set
// its speed (165 registers gave 12 warps per SM).
template <typename TP, int MAXP>
__global__ void __launch_bounds__(64, 8) k_newton_inter(SurfView<double> sa, SurfView<double> sb, const RegionRec<TP> *reg1,
                               const RegionRec<TP> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                               const unsigned long long *keys, long long n, int ij_bits, const double *dom,
                               double *out) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= n) return;
  const unsigned long long k = keys[e];
  const unsigned long long mij = (1ull << ij_bits) - 1ull;
  const int slot = static_cast<int>(k >> (2 * ij_bits));
  const int ci = static_cast<int>((k >> ij_bits) & mij), cj = static_cast<int>(k & mij);
  const RegionRec<TP> R1 = reg1[map1[slot]], R2 = reg2[map2[slot]];
  const int w1 = nuv1 - 1, w2 = nuv2 - 1;
  const double du1 = (double(R1.u1) - double(R1.u0)) / nuv1, dv1 = (double(R1.v1) - double(R1.v0)) / nuv1;
  const double du2 = (double(R2.u1) - double(R2.u0)) / nuv2, dv2 = (double(R2.v1) - double(R2.v0)) / nuv2;
  double x[4] = {double(R1.u0) + du1 * ((ci % w1) + 0.5), double(R1.v0) + dv1 * ((ci / w1) + 0.5),
                 double(R2.u0) + du2 * ((cj % w2) + 0.5), double(R2.v0) + dv2 * ((cj / w2) + 0.5)};
  double d[8];
  for (int q = 0; q < 8; ++q) d[q] = dom[q];
  double o[8];
  newton_point<MAXP>(sa, sb, d, x, o);
  for (int q = 0; q < 8; ++q) out[e * 8 + q] = o[q];
}

// Resident surface layout from the raw EGADS record (knots, xyz net, weights;
// include/nurbs_data.hpp:1-10): the record itself (its first nku + nkv floats
// are the FP32 knot vectors), FP64 knot vectors and the (x, y, z, w) nets in
// FP32 and FP64 (w = 1 when non-rational).  Exact conversions.  One block row
// (blockIdx.y) per surface of the upload.
__global__ void k_surface_prep(const SurfacePrep *jobs) {
  const SurfacePrep J = jobs[blockIdx.y];
  const long long nk = J.nku + J.nkv;
  const long long n = J.ndata > J.ncp ? J.ndata : J.ncp;
  const float *cp = J.src + nk;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < n;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (t < J.ndata) J.raw[t] = J.src[t];
    if (t < J.nku) J.U64[t] = static_cast<double>(J.src[t]);
    else if (t < nk) J.V64[t - J.nku] = static_cast<double>(J.src[t]);
    if (t < J.ncp) {
      const float w = J.rat ? cp[3 * J.ncp + t] : 1.0f;
      const float x = cp[3 * t], y = cp[3 * t + 1], z = cp[3 * t + 2];
      J.cpw32[t] = Vec4<float>{x, y, z, w};
      J.cpw64[t] = Vec4<double>{x, y, z, w};
    }
  }
}

// Unit tangent of the intersection curve at each refined point: the cross
// product of the two surface normals (Su x Sv, Ss x St) at the point's
// parameters; and the size of the point's source cells (the final-round
// pair it was refined from), |Su| du + |Sv| dv on the larger side, the
// spacing scale of the points.  out: tx, ty, tz, ok (0 where the normals are
// parallel or vanish), scale.  pts: 8 doubles per point (x, y, z, u, v, s, t,
// residual), in the order of the pair keys.
template <typename TP, int MAXP>
__global__ void k_curve_tangents(SurfView<double> sa, SurfView<double> sb, const RegionRec<TP> *reg1,
                                 const RegionRec<TP> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                                 const unsigned long long *keys, int ij_bits, const double *pts, long long n,
                                 double *out) {
  const long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (e >= n) return;
  const double *q = pts + e * 8;
  const unsigned long long key = keys[e];
  const int slot = static_cast<int>(key >> (2 * ij_bits));
  const RegionRec<TP> R1 = reg1[map1[slot]], R2 = reg2[map2[slot]];
  double r1[18], r2[18];
  point_record<MAXP>(sa, q[3], q[4], r1);
  point_record<MAXP>(sb, q[5], q[6], r2);
  auto cross = [](const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
  };
  double n1[3], n2[3], t[3];
  cross(r1 + 3, r1 + 6, n1);
  cross(r2 + 3, r2 + 6, n2);
  cross(n1, n2, t);
  const double tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  const double nn = sqrt((n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]) * (n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]));
  const bool ok = tn > 1e-12 * nn && tn > 0.0;
  auto len3 = [](const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); };
  const double s1 = len3(r1 + 3) * fabs(double(R1.u1) - double(R1.u0)) / nuv1 +
                    len3(r1 + 6) * fabs(double(R1.v1) - double(R1.v0)) / nuv1;
  const double s2 = len3(r2 + 3) * fabs(double(R2.u1) - double(R2.u0)) / nuv2 +
                    len3(r2 + 6) * fabs(double(R2.v1) - double(R2.v0)) / nuv2;
  double *o = out + e * 5;
  o[0] = ok ? t[0] / tn : 0.0;
  o[1] = ok ? t[1] / tn : 0.0;
  o[2] = ok ? t[2] / tn : 0.0;
  o[3] = ok ? 1.0 : 0.0;
  o[4] = fmax(s1, s2);
}

inline int grid_for(long long n, int block, int max_blocks = 148 * 16) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return static_cast<int>(g);
}

std::atomic<unsigned long long> g_launches{0};

inline void counted(int n = 1) { g_launches.fetch_add(static_cast<unsigned long long>(n), std::memory_order_relaxed); }

}  // namespace

unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }
void add_launches(unsigned long long n) { counted(static_cast<int>(n)); }

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------

// Blocks per query: the single-query grid, shrunk so that a batch of bt.n
// queries stays within max_total blocks.
inline int bgrid(long long want, const Batch &bt, int max_total) {
  long long g = want < 1 ? 1 : want;
  const long long per = max_total / (bt.n > 0 ? bt.n : 1);
  if (g > per) g = per;
  if (g < 1) g = 1;
  return static_cast<int>(g);
}

inline dim3 bdim(int gx, const Batch &bt) { return dim3(static_cast<unsigned>(gx), static_cast<unsigned>(bt.n), 1u); }

template <typename T>
void launch_basis(const SurfView<T> &s, const SideRound<T> &sr, cudaStream_t st, const Batch &bt,
                  const SurfView<T> *vdev, bool cover, bool values_only) {
  const int md = values_only ? 0 : 2;
  counted();
  const long long n = static_cast<long long>(sr.nreg) * 2 * sr.g.nuv;
  // Degrees are part of a batch's shape: the host view decides the variant.
  const int maxdeg = s.degu > s.degv ? s.degu : s.degv;
  if (maxdeg < 8)
    k_basis<T, 9><<<bdim(bgrid((n + 127) / 128, bt, 148 * 16), bt), 128, 0, st>>>(
        s, vdev, sr.regions, sr.nreg, sr.dnreg, sr.g.nuv, sr.g.p1max, sr.spans, sr.basis, bt.qs, cover ? 1 : 0, md);
  else
    k_basis<T, kMaxDeg + 1><<<bdim(bgrid((n + 63) / 64, bt, 148 * 16), bt), 64, 0, st>>>(
        s, vdev, sr.regions, sr.nreg, sr.dnreg, sr.g.nuv, sr.g.p1max, sr.spans, sr.basis, bt.qs, cover ? 1 : 0, md);
}

template <typename T>
void launch_samples(const SurfView<T> &s, const SideRound<T> &sr, bool need_k, cudaStream_t st, const Batch &bt,
                    const SurfView<T> *vdev) {
  counted();
  const long long n = static_cast<long long>(sr.nreg) * sr.g.nuv * sr.g.nuv;
  k_samples<T><<<bdim(bgrid((n + 127) / 128, bt, 148 * 32), bt), 128, 0, st>>>(s, vdev, sr, need_k ? 1 : 0, bt.qs);
}

template <typename T>
void launch_pad(const SideRound<T> &sr, bool use_k, T span_u0, T span_v0, cudaStream_t st) {
  counted();
  k_pad<T><<<(sr.nreg + 127) / 128, 128, 0, st>>>(sr, use_k ? 1 : 0, span_u0, span_v0);
}

template <typename T>
void launch_cells(const SideRound<T> &sr, bool intersect, cudaStream_t st, const Batch &bt) {
  counted();
  const long long warps = static_cast<long long>(sr.nreg) * sr.g.ntiles;
  k_cells<T><<<bdim(bgrid((warps + 7) / 8, bt, 148 * 32), bt), 256, 0, st>>>(sr, intersect ? 1 : 0, bt.qs);
}

template <typename T>
bool region_cells_fits(const SideRound<T> &sr) {
  return sr.g.nuv <= kRegNuv && sr.g.p1max <= kRegP1;
}

template <typename T>
void launch_region_cells(const SurfView<T> &s, const SideRound<T> &sr, bool need_k, T span_u0, T span_v0, bool cover,
                         cudaStream_t st) {
  counted();
  if (sr.nreg <= 0) return;
  const int rpb = region_cells_rpb(sr.g.nuv);
  size_t offs[5];
  const size_t smem = region_cells_smem<T>(sr.g, rpb, offs);
  const long long groups = (sr.nreg + rpb - 1) / rpb;
  const int blocks = static_cast<int>(groups < 148 * 16 ? groups : 148 * 16);
  k_region_cells<T><<<blocks, kRegThreads, smem, st>>>(s, sr, need_k ? 1 : 0, span_u0, span_v0, cover ? 1 : 0);
}

template <typename T>
void launch_records(const SurfView<T> &s, T ustep, T vstep, T ustart, T vstart, int nuv, T *out, cudaStream_t st) {
  counted();
  const long long n = static_cast<long long>(nuv) * nuv;
  k_records<T><<<grid_for(n, 64, 148 * 32), 64, 0, st>>>(s, ustep, vstep, ustart, vstart, nuv, out);
}

// nslots < 0: the slot count is read on the device; the host passes the
// largest it can be as -(max slots).
inline int rows_for(int nslots, int per_slot) { return (nslots < 0 ? -nslots : nslots) * per_slot; }
inline int dev_slots(int nslots) { return nslots < 0 ? -1 : nslots; }

template <typename T>
void launch_dist_tau(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                     int k, ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt) {
  if (!dist_tau_folds(b.g, k)) return;
  counted();
  const dim3 grid = bdim(bgrid(rows_for(nslots, a.g.ntiles), bt, 148 * 8), bt);
  const int ns = dev_slots(nslots);
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_tau<float, true><<<grid, 256, 0, st>>>(a, b, map1, map2, ns, k, stats, e, bt.qs);
      return;
    }
  }
  k_dist_tau<T, false><<<grid, 256, 0, st>>>(a, b, map1, map2, ns, k, stats, e, bt.qs);
}

template <typename T>
void launch_dist_cull(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                      unsigned long long *surv, unsigned *surv_lb, unsigned long long surv_cap, ScreenStats *stats,
                      bool screen, float e, cudaStream_t st, const Batch &bt) {
  counted();
  const int block = b.g.ntiles >= 256 ? 256 : (b.g.ntiles >= 128 ? 128 : (b.g.ntiles >= 64 ? 64 : 32));
  const dim3 grid = bdim(bgrid(rows_for(nslots, a.g.ntiles), bt, 148 * 16), bt);
  const int ns = dev_slots(nslots);
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_cull<float, true><<<grid, block, 0, st>>>(a, b, map1, map2, ns, surv, surv_lb, surv_cap, stats, e,
                                                       bt.qs);
      return;
    }
  }
  k_dist_cull<T, false><<<grid, block, 0, st>>>(a, b, map1, map2, ns, surv, surv_lb, surv_cap, stats, e, bt.qs);
}

template <typename T>
void launch_dist_leaf(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                      const unsigned long long *surv, const unsigned *surv_lb, unsigned long long nsurv,
                      unsigned long long surv_cap, bool sorted, int k, int collect, DistCand<T> *cand,
                      unsigned long long cand_cap, ScreenStats *stats, bool screen, float e, cudaStream_t st,
                      const Batch &bt) {
  counted();
  if (nsurv == 0) return;
  const unsigned long long most = nsurv == kFromDevice ? surv_cap : nsurv;
  const unsigned long long warps = most < 148ull * 64 ? most : 148ull * 64;
  const dim3 grid = bdim(bgrid(static_cast<long long>((warps + 7) / 8), bt, 148 * 8), bt);
  const int so = sorted ? 1 : 0;
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_leaf<float, true><<<grid, 256, 0, st>>>(a, b, map1, map2, surv, surv_lb, nsurv, surv_cap, so, k, collect,
                                                     cand, cand_cap, stats, e, bt.qs);
      return;
    }
  }
  k_dist_leaf<T, false><<<grid, 256, 0, st>>>(a, b, map1, map2, surv, surv_lb, nsurv, surv_cap, so, k, collect, cand,
                                              cand_cap, stats, e, bt.qs);
}

template <typename T>
void launch_supertiles(const SideRound<T> &sr, cudaStream_t st, const Batch &bt) {
  counted();
  const long long warps = static_cast<long long>(sr.nreg) * sr.g.nst;
  k_supertiles<T><<<bdim(bgrid((warps + 7) / 8, bt, 148 * 32), bt), 256, 0, st>>>(sr, bt.qs);
}

template <typename T>
void launch_dist_tau_st(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                        int k, ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt) {
  counted();
  // k <= kStKL: a block's merge takes the exact k-th of the pairs it saw,
  // and the smallest block k-th enters tau, so every block should see many
  // pairs: a query is split over more blocks only past 64 supertile pairs
  // per thread (16,384 per block), and up to 16,384 pairs it runs as one
  // block, whose k-th is the query's exact one.  Split by the batch size
  // instead, tau loosened as batches shrank: for the hard-wave pair at
  // nuv0 = 512 (4096 supertile pairs), it grew 1.25x at 4 blocks, 2.8x at 9
  // and 6x at 18, and the tile pairs under it from about 3.7k to 6k, 45k and
  // 234k (past the survivor list's 65,536, so those queries re-ran alone).
  const long long st_pairs = static_cast<long long>(rows_for(nslots, a.g.nst)) * b.g.nst;
  const long long per_block = 256LL * 64;
  const dim3 grid = k <= kStKL ? bdim(bgrid((st_pairs + per_block - 1) / per_block, bt, 148 * 8), bt)
                               : bdim(bgrid(rows_for(nslots, a.g.nst), bt, 148 * 8), bt);
  const int ns = dev_slots(nslots);
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_tau_st<float, true><<<grid, 256, 0, st>>>(a, b, map1, map2, ns, k, stats, e, bt.qs);
      return;
    }
  }
  k_dist_tau_st<T, false><<<grid, 256, 0, st>>>(a, b, map1, map2, ns, k, stats, e, bt.qs);
}

template <typename T>
void launch_dist_cull_st(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                         unsigned long long *surv, unsigned long long cap, ScreenStats *stats, bool screen, float e,
                         cudaStream_t st, const Batch &bt) {
  counted();
  const dim3 grid = bdim(bgrid(rows_for(nslots, a.g.nst), bt, 148 * 16), bt);
  const int block = b.g.nst >= 256 ? 256 : (b.g.nst >= 128 ? 128 : (b.g.nst >= 64 ? 64 : 32));
  const int ns = dev_slots(nslots);
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_cull_st<float, true><<<grid, block, 0, st>>>(a, b, map1, map2, ns, surv, cap, stats, e, bt.qs);
      return;
    }
  }
  k_dist_cull_st<T, false><<<grid, block, 0, st>>>(a, b, map1, map2, ns, surv, cap, stats, e, bt.qs);
}

template <typename T>
void launch_dist_expand(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                        const unsigned long long *st_surv, unsigned long long nst_surv, unsigned long long st_cap,
                        int k, int cull, unsigned long long *surv, unsigned *surv_lb, unsigned long long cap,
                        ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt) {
  counted();
  if (nst_surv == 0) return;
  // 128-thread blocks, one warp per supertile pair.
  const unsigned long long most = nst_surv == kFromDevice ? st_cap : nst_surv;
  const dim3 grid = bdim(bgrid(static_cast<long long>(most < 148ull * 32 ? most : 148ull * 32), bt, 148 * 32), bt);
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_expand<float, true><<<grid, 128, 0, st>>>(a, b, map1, map2, st_surv, nst_surv, st_cap, k, cull, surv,
                                                        surv_lb, cap, stats, e, bt.qs);
      return;
    }
  }
  k_dist_expand<T, false><<<grid, 128, 0, st>>>(a, b, map1, map2, st_surv, nst_surv, st_cap, k, cull, surv, surv_lb,
                                                 cap, stats, e, bt.qs);
}

template <typename T>
void launch_dist_head(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                      const unsigned long long *surv, unsigned long long nhead, unsigned long long head_cap, int k,
                      ScreenStats *stats, bool screen, float e, cudaStream_t st, const Batch &bt) {
  counted();
  if (nhead == 0) return;
  const unsigned long long most = nhead == kFromDevice ? head_cap : nhead;
  const dim3 grid = bdim(bgrid(static_cast<long long>((most + 7) / 8), bt, 148 * 8), bt);
  if constexpr (std::is_same<T, float>::value) {
    if (screen) {
      k_dist_head<float, 8, true><<<grid, 256, 0, st>>>(a, b, map1, map2, surv, nhead, k, stats, e, bt.qs);
      return;
    }
  }
  k_dist_head<T, 8, false><<<grid, 256, 0, st>>>(a, b, map1, map2, surv, nhead, k, stats, e, bt.qs);
}

template <typename T>
void launch_dist_select(const DistCand<T> *cand, unsigned long long cand_cap, int k, DistCand<T> *out,
                        ScreenStats *stats, cudaStream_t st, const Batch &bt) {
  counted();
  const size_t smem = sizeof(DistCand<T>) * kSelectCap;
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_dist_select<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    configured = true;
  }
  k_dist_select<T><<<bdim(1, bt), 1024, smem, st>>>(cand, cand_cap, k, out, stats, bt.qs);
}

template <typename T>
void launch_dist_next(const DistCand<T> *top, ScreenStats *stats, const SideRound<T> &a, const SideRound<T> &b,
                      const int *map1, const int *map2, int nuv_next, RegionRec<T> *next1, RegionRec<T> *next2,
                      int *nmap1, int *nmap2, cudaStream_t st, const Batch &bt) {
  counted();
  k_dist_next<T><<<bdim(1, bt), 1024, 0, st>>>(top, stats, a, b, map1, map2, nuv_next, next1, next2, nmap1, nmap2,
                                               bt.qs);
}

template <typename TP>
void launch_dist_close(ScreenStats *stats, const DistCand<TP> *top, DistRecord<TP> *rec, int round,
                       unsigned long long surv_cap, unsigned long long cand_cap, bool last, cudaStream_t st,
                       const Batch &bt) {
  counted();
  k_dist_close<TP><<<bdim(1, bt), 32, 0, st>>>(stats, top, rec, round, surv_cap, cand_cap, last ? 1 : 0, bt.qs);
}

void launch_dist_pick(const unsigned long long *surv, const unsigned *surv_lb, unsigned long long surv_cap,
                      unsigned long long *head, unsigned long long head_cap, unsigned want, ScreenStats *stats,
                      cudaStream_t st, const Batch &bt) {
  counted();
  k_dist_pick<<<bdim(1, bt), 1024, 0, st>>>(surv, surv_lb, surv_cap, head, head_cap, want, stats, bt.qs);
}

template <typename T>
void launch_inter_cull(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2, int nslots,
                       unsigned long long *surv, unsigned long long surv_cap, ScreenStats *stats, cudaStream_t st) {
  counted();
  const long long n = static_cast<long long>(nslots) * a.g.ntiles * b.g.ntiles;
  k_inter_cull<T, false><<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(a, b, map1, map2, nslots, surv, surv_cap, stats,
                                                                       Vec4<float>{}, nullptr, nullptr);
}

template <typename T>
void launch_inter_leaf(const SideRound<T> &a, const SideRound<T> &b, const int *map1, const int *map2,
                       const unsigned long long *surv, unsigned long long nsurv, int ij_bits,
                       unsigned long long *keys, unsigned long long key_cap, ScreenStats *stats, cudaStream_t st) {
  counted();
  if (nsurv == 0) return;
  const unsigned long long warps = nsurv < 148ull * 64 ? nsurv : 148ull * 64;
  const int blocks = static_cast<int>((warps + 7) / 8);
  k_inter_leaf<T, false><<<blocks, 256, 0, st>>>(a, b, map1, map2, surv, nsurv, ij_bits, keys, key_cap, stats,
                                                  Vec4<float>{}, nullptr, nullptr);
}

void launch_inter_cull_screen(const SideRound<float> &a, const SideRound<float> &b, const int *map1, const int *map2,
                              int nslots, unsigned long long *surv, unsigned long long surv_cap, ScreenStats *stats,
                              const float w[3], const double *pad64a, const double *pad64b, cudaStream_t st) {
  counted();
  const long long n = static_cast<long long>(nslots) * a.g.ntiles * b.g.ntiles;
  k_inter_cull<float, true><<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(
      a, b, map1, map2, nslots, surv, surv_cap, stats, Vec4<float>{w[0], w[1], w[2], 0.0f}, pad64a, pad64b);
}

void launch_inter_leaf_screen(const SideRound<float> &a, const SideRound<float> &b, const int *map1, const int *map2,
                              const unsigned long long *surv, unsigned long long nsurv, int ij_bits,
                              unsigned long long *keys, unsigned long long key_cap, ScreenStats *stats,
                              const float w[3], const double *pad64a, const double *pad64b, cudaStream_t st) {
  counted();
  if (nsurv == 0) return;
  const unsigned long long warps = nsurv < 148ull * 64 ? nsurv : 148ull * 64;
  const int blocks = static_cast<int>((warps + 7) / 8);
  k_inter_leaf<float, true><<<blocks, 256, 0, st>>>(a, b, map1, map2, surv, nsurv, ij_bits, keys, key_cap, stats,
                                                    Vec4<float>{w[0], w[1], w[2], 0.0f}, pad64a, pad64b);
}

void launch_iscreen_samples(const SurfView<float> &s, const SideRound<double> &bs, const SideRound<float> &out,
                            bool need_k, Vec4<float> *khi, unsigned *klo, double g, const double cmax[3],
                            const double wcmax[3], double wmax, cudaStream_t st) {
  counted();
  IScreenConst c;
  c.g = g;
  for (int q = 0; q < 3; ++q) {
    c.cmax[q] = cmax[q];
    c.wcmax[q] = wcmax[q];
  }
  c.wmax = wmax;
  const long long n = static_cast<long long>(bs.nreg) * bs.g.nuv * bs.g.nuv;
  const int blocks = grid_for(n, 128, 148 * 32);
  if (need_k)
    k_iscreen_samples<true><<<blocks, 128, 0, st>>>(s, bs, out, khi, klo, c);
  else
    k_iscreen_samples<false><<<blocks, 128, 0, st>>>(s, bs, out, khi, klo, c);
}

void launch_kmax_recheck(const SurfView<double> &s, const SideRound<double> &bs, const Vec4<float> *khi,
                         const unsigned *klo, unsigned long long *count, cudaStream_t st) {
  counted();
  const long long n = static_cast<long long>(bs.nreg) * bs.g.nuv * bs.g.nuv;
  k_kmax_recheck<<<grid_for(n, 128, 148 * 32), 128, 0, st>>>(s, bs, khi, klo, count);
}

void launch_inter_verify_cells(const SideRound<double> &a, const SideRound<double> &b, const int *map1,
                               const int *map2, const unsigned long long *keys, unsigned long long n, int ij_bits,
                               unsigned long long *out, unsigned long long cap, ScreenStats *stats, cudaStream_t st) {
  counted();
  if (n == 0) return;
  k_inter_verify_cells<<<grid_for(static_cast<long long>(n), 128, 148 * 32), 128, 0, st>>>(a, b, map1, map2, keys, n,
                                                                                          ij_bits, out, cap, stats);
}


void launch_curve_tangents(const SurfView<double> &sa, const SurfView<double> &sb, const RegionRec<double> *reg1,
                           const RegionRec<double> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                           const unsigned long long *keys, int ij_bits, const double *pts, long long n, double *out,
                           cudaStream_t st) {
  counted();
  if (n <= 0) return;
  const unsigned grid = static_cast<unsigned>((n + 127) / 128);
  if (newton_maxp(sa, sb) == 9)
    k_curve_tangents<double, 9><<<grid, 128, 0, st>>>(sa, sb, reg1, reg2, map1, map2, nuv1, nuv2, keys, ij_bits, pts,
                                                      n, out);
  else
    k_curve_tangents<double, kMaxDeg + 1><<<grid, 128, 0, st>>>(sa, sb, reg1, reg2, map1, map2, nuv1, nuv2, keys,
                                                                ij_bits, pts, n, out);
}

void launch_pad_bound(const SideRound<double> &sr, const SurfView<double> &v, const Vec4<double> *tab, double eps,
                      cudaStream_t st) {
  counted();
  k_pad_bound<<<(sr.nreg + 127) / 128, 128, 0, st>>>(sr, reinterpret_cast<Vec4<double> *>(sr.pad), v, tab, eps);
}

void launch_bound_cull(const SideRound<double> &a, const SideRound<double> &b, const int *map1, const int *map2,
                       int nslots, double ub2, unsigned long long *surv, unsigned long long surv_cap,
                       ScreenStats *stats, cudaStream_t st) {
  counted();
  const long long n = static_cast<long long>(nslots) * a.g.ntiles * b.g.ntiles;
  k_bound_cull<<<grid_for(n, 256, 148 * 16), 256, 0, st>>>(a, b, map1, map2, nslots, ub2, surv, surv_cap, stats);
}

void launch_bound_leaf(const SideRound<double> &a, const SideRound<double> &b, const int *map1, const int *map2,
                       const unsigned long long *surv, unsigned long long nsurv, int ij_bits, double ub2,
                       unsigned long long *keys, unsigned long long key_cap, ScreenStats *stats, cudaStream_t st) {
  counted();
  if (nsurv == 0) return;
  const unsigned long long warps = nsurv < 148ull * 64 ? nsurv : 148ull * 64;
  const int blocks = static_cast<int>((warps + 7) / 8);
  k_bound_leaf<<<blocks, 256, 0, st>>>(a, b, map1, map2, surv, nsurv, ij_bits, ub2, keys, key_cap, stats);
}

void launch_inter_prep(const unsigned long long *keys, long long n, int ij_bits, unsigned long long *key2, int *idx,
                       unsigned *flag1, cudaStream_t st) {
  counted();
  k_inter_prep<<<grid_for(n, 256), 256, 0, st>>>(keys, n, ij_bits, key2, idx, flag1);
}

void launch_flag_runs(const unsigned long long *sorted, long long n, unsigned *flags, cudaStream_t st) {
  counted();
  k_flag_runs<<<grid_for(n, 256), 256, 0, st>>>(sorted, n, flags);
}

template <typename T>
void launch_inter_side1(const unsigned long long *keys, long long n, int ij_bits, const unsigned *flag1,
                        const unsigned *ex1, const SideRound<T> &cur, const int *map1, RegionRec<T> *next,
                        int *nmap1, cudaStream_t st, bool cover) {
  counted();
  k_inter_side1<T><<<grid_for(n, 256), 256, 0, st>>>(keys, n, ij_bits, flag1, ex1, cur, map1, next, nmap1,
                                                     cover ? 1 : 0);
}

template <typename T>
void launch_inter_side2(const unsigned long long *key2s, const int *idxs, long long n, int ij_bits,
                        const unsigned *flag2, const unsigned *ex2, const SideRound<T> &cur, const int *map2,
                        RegionRec<T> *next, int *nmap2, cudaStream_t st, bool cover) {
  counted();
  k_inter_side2<T><<<grid_for(n, 256), 256, 0, st>>>(key2s, idxs, n, ij_bits, flag2, ex2, cur, map2, next, nmap2,
                                                     cover ? 1 : 0);
}

void launch_samples_screen(const SurfView<float> &s, const SideRound<double> &basis_side, const SideRound<float> &out,
                           cudaStream_t st, const Batch &bt, const SurfView<float> *vdev) {
  counted();
  const long long n = static_cast<long long>(basis_side.nreg) * basis_side.g.nuv * basis_side.g.nuv;
  k_samples_screen<<<bdim(bgrid((n + 127) / 128, bt, 148 * 32), bt), 128, 0, st>>>(s, vdev, basis_side, out, bt.qs);
}

void launch_surface_prep(const SurfacePrep *jobs, int n, long long most, cudaStream_t st) {
  counted();
  if (n <= 0) return;
  const int gx = static_cast<int>(std::min<long long>((most + 255) / 256, 64));
  k_surface_prep<<<dim3(gx > 0 ? gx : 1, n, 1), 256, 0, st>>>(jobs);
}

template <typename TB, typename TC, int D, bool RAT>
void launch_bandw(const SurfView<TC> &s, const SideRound<TB> &bs, const SideRound<TC> &out, cudaStream_t st,
                  const Batch &bt, const SurfView<TC> *vdev) {
  constexpr size_t smem = bandw_smem<TC>();
  static bool configured = false;  // once per instantiation
  if (!configured) {
    cudaFuncSetAttribute(k_cells_bandw<TB, TC, D, RAT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(smem));
    configured = true;
  }
  const Geom &g = out.g;
  const long long units = static_cast<long long>(bs.nreg) * g.tw * ((g.tw + kWT - 1) / kWT);
  k_cells_bandw<TB, TC, D, RAT><<<bdim(bgrid((units + kWWarps - 1) / kWWarps, bt, 148 * 16), bt), kWWarps * 32, smem,
                                   st>>>(s, vdev, bs, out, bt.qs);
}

template <typename TB, typename TC>
void launch_cells_fused(const SurfView<TC> &s, const SideRound<TB> &bs, const SideRound<TC> &out, cudaStream_t st,
                        const Batch &bt, const SurfView<TC> *vdev, bool mixed) {
  counted();
  const Geom &g = out.g;
  if (!mixed && g.tw >= 16 && g.te == kMaxTile && !s.zero && s.degu == s.degv && (s.degu == 3 || s.degu == 2)) {
    // Large grids with equal degrees 2 or 3 (degrees, the rational flag and
    // the zero flag are part of a batch's shape): warp-independent bands.
    if (s.degu == 3) {
      if (s.rat) launch_bandw<TB, TC, 3, true>(s, bs, out, st, bt, vdev);
      else launch_bandw<TB, TC, 3, false>(s, bs, out, st, bt, vdev);
    } else {
      if (s.rat) launch_bandw<TB, TC, 2, true>(s, bs, out, st, bt, vdev);
      else launch_bandw<TB, TC, 2, false>(s, bs, out, st, bt, vdev);
    }
    return;
  }
  if (!mixed && g.tw >= 16 && g.te == kMaxTile && s.degu <= 3 && s.degv <= 3) {
    // Large grids of bicubic-or-lower surfaces (degrees are part of a batch's
    // shape): whole bands per block.
    constexpr size_t smem = band_smem<TC>();
    static bool configured = false;
    if (!configured) {
      cudaFuncSetAttribute(k_cells_band<TB, TC, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(smem));
      configured = true;
    }
    const long long units = static_cast<long long>(bs.nreg) * g.tw * ((g.tw + kBandTiles - 1) / kBandTiles);
    k_cells_band<TB, TC, 3><<<bdim(bgrid(units, bt, 148 * 16), bt), kBandThreads, smem, st>>>(s, vdev, bs, out,
                                                                                              bt.qs);
    return;
  }
  const long long warps = static_cast<long long>(bs.nreg) * g.ntiles;
  const dim3 grid = bdim(bgrid((warps + 3) / 4, bt, 148 * 64), bt);
  if (g.p1max <= 9)
    k_cells_fused<TB, TC, 9><<<grid, 128, 0, st>>>(s, vdev, bs, out, bt.qs);
  else
    k_cells_fused<TB, TC, kMaxDeg + 1><<<grid, 128, 0, st>>>(s, vdev, bs, out, bt.qs);
}

template void launch_cells_fused<float, float>(const SurfView<float> &, const SideRound<float> &,
                                               const SideRound<float> &, cudaStream_t, const Batch &,
                                               const SurfView<float> *, bool);
template void launch_cells_fused<double, double>(const SurfView<double> &, const SideRound<double> &,
                                                 const SideRound<double> &, cudaStream_t, const Batch &,
                                                 const SurfView<double> *, bool);
template void launch_cells_fused<double, float>(const SurfView<float> &, const SideRound<double> &,
                                                const SideRound<float> &, cudaStream_t, const Batch &,
                                                const SurfView<float> *, bool);

void launch_dist_verify(const SurfView<double> &sa, const SurfView<double> &sb, const SideRound<double> &a,
                        const SideRound<double> &b, const int *map1, const int *map2, const DistCand<float> *cand,
                        long long n, DistCand<double> *out, cudaStream_t st, const Batch &bt,
                        const SurfView<double> *va, const SurfView<double> *vb, const ScreenStats *stats,
                        unsigned long long cap) {
  counted();
  if (n <= 0 && !stats) return;
  const long long most = stats ? static_cast<long long>(cap) : n;
  k_dist_verify<<<bdim(bgrid((most + 127) / 128, bt, 148 * 16), bt), 128, 0, st>>>(sa, sb, va, vb, a, b, map1, map2,
                                                                                   cand, n, cap, stats, out, bt.qs);
}

template <typename TP>
void launch_newton_dist(const SurfView<double> &sa, const SurfView<double> &sb, const RegionRec<TP> *reg1,
                        const RegionRec<TP> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                        const DistCand<TP> *top, int n, const double *dom, double *out, cudaStream_t st,
                        const Batch &bt, const SurfView<double> *va, const SurfView<double> *vb,
                        const ScreenStats *stats) {
  counted();
  if (n <= 0) return;
  // sa / sb carry the largest degrees of a batch (the queries' own views
  // come from va / vb).
  if (newton_maxp(sa, sb) == 9)
    k_newton_dist<TP, 9><<<bdim((n + 63) / 64, bt), 64, 0, st>>>(sa, sb, va, vb, reg1, reg2, map1, map2, nuv1, nuv2,
                                                                 top, n, stats, dom, out, bt.qs);
  else
    k_newton_dist<TP, kMaxDeg + 1><<<bdim((n + 63) / 64, bt), 64, 0, st>>>(sa, sb, va, vb, reg1, reg2, map1, map2,
                                                                           nuv1, nuv2, top, n, stats, dom, out, bt.qs);
}

template <typename TP>
void launch_newton_inter(const SurfView<double> &sa, const SurfView<double> &sb, const RegionRec<TP> *reg1,
                         const RegionRec<TP> *reg2, const int *map1, const int *map2, int nuv1, int nuv2,
                         const unsigned long long *keys, long long n, int ij_bits, const double *dom, double *out,
                         cudaStream_t st) {
  counted();
  if (n <= 0) return;
  const unsigned grid = static_cast<unsigned>((n + 63) / 64);
  if (newton_maxp(sa, sb) == 9)
    k_newton_inter<TP, 9><<<grid, 64, 0, st>>>(sa, sb, reg1, reg2, map1, map2, nuv1, nuv2, keys, n, ij_bits, dom, out);
  else
    k_newton_inter<TP, kMaxDeg + 1><<<grid, 64, 0, st>>>(sa, sb, reg1, reg2, map1, map2, nuv1, nuv2, keys, n, ij_bits,
                                                         dom, out);
}

#define JSI_INSTANTIATE(T)                                                                                        \
  template void launch_basis<T>(const SurfView<T> &, const SideRound<T> &, cudaStream_t, const Batch &,           \
                                const SurfView<T> *, bool, bool);                                                 \
  template void launch_samples<T>(const SurfView<T> &, const SideRound<T> &, bool, cudaStream_t, const Batch &,   \
                                  const SurfView<T> *);                                                           \
  template void launch_pad<T>(const SideRound<T> &, bool, T, T, cudaStream_t);                                    \
  template bool region_cells_fits<T>(const SideRound<T> &);                                                       \
  template void launch_region_cells<T>(const SurfView<T> &, const SideRound<T> &, bool, T, T, bool, cudaStream_t); \
  template void launch_cells<T>(const SideRound<T> &, bool, cudaStream_t, const Batch &);                         \
  template void launch_records<T>(const SurfView<T> &, T, T, T, T, int, T *, cudaStream_t);                       \
  template void launch_dist_tau<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *, int, int, \
                                   ScreenStats *, bool, float, cudaStream_t, const Batch &);                      \
  template void launch_dist_cull<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *, int,    \
                                    unsigned long long *, unsigned *, unsigned long long, ScreenStats *, bool,    \
                                    float, cudaStream_t, const Batch &);                                          \
  template void launch_dist_leaf<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *,         \
                                    const unsigned long long *, const unsigned *, unsigned long long,             \
                                    unsigned long long, bool, int, int, DistCand<T> *, unsigned long long,        \
                                    ScreenStats *, bool, float, cudaStream_t, const Batch &);                     \
  template void launch_supertiles<T>(const SideRound<T> &, cudaStream_t, const Batch &);                          \
  template void launch_dist_tau_st<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *, int,  \
                                      int, ScreenStats *, bool, float, cudaStream_t, const Batch &);              \
  template void launch_dist_cull_st<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *, int, \
                                       unsigned long long *, unsigned long long, ScreenStats *, bool, float,      \
                                       cudaStream_t, const Batch &);                                              \
  template void launch_dist_expand<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *,       \
                                      const unsigned long long *, unsigned long long, unsigned long long, int,    \
                                      int, unsigned long long *, unsigned *, unsigned long long, ScreenStats *,   \
                                      bool, float, cudaStream_t, const Batch &);                                  \
  template void launch_dist_head<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *,         \
                                    const unsigned long long *, unsigned long long, unsigned long long, int,      \
                                    ScreenStats *, bool, float, cudaStream_t, const Batch &);                     \
  template void launch_dist_select<T>(const DistCand<T> *, unsigned long long, int, DistCand<T> *, ScreenStats *, \
                                      cudaStream_t, const Batch &);                                               \
  template void launch_dist_next<T>(const DistCand<T> *, ScreenStats *, const SideRound<T> &,                     \
                                    const SideRound<T> &, const int *, const int *, int, RegionRec<T> *,          \
                                    RegionRec<T> *, int *, int *, cudaStream_t, const Batch &);                   \
  template void launch_dist_close<T>(ScreenStats *, const DistCand<T> *, DistRecord<T> *, int,                    \
                                     unsigned long long, unsigned long long, bool, cudaStream_t, const Batch &);  \
  template void launch_inter_cull<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *, int,   \
                                     unsigned long long *, unsigned long long, ScreenStats *, cudaStream_t);      \
  template void launch_inter_leaf<T>(const SideRound<T> &, const SideRound<T> &, const int *, const int *,        \
                                     const unsigned long long *, unsigned long long, int, unsigned long long *,   \
                                     unsigned long long, ScreenStats *, cudaStream_t);                            \
  template void launch_inter_side1<T>(const unsigned long long *, long long, int, const unsigned *,               \
                                      const unsigned *, const SideRound<T> &, const int *, RegionRec<T> *, int *, \
                                      cudaStream_t, bool);                                                        \
  template void launch_inter_side2<T>(const unsigned long long *, const int *, long long, int, const unsigned *,  \
                                      const unsigned *, const SideRound<T> &, const int *, RegionRec<T> *, int *, \
                                      cudaStream_t, bool);

JSI_INSTANTIATE(float)
JSI_INSTANTIATE(double)

template void launch_newton_dist<float>(const SurfView<double> &, const SurfView<double> &, const RegionRec<float> *,
                                        const RegionRec<float> *, const int *, const int *, int, int,
                                        const DistCand<float> *, int, const double *, double *, cudaStream_t,
                                        const Batch &, const SurfView<double> *, const SurfView<double> *,
                                        const ScreenStats *);
template void launch_newton_dist<double>(const SurfView<double> &, const SurfView<double> &,
                                         const RegionRec<double> *, const RegionRec<double> *, const int *,
                                         const int *, int, int, const DistCand<double> *, int, const double *,
                                         double *, cudaStream_t, const Batch &, const SurfView<double> *,
                                         const SurfView<double> *, const ScreenStats *);
template void launch_newton_inter<float>(const SurfView<double> &, const SurfView<double> &, const RegionRec<float> *,
                                         const RegionRec<float> *, const int *, const int *, int, int,
                                         const unsigned long long *, long long, int, const double *, double *,
                                         cudaStream_t);
template void launch_newton_inter<double>(const SurfView<double> &, const SurfView<double> &,
                                          const RegionRec<double> *, const RegionRec<double> *, const int *,
                                          const int *, int, int, const unsigned long long *, long long, int,
                                          const double *, double *, cudaStream_t);

template <typename T, int MAXP>
void launch_dist_refine_p(const SurfView<T> &sa, const SurfView<T> &sb, const SurfView<T> *va, const SurfView<T> *vb,
                          ScreenStats *stats, DistRecord<T> *rec, const RefineArgs<T> &args, cudaStream_t st,
                          const Batch &bt) {
  constexpr size_t smem = refine_smem<T, MAXP>();
  cudaFuncSetAttribute(k_dist_refine<T, MAXP>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  counted();
  k_dist_refine<T, MAXP><<<bdim(1, bt), kRefineThreads, smem, st>>>(sa, sb, va, vb, stats, rec, args, bt.qs);
}

template <typename T>
void launch_dist_refine(const SurfView<T> &sa, const SurfView<T> &sb, const SurfView<T> *va, const SurfView<T> *vb,
                        ScreenStats *stats, DistRecord<T> *rec, const RefineArgs<T> &args, cudaStream_t st,
                        const Batch &bt) {
  const int deg = std::max(std::max(sa.degu, sa.degv), std::max(sb.degu, sb.degv));
  if (deg <= 8)
    launch_dist_refine_p<T, 9>(sa, sb, va, vb, stats, rec, args, st, bt);
  else
    launch_dist_refine_p<T, kMaxDeg + 1>(sa, sb, va, vb, stats, rec, args, st, bt);
}

template void launch_dist_refine<float>(const SurfView<float> &, const SurfView<float> &, const SurfView<float> *,
                                        const SurfView<float> *, ScreenStats *, DistRecord<float> *,
                                        const RefineArgs<float> &, cudaStream_t, const Batch &);
template void launch_dist_refine<double>(const SurfView<double> &, const SurfView<double> &, const SurfView<double> *,
                                         const SurfView<double> *, ScreenStats *, DistRecord<double> *,
                                         const RefineArgs<double> &, cudaStream_t, const Batch &);

}  // namespace jsi
