// Grid evaluation for callers that cannot allocate device memory.
//
// jsi_eval_grid() needs a context, and a context's arena and the device
// copies of the surface come from cudaMalloc.  Some callers of this library
// cannot allocate device memory when they need a grid: a host CAD application
// that has already handed the whole device to its own memory pool and refuses
// any allocation outside it, or a tight interactive loop that cannot absorb the
// implicit device-wide synchronisation of cudaMalloc/cudaFree.  For them,
// jsi_eval_grid_noalloc() runs the same record kernel as jsi_eval_grid()
// (k_records, through launch_records) with every device buffer it needs — the
// knot vectors, the packed control net and the records — carved out of one
// fixed, file-scope __device__ array.  It calls no cudaMalloc, cudaFree or any
// other allocating routine.
//
// Limits and sharing:
//  * The array is kNoAllocScratchBytes (32 MiB).  Its segments (U knots,
//    V knots, control net as 16-byte points, nuv*nuv*18 float records), each
//    rounded up to 256 bytes, must fit; larger requests return
//    JSI_ERR_CAPACITY before touching the device.
//  * Every GPU on which this library's code is loaded holds the 32 MiB until
//    the process exits.
//  * Every call works on the CUDA context current on the calling thread: it
//    looks up the array's device address in that context with
//    cudaGetSymbolAddress (which allocates nothing), so a caller that switches
//    contexts or resets the device gets the address valid in the new one.
//  * The copies are synchronous cudaMemcpy calls on the legacy default stream.
//    No call may run while any thread of the process is capturing a stream in
//    global capture mode: the copies would invalidate that capture.
//  * All calls share the one array and it keeps the previous call's contents.
//    Nothing in it has to start at zero: every knot, control point and record
//    this call reads is written by this call first (the weight lane of the
//    packed control net is only read for rational surfaces, and then it is
//    copied in).  Calls whose device work overlaps — from several host threads,
//    or alongside another process's use of the same device's array — race on
//    the array; serialise them.
#include <cuda_runtime.h>

#include <cstddef>

#include "jsi_b200.h"
#include "jsi_internal.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

size_t round256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Device address of the array in the context current on this thread.
int scratch_address(unsigned char **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    cudaGetLastError();
    return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? JSI_ERR_NO_DEVICE : JSI_ERR_CUDA;
  }
  *out = static_cast<unsigned char *>(p);
  return JSI_OK;
}

}  // namespace

extern "C" int jsi_eval_grid_noalloc(const int ivec[7], const float *data, int ndata, float ustep, float vstep,
                                     float ustart, float vstart, int nuv, float *results) {
  if (!ivec || !data || !results || nuv < 1) return JSI_ERR_INVALID;
  const int degu = ivec[1], ncpu = ivec[2], nku = ivec[3], degv = ivec[4], ncpv = ivec[5], nkv = ivec[6];
  // Header and length checks come before any size arithmetic, in 64-bit
  // signed integers, so that no product below can wrap.
  if (ndata < 0 || degu < 0 || degv < 0 || ncpu < 1 || ncpv < 1) return JSI_ERR_SURFACE;
  if (ncpu < degu + 1 || ncpv < degv + 1) return JSI_ERR_SURFACE;
  if (nku != ncpu + degu + 1 || nkv != ncpv + degv + 1) return JSI_ERR_SURFACE;
  const bool rational = (ivec[0] & 2) != 0;
  const long long ncp_ll = static_cast<long long>(ncpu) * ncpv;  // < 2^62
  const long long need = static_cast<long long>(nku) + nkv + (rational ? 4 : 3) * ncp_ll;
  if (static_cast<long long>(ndata) < need) return JSI_ERR_SURFACE;
  // Any of these alone exceeds the array (32 MiB / 16 B points; 4096^2 records).
  if (ncp_ll > static_cast<long long>(kNoAllocScratchBytes / sizeof(jsi::Vec4<float>)) || nuv > 4096)
    return JSI_ERR_CAPACITY;
  const size_t ncp = static_cast<size_t>(ncp_ll);

  const size_t bu = round256(static_cast<size_t>(nku) * sizeof(float));
  const size_t bv = round256(static_cast<size_t>(nkv) * sizeof(float));
  const size_t bc = round256(ncp * sizeof(jsi::Vec4<float>));
  const size_t nrec = static_cast<size_t>(nuv) * nuv * JSI_RECORD_SIZE;
  const size_t br = round256(nrec * sizeof(float));
  if (bu + bv + bc + br > kNoAllocScratchBytes) return JSI_ERR_CAPACITY;

  unsigned char *base = nullptr;
  if (const int st = scratch_address(&base); st != JSI_OK) return st;

  float *dU = reinterpret_cast<float *>(base);
  float *dV = reinterpret_cast<float *>(base + bu);
  jsi::Vec4<float> *dcp = reinterpret_cast<jsi::Vec4<float> *>(base + bu + bv);
  float *drec = reinterpret_cast<float *>(base + bu + bv + bc);
  const float *cp = data + nku + nkv;
  // Knots as given; control points (x, y, z) into 16-byte slots; weights, for
  // rational surfaces, into the fourth lane.  All on the legacy default stream.
  if (cudaMemcpy(dU, data, nku * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dV, data + nku, nkv * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy2D(dcp, sizeof(jsi::Vec4<float>), cp, 3 * sizeof(float), 3 * sizeof(float), ncp,
                   cudaMemcpyHostToDevice) != cudaSuccess ||
      (rational && cudaMemcpy2D(reinterpret_cast<unsigned char *>(dcp) + 3 * sizeof(float),
                                sizeof(jsi::Vec4<float>), cp + 3 * ncp, sizeof(float), sizeof(float), ncp,
                                cudaMemcpyHostToDevice) != cudaSuccess)) {
    cudaGetLastError();
    return JSI_ERR_CUDA;
  }
  jsi::SurfView<float> v;
  v.degu = degu;
  v.degv = degv;
  v.ncpu = ncpu;
  v.ncpv = ncpv;
  v.nku = nku;
  v.nkv = nkv;
  v.rat = rational ? 1 : 0;
  v.zero = ((!(ivec[0] & 1)) && (ivec[0] & 12)) || degu >= jsi::kMaxDeg || degv >= jsi::kMaxDeg;
  v.du = degu < 2 ? degu : 2;
  v.dv = degv < 2 ? degv : 2;
  v.U = dU;
  v.V = dV;
  v.cpw = dcp;
  jsi::launch_records<float>(v, ustep, vstep, ustart, vstart, nuv, drec, 0);
  if (cudaGetLastError() != cudaSuccess) return JSI_ERR_CUDA;
  if (cudaMemcpy(results, drec, nrec * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return JSI_ERR_CUDA;
  }
  return JSI_OK;
}
