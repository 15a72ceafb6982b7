// Per-state overlap <a_s|b_s> (operations::overlap_diagonal) without any device allocation.
//
// Some callers cannot let this library call cudaMalloc: a serving loop that has divided all
// device memory among the orbital sets it keeps resident (its admission control counts every
// byte, so a surprise allocation can fail or push out a request), and latency-sensitive callers
// that must not risk the implicit device-wide synchronisation cudaMalloc/cudaFree can trigger.
// inqb_overlap_diagonal_noalloc serves them: the caller passes the orbital sets and a device
// buffer for the result, and the block partial sums live in the fixed array below, which is
// part of the library image (every GPU that loads the library holds its 2.3 MiB until exit).

#include <mutex>

#include "inqb_internal.h"

namespace inqb {
namespace {

constexpr int NOALLOC_BLOCKS = 296;       // partial sums per state (2 x 148 SMs)
constexpr int NOALLOC_MAX_STATES = 512;   // largest orbital set accepted

// Partial sums [NOALLOC_BLOCKS][nst] of the reduction.  Stage 1 overwrites every entry it
// stage 2 reads, so nothing has to be cleared between calls.  All calls share this array:
// calls whose kernels overlap on the GPU (different streams or contexts) race on it.
static __device__ __align__(256) double2 g_noalloc_partial[NOALLOC_BLOCKS * NOALLOC_MAX_STATES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
double2 *g_partial_addr[MAX_DEVICES] = {};

// Device address of the array on the current device.  In host code the array's name is only a
// host-side handle, so it must never be passed to a kernel; the address comes from the runtime,
// looked up once per device with that device current.
double2 *partial_address(int device) {
  INQB_REQUIRE(device >= 0 && device < MAX_DEVICES, INQB_ERR_UNSUPPORTED, "device index too large");
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_partial_addr[device]) {
    void *p = nullptr;
    INQB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partial));
    INQB_REQUIRE(p != nullptr, INQB_ERR_CUDA, "cudaGetSymbolAddress returned no address");
    g_partial_addr[device] = static_cast<double2 *>(p);
  }
  return g_partial_addr[device];
}

// stage 1: block b sums conj(a) b over its contiguous point range, one thread per state
template <typename R>
__global__ void noalloc_partial_kernel(const C2<R> *__restrict__ a, const C2<R> *__restrict__ b, int S,
                                       long long npoints, double2 *partial) {
  const long long chunk = (npoints + gridDim.x - 1) / gridDim.x;
  const long long p0 = blockIdx.x * chunk;
  const long long p1 = min(npoints, p0 + chunk);
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    double re = 0.0, im = 0.0;
    for (long long p = p0; p < p1; p++) {
      const C2<R> x = a[p * S + s], y = b[p * S + s];
      re += double(x.x) * double(y.x) + double(x.y) * double(y.y);
      im += double(x.x) * double(y.y) - double(x.y) * double(y.x);
    }
    partial[(long long)blockIdx.x * S + s] = make_double2(re, im);
  }
}

// stage 2: partials summed in block order, times the volume element
__global__ void noalloc_sum_kernel(const double2 *partial, int nblk, int S, double scale, double2 *out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nblk; k++) {
      re += partial[(long long)k * S + s].x;
      im += partial[(long long)k * S + s].y;
    }
    out[s] = make_double2(scale * re, scale * im);
  }
}

}  // namespace
}  // namespace inqb

using namespace inqb;

extern "C" int inqb_overlap_diagonal_noalloc(const inqb_orbitals *a, const inqb_orbitals *b, double *out_dev) {
  Ctx *ctx = a ? a->ctx : nullptr;
  try {
    INQB_REQUIRE(a && b && out_dev, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(a->basis == b->basis && a->nst == b->nst && a->precision == b->precision, INQB_ERR_ARG,
                 "overlap_diagonal of sets with different shapes or precisions");
    INQB_REQUIRE(a->nst <= NOALLOC_MAX_STATES, INQB_ERR_ARG,
                 "inqb_overlap_diagonal_noalloc accepts at most " + std::to_string(NOALLOC_MAX_STATES) +
                     " states (got " + std::to_string(a->nst) + "); use inqb_overlap_diagonal");
    INQB_CUDA(cudaSetDevice(ctx->device));
    double2 *partial = partial_address(ctx->device);
    const int S = a->nst;
    const long long np = a->basis->npoints;
    const double dv = set_volume_element(*a);
    if (a->precision == INQB_F64)
      noalloc_partial_kernel<double><<<NOALLOC_BLOCKS, 256, 0, ctx->stream>>>(
          static_cast<const double2 *>(a->data), static_cast<const double2 *>(b->data), S, np, partial);
    else
      noalloc_partial_kernel<float><<<NOALLOC_BLOCKS, 256, 0, ctx->stream>>>(
          static_cast<const float2 *>(a->data), static_cast<const float2 *>(b->data), S, np, partial);
    INQB_CUDA(cudaGetLastError());
    noalloc_sum_kernel<<<(S + 255) / 256, 256, 0, ctx->stream>>>(partial, NOALLOC_BLOCKS, S, dv,
                                                                 reinterpret_cast<double2 *>(out_dev));
    INQB_CUDA(cudaGetLastError());
    ctx->launches += 2;
    return INQB_OK;
  } catch (const Error &e) {
    if (ctx) ctx->err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    if (ctx) ctx->err = e.what();
    return INQB_ERR_STATE;
  }
}
