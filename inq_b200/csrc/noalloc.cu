// Per-state overlap <a_s|b_s> (operations::overlap_diagonal) without any device allocation.
//
// Some callers cannot let this library call cudaMalloc: a serving loop that has divided all
// device memory among the orbital sets it keeps resident (its admission control counts every
// byte, so a surprise allocation can fail or push out a request), and latency-sensitive callers
// that must not risk the implicit device-wide synchronisation cudaMalloc/cudaFree can trigger.
// inqb_overlap_diagonal_noalloc serves them: the caller passes the orbital sets and a device
// buffer for the result, and the block partial sums live in the fixed array below.
//
// When the memory is taken: CUDA loads a library's device code lazily by default, so the array
// would otherwise be placed on a device at the first use of this file's code there.  Every
// inqb_ctx_create calls noalloc_prepare, which looks the array's address up (loading this file's
// module, array included) and loads the two kernels; from then on the device holds the array's
// 2.3 MiB until the process exits, and the entry point's calls on that context allocate nothing.

#include "inqb_internal.h"

namespace inqb {
namespace {

constexpr int NOALLOC_BLOCKS = 296;       // partial sums per state (2 x 148 SMs)
constexpr int NOALLOC_MAX_STATES = 512;   // largest orbital set accepted

// Partial sums [NOALLOC_BLOCKS][nst] of the reduction.  Stage 1 overwrites every entry it
// stage 2 reads, so nothing has to be cleared between calls.  All calls share this array:
// calls whose kernels overlap on the GPU (different streams or contexts) race on it.
static __device__ __align__(256) double2 g_noalloc_partial[NOALLOC_BLOCKS * NOALLOC_MAX_STATES];

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

// stage 2: partials summed in block order, times the volume element; the result is written as
// two separate doubles, so out needs only the 8-byte alignment of a double
__global__ void noalloc_sum_kernel(const double2 *partial, int nblk, int S, double scale, double *out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nblk; k++) {
      re += partial[(long long)k * S + s].x;
      im += partial[(long long)k * S + s].y;
    }
    out[2 * s] = scale * re;
    out[2 * s + 1] = scale * im;
  }
}

// A device buffer the kernels may store to: device memory or managed memory reachable from the
// context's device.  Host memory (pageable or pinned) and other devices' memory are refused, as
// the store would fault the GPU or silently write somewhere else.
void check_output_buffer(const Ctx &ctx, const double *out_dev) {
  INQB_REQUIRE(reinterpret_cast<uintptr_t>(out_dev) % alignof(double) == 0, INQB_ERR_ARG,
               "out_dev is not aligned to 8 bytes");
  cudaPointerAttributes attr{};
  const cudaError_t e = cudaPointerGetAttributes(&attr, out_dev);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw Error(INQB_ERR_ARG, std::string("out_dev is not a CUDA pointer: ") + cudaGetErrorString(e));
  }
  if (attr.type == cudaMemoryTypeDevice) {
    INQB_REQUIRE(attr.device == ctx.device, INQB_ERR_ARG,
                 "out_dev is device memory of device " + std::to_string(attr.device) + ", the sets live on device " +
                     std::to_string(ctx.device));
  } else {
    INQB_REQUIRE(attr.type == cudaMemoryTypeManaged, INQB_ERR_ARG,
                 "out_dev must be device or managed memory (got host or unregistered memory)");
  }
}

}  // namespace

void noalloc_prepare(Ctx &ctx) {
  void *p = nullptr;
  INQB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partial));
  INQB_REQUIRE(p != nullptr, INQB_ERR_CUDA, "cudaGetSymbolAddress returned no address");
  cudaFuncAttributes fa;
  INQB_CUDA(cudaFuncGetAttributes(&fa, noalloc_partial_kernel<double>));
  INQB_CUDA(cudaFuncGetAttributes(&fa, noalloc_partial_kernel<float>));
  INQB_CUDA(cudaFuncGetAttributes(&fa, noalloc_sum_kernel));
  ctx.noalloc_partial = p;
}

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
    INQB_REQUIRE(ctx->noalloc_partial != nullptr, INQB_ERR_STATE, "context was not prepared for this entry point");
    check_output_buffer(*ctx, out_dev);
    double2 *partial = static_cast<double2 *>(ctx->noalloc_partial);
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
    noalloc_sum_kernel<<<(S + 255) / 256, 256, 0, ctx->stream>>>(partial, NOALLOC_BLOCKS, S, dv, out_dev);
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
