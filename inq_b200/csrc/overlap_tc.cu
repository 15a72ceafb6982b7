// Overlap matrix of single-precision orbital sets on the 5th-generation tensor cores.
//
//   S_ij = dV sum_r conj(a_i(r)) b_j(r)          (operations::overlap, src/operations/overlap.hpp:26-95,
//                                                 a ZGEMM a^H b over the grid points)
//
// Split-BF16 compensated products: every FP32 component x is held as hi + lo with hi = bf16(x) and
// lo = bf16(x - hi) (16 significant bits), and a product is formed as hi*hi + hi*lo + lo*hi + lo*lo.
// The lo*lo term is kept: |lo| reaches 2^-8 |x|, and in a norm (a = b) the dropped squares would all
// have the same sign, a bias of ~4e-6 on the diagonal.  The complex product is four real ones,
//   Re S = ar.br + ai.bi,   Im S = ar.bi - ai.br   (the minus by the instruction's negate-A bit),
// so one 16-point chunk costs 16 MMAs of 128 x N x 16 (kind::f16, BF16 in, FP32 accumulate).
//
// One CTA per SM holds a 128-state block of a (tensor-memory lanes) against up to 256 states of b: the
// real and imaginary FP32 accumulators take N + N of the 512 tensor-memory columns.  The points are
// split over the CTAs; each CTA streams its range in 16-point chunks: all 256 threads read the FP32
// values (8-byte loads, one state per thread and eight consecutive points, coalesced across the
// warp), split them and store the BF16 planes in the canonical K-major layout (core matrices of 8
// rows x 16 bytes), and one thread issues the chunk's MMAs and commits them to the buffer's
// mbarrier.  Two operand buffers alternate; the next chunk's loads are in flight while the current
// chunk is converted.  The per-CTA FP32 partial sums go to global memory and a second kernel adds
// them in a fixed order in FP64, so the result does not depend on scheduling.
//
// Every mbarrier wait is bounded (2 s by %globaltimer); on expiry the kernel raises the context's
// error flag, waits (again bounded) for the MMAs it issued, frees its tensor memory and returns.

#include <cuda_bf16.h>

#include "inqb_internal.h"
#include "ptx.cuh"

namespace inqb {
namespace {

constexpr int TC_M = 128;         // states of a per CTA = tensor-memory lanes = MMA M
constexpr int TC_NMAX = 256;      // states of b per CTA at most = MMA N
constexpr int TC_KC = 16;         // points per chunk = MMA K
constexpr int TC_THREADS = 256;
constexpr uint32_t A_PLANE = TC_M * TC_KC * 2;       // bytes of one BF16 plane of the a chunk (4 KB)
constexpr uint32_t B_PLANE = TC_NMAX * TC_KC * 2;    // bytes of one BF16 plane of the b chunk (8 KB)
constexpr uint32_t BUF_BYTES = 4 * A_PLANE + 4 * B_PLANE;  // re_hi, re_lo, im_hi, im_lo of a and b
// The CTA uses 2 * 48 KB of operands; it asks for 120 KB so that only one CTA fits on an SM, since
// each CTA allocates all 512 tensor-memory columns.
constexpr size_t TC_SMEM = 120 * 1024;
constexpr uint64_t WAIT_NS = 2000000000ull;

__device__ __forceinline__ void split2(float x0, float x1, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
  const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
  const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
  const __nv_bfloat162 h = __halves2bfloat162(h0, h1), l = __halves2bfloat162(l0, l1);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// Eight consecutive points of one row (state), split into the four planes of a buffer at `plane0`
// (planes `plane_bytes` apart): byte offset of (row, k) = (row / 8) * 256 + (k / 8) * 128 + (row % 8) * 16
// + (k % 8) * 2, i.e. K-major core matrices with 128 bytes between the two K halves and 256 bytes
// between 8-row groups.
__device__ __forceinline__ void store_unit(unsigned char *plane0, uint32_t plane_bytes, int row, int kh,
                                           const float2 (&x)[8]) {
  uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    split2(x[2 * p].x, x[2 * p + 1].x, rh[p], rl[p]);
    split2(x[2 * p].y, x[2 * p + 1].y, ih[p], il[p]);
  }
  const uint32_t off = uint32_t(row >> 3) * 256u + uint32_t(kh) * 128u + uint32_t(row & 7) * 16u;
  *reinterpret_cast<uint4 *>(plane0 + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
  *reinterpret_cast<uint4 *>(plane0 + plane_bytes + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
  *reinterpret_cast<uint4 *>(plane0 + 2 * plane_bytes + off) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
  *reinterpret_cast<uint4 *>(plane0 + 3 * plane_bytes + off) = make_uint4(il[0], il[1], il[2], il[3]);
}

// Eight consecutive points [k, k + 8) of state `col` of a [npoints][S] set; zero outside.
__device__ __forceinline__ void load_unit(const float2 *__restrict__ src, int S, int col, bool colok, long long k,
                                          long long kend, float2 (&x)[8]) {
#pragma unroll
  for (int u = 0; u < 8; u++)
    x[u] = (colok && k + u < kend) ? __ldg(&src[(k + u) * S + col]) : make_float2(0.f, 0.f);
}

__global__ void __launch_bounds__(TC_THREADS, 1)
    overlap_tc_kernel(const float2 *__restrict__ a, int Sa, const float2 *__restrict__ b, int Sb,
                      long long npoints, int mtiles, int ntiles, int N, long long kper, float *__restrict__ partial,
                      int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t *done = reinterpret_cast<uint64_t *>(smem + 2 * BUF_BYTES);  // one mbarrier per operand buffer
  uint32_t *tslot = reinterpret_cast<uint32_t *>(done + 2);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);

  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int tiles = mtiles * ntiles;
  const int mt = blockIdx.x % mtiles, nt = (blockIdx.x / mtiles) % ntiles, ks = blockIdx.x / tiles;
  const int m0 = mt * TC_M, n0 = nt * N;
  const long long kbeg = (long long)ks * kper;
  const long long kend = kbeg + kper < npoints ? kbeg + kper : npoints;
  const int nchunks = kend > kbeg ? int((kend - kbeg + TC_KC - 1) / TC_KC) : 0;

  if (t == 0) {
    ptx::mbar_init(&done[0], 1);
    ptx::mbar_init(&done[1], 1);
    *abort_flag = 0;
    ptx::mbar_init_fence();
  }
  if (warp == 0) ptx::tmem_alloc(tslot, 512);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t d_re = tmem, d_im = tmem + uint32_t(N);
  const uint32_t id = ptx::idesc_bf16_f32(TC_M, N, false), idn = ptx::idesc_bf16_f32(TC_M, N, true);

  // conversion units: the a chunk has 128 rows x 2 K halves (one per thread), the b chunk 256 x 2 (two)
  const int arow = t & (TC_M - 1), akh = t >> 7;
  const int acol = m0 + arow, bcol = n0 + t;
  const bool aok = acol < Sa, bok = t < N && bcol < Sb;
  float2 ca[8], cb0[8], cb1[8], na[8], nb0[8], nb1[8];
  if (nchunks > 0) {
    load_unit(a, Sa, acol, aok, kbeg + akh * 8, kend, ca);
    load_unit(b, Sb, bcol, bok, kbeg, kend, cb0);
    load_unit(b, Sb, bcol, bok, kbeg + 8, kend, cb1);
  }

  int issued = 0;
  for (int c = 0; c < nchunks; c++) {
    const int bsel = c & 1;
    unsigned char *bufA = smem + bsel * BUF_BYTES;
    unsigned char *bufB = bufA + 4 * A_PLANE;
    if (c + 1 < nchunks) {
      const long long k1 = kbeg + (long long)(c + 1) * TC_KC;
      load_unit(a, Sa, acol, aok, k1 + akh * 8, kend, na);
      load_unit(b, Sb, bcol, bok, k1, kend, nb0);
      load_unit(b, Sb, bcol, bok, k1 + 8, kend, nb1);
    }
    // the MMAs of chunk c - 2 read this buffer
    if (c >= 2 && !ptx::mbar_wait_bounded(&done[bsel], uint32_t((c - 2) >> 1) & 1u, WAIT_NS)) {
      *abort_flag = 1;
      atomicExch(err, 1);
    }
    __syncthreads();
    if (*abort_flag) break;
    store_unit(bufA, A_PLANE, arow, akh, ca);
    store_unit(bufB, B_PLANE, t, 0, cb0);
    store_unit(bufB, B_PLANE, t, 1, cb1);
    ptx::fence_proxy_async();
    __syncthreads();
    if (t == 0) {
      ptx::tc_fence_after();
      const uint32_t ab = ptx::smem_u32(bufA), bb = ptx::smem_u32(bufB);
      uint64_t da[4], db[4];
#pragma unroll
      for (int p = 0; p < 4; p++) {
        da[p] = ptx::smem_desc_kmajor(ab + p * A_PLANE, 128, 256);
        db[p] = ptx::smem_desc_kmajor(bb + p * B_PLANE, 128, 256);
      }
      const bool acc = c > 0;
      // planes: 0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo
      // smallest products first into each accumulator's chunk sum
      ptx::mma_bf16(d_re, da[1], db[1], id, acc);
      ptx::mma_bf16(d_re, da[3], db[3], id, true);
      ptx::mma_bf16(d_re, da[0], db[1], id, true);
      ptx::mma_bf16(d_re, da[1], db[0], id, true);
      ptx::mma_bf16(d_re, da[2], db[3], id, true);
      ptx::mma_bf16(d_re, da[3], db[2], id, true);
      ptx::mma_bf16(d_re, da[0], db[0], id, true);
      ptx::mma_bf16(d_re, da[2], db[2], id, true);
      ptx::mma_bf16(d_im, da[1], db[3], id, acc);
      ptx::mma_bf16(d_im, da[3], db[1], idn, true);
      ptx::mma_bf16(d_im, da[0], db[3], id, true);
      ptx::mma_bf16(d_im, da[1], db[2], id, true);
      ptx::mma_bf16(d_im, da[2], db[1], idn, true);
      ptx::mma_bf16(d_im, da[3], db[0], idn, true);
      ptx::mma_bf16(d_im, da[0], db[2], id, true);
      ptx::mma_bf16(d_im, da[2], db[0], idn, true);
      ptx::mma_commit(&done[bsel]);
    }
    issued = c + 1;
#pragma unroll
    for (int u = 0; u < 8; u++) {
      ca[u] = na[u];
      cb0[u] = nb0[u];
      cb1[u] = nb1[u];
    }
  }

  // the last commit covers every MMA issued before it
  if (issued > 0) {
    const int last = issued - 1;
    if (!ptx::mbar_wait_bounded(&done[last & 1], uint32_t(last >> 1) & 1u, WAIT_NS)) {
      *abort_flag = 1;
      atomicExch(err, 1);
    }
  }
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  if (!*abort_flag) {
    const int q = warp & 3, h = warp >> 2;  // lane quarter of this warp; 0 real, 1 imaginary columns
    const int ia = m0 + q * 32 + lane;
    float *dst = partial + ((size_t(ks) * 2 + h) * size_t(Sa) + size_t(ia)) * size_t(Sb) + n0;
    for (int j0 = 0; j0 < N; j0 += 16) {
      float v[16];
      if (issued > 0) {
        ptx::tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(h * N + j0), v);
      } else {
#pragma unroll
        for (int u = 0; u < 16; u++) v[u] = 0.f;
      }
      if (ia < Sa) {
#pragma unroll
        for (int u = 0; u < 16; u++)
          if (n0 + j0 + u < Sb) dst[j0 + u] = v[u];
      }
    }
  }
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 0) ptx::tmem_dealloc(tmem, 512);
}

// out[i][j] = dv * sum over the point splits, in split order, in FP64
__global__ void overlap_tc_reduce(const float *__restrict__ partial, int nsplit, int Sa, int Sb, double dv,
                                  double2 *__restrict__ out) {
  const long long n = (long long)Sa * Sb;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int z = 0; z < nsplit; z++) {
      re += double(partial[(2LL * z) * n + e]);
      im += double(partial[(2LL * z + 1) * n + e]);
    }
    out[e] = make_double2(dv * re, dv * im);
  }
}

}  // namespace

void launch_overlap_tc(Ctx &ctx, const float2 *a, int Sa, const float2 *b, int Sb, long long npoints, double dv,
                       double2 *out) {
  INQB_REQUIRE(Sa > 0 && Sb > 0 && npoints > 0, INQB_ERR_ARG, "empty overlap");
  const int mtiles = (Sa + TC_M - 1) / TC_M;
  const int N = Sb < TC_NMAX ? (Sb + 15) / 16 * 16 : TC_NMAX;
  const int ntiles = (Sb + N - 1) / N;
  const int tiles = mtiles * ntiles;
  int nsplit = ctx.num_sms / tiles;
  if (nsplit < 1) nsplit = 1;
  long long kper = ((npoints + nsplit - 1) / nsplit + TC_KC - 1) / TC_KC * TC_KC;
  nsplit = int((npoints + kper - 1) / kper);  // every split holds at least one point
  float *partial = static_cast<float *>(dev_alloc(ctx, sizeof(float) * size_t(nsplit) * 2 * Sa * Sb));
  ensure_smem_attr(reinterpret_cast<const void *>(overlap_tc_kernel), TC_SMEM);
  overlap_tc_kernel<<<unsigned(tiles * nsplit), TC_THREADS, TC_SMEM, ctx.stream>>>(
      a, Sa, b, Sb, npoints, mtiles, ntiles, N, kper, partial, ctx.d_err);
  INQB_CUDA(cudaGetLastError());
  ctx.launches++;
  const long long n = (long long)Sa * Sb;
  long long blocks = (n + 255) / 256;
  if (blocks > 4L * ctx.num_sms) blocks = 4L * ctx.num_sms;
  overlap_tc_reduce<<<unsigned(blocks), 256, 0, ctx.stream>>>(partial, nsplit, Sa, Sb, dv, out);
  INQB_CUDA(cudaGetLastError());
  ctx.launches++;
  dev_free(ctx, partial);
}

}  // namespace inqb
