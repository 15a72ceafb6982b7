// Overlap matrix of single-precision orbital sets on the 5th-generation tensor cores.
//
//   S_ij = dV sum_r conj(a_i(r)) b_j(r)          (operations::overlap, src/operations/overlap.hpp:26-95,
//                                                 a ZGEMM a^H b over the grid points)
//
// Split-BF16 compensated products: every FP32 component x is held as hi + lo with hi = bf16(x) and
// lo = bf16(x - hi) (16 significant bits), and a product is formed as hi*hi + (hi*lo + lo*hi + lo*lo).
// The complex product is four real ones,
//   Re S = ar.br + ai.bi,   Im S = ar.bi - ai.br   (the minus by the instruction's negate-A bit).
//
// Accumulation.  The tensor core adds each MMA's products into its FP32 accumulator with truncation,
// so a sum whose partial values grow steadily (a norm, a diagonal element) loses about 0.4 ulp per
// MMA, always downwards: over the ~375 chunks a CTA streams at 96^3 that was a -7e-5 relative bias.
// Hence two accumulators per component in tensor memory: the large hi*hi products go into a "main"
// accumulator that is restarted every WIN chunks, its window sum read out (tcgen05.ld) and added with
// round-to-nearest into an FP32 running sum in shared memory; the small correction products (2^-8 of
// the main ones, random in sign) go into a "corr" accumulator kept over the whole range.  Remaining
// bias: ~2 MMAs per chunk x WIN chunks x 2^-25.  Measured at 96^3 x 256: WIN = 2, 4, 8 give diagonal
// biases of -1.0e-7, -1.9e-7, -4.0e-7 and 4.1, 3.5, 3.2 ms per overlap; 4 keeps a 5x margin to 1e-6.
//
// Tiles.  One CTA per SM holds 128 states of a (tensor-memory lanes) against 128 states of b: the
// main and corr accumulators of the real and imaginary parts take the 4 x 128 tensor-memory columns;
// the running sums take 2 x 64 KB of shared memory.  The points are split over the CTAs; each CTA
// streams its range in 16-point chunks.  Eight converter warps read the FP32 values (8-byte loads, one
// state per thread and eight consecutive points, coalesced across the warp), split them, store the
// BF16 planes in the canonical K-major layout (core matrices of 8 rows x 16 bytes) into one of three
// operand buffers and arrive on its "full" mbarrier; lane 0 of a ninth, issuer warp waits for it,
// issues the chunk's 16 MMAs (128 x N x 16, kind::f16, BF16 in, FP32 accumulate) and commits them to
// the buffer's "empty" mbarrier (and, at a window's end, to the window's).  The converters flush a
// finished window and arrive on "flushed" before the issuer restarts the main accumulators.  The loads
// of the chunk two ahead are in flight while the current chunk is converted (one ahead: 3.5 ms per
// overlap at 96^3 x 256 before the issuer warp; two: 3.0; more gains nothing; with the issuer warp
// 2.7).  The per-CTA FP32 partial sums go to global memory and a second kernel
// adds them in a fixed order in FP64, so the result does not depend on scheduling.
//
// Every mbarrier wait is bounded (2 s by %globaltimer); on expiry the kernel raises the context's
// error flag, waits (again bounded) for the MMAs it issued, frees its tensor memory and returns.

#include <cuda_bf16.h>

#include "inqb_internal.h"
#include "ptx.cuh"

namespace inqb {
namespace {

constexpr int TC_M = 128;         // states of a per CTA = tensor-memory lanes = MMA M
constexpr int TC_N = 128;         // states of b per CTA at most = MMA N
constexpr int TC_KC = 16;         // points per chunk = MMA K
constexpr int TC_THREADS = 256;
constexpr int WIN = 4;            // chunks per window of the main accumulators
constexpr int LOOK = 3;           // chunks whose values are held in registers (current + 2 in flight)
constexpr uint32_t PLANE = TC_M * TC_KC * 2;            // bytes of one BF16 plane (4 KB; a and b alike)
constexpr uint32_t BUF_BYTES = 8 * PLANE;               // re_hi, re_lo, im_hi, im_lo of a, then of b
constexpr uint32_t SUM_BYTES = 2 * TC_N * TC_M * 4;     // FP32 running sums of the main products
constexpr int NB = 3;             // operand buffers (converted chunks in flight to the tensor cores)
constexpr size_t TC_SMEM = NB * BUF_BYTES + SUM_BYTES + 128;
constexpr uint64_t WAIT_NS = 2000000000ull;
// tensor-memory columns of the four accumulators
constexpr uint32_t COL_MAIN_RE = 0, COL_MAIN_IM = 128, COL_CORR_RE = 256, COL_CORR_IM = 384;

__device__ __forceinline__ void split2(float x0, float x1, uint32_t &hi, uint32_t &lo) {
  // packed conversions (two values per instruction), each value rounded to nearest as on its own
  const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}

// Eight consecutive points of one row (state), split into the four planes of an operand at `plane0`:
// byte offset of (row, k) = (row / 8) * 256 + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2, i.e. K-major
// core matrices with 128 bytes between the two K halves and 256 bytes between 8-row groups.
__device__ __forceinline__ void store_unit(unsigned char *plane0, int row, int kh, const float2 (&x)[8]) {
  uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    split2(x[2 * p].x, x[2 * p + 1].x, rh[p], rl[p]);
    split2(x[2 * p].y, x[2 * p + 1].y, ih[p], il[p]);
  }
  const uint32_t off = uint32_t(row >> 3) * 256u + uint32_t(kh) * 128u + uint32_t(row & 7) * 16u;
  *reinterpret_cast<uint4 *>(plane0 + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
  *reinterpret_cast<uint4 *>(plane0 + PLANE + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
  *reinterpret_cast<uint4 *>(plane0 + 2 * PLANE + off) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
  *reinterpret_cast<uint4 *>(plane0 + 3 * PLANE + off) = make_uint4(il[0], il[1], il[2], il[3]);
}

// Eight consecutive points [k, k + 8) of state `col` of a [npoints][S] set; zero outside.
__device__ __forceinline__ void load_unit(const float2 *__restrict__ src, int S, int col, bool colok, long long k,
                                          long long kend, float2 (&x)[8]) {
#pragma unroll
  for (int u = 0; u < 8; u++)
    x[u] = (colok && k + u < kend) ? __ldg(&src[(k + u) * S + col]) : make_float2(0.f, 0.f);
}

__global__ void __launch_bounds__(TC_THREADS + 32, 1)
    overlap_tc_kernel(const float2 *__restrict__ a, int Sa, const float2 *__restrict__ b, int Sb,
                      long long npoints, int mtiles, int ntiles, int N, long long kper, int sym,
                      float *__restrict__ partial, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  float *sums = reinterpret_cast<float *>(smem + NB * BUF_BYTES);                    // [2][TC_N][TC_M]
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + NB * BUF_BYTES + SUM_BYTES);  // chunk converted, per buffer
  uint64_t *empty = full + NB;                                                      // chunk's MMAs done, per buffer
  uint64_t *win_done = empty + NB;                                                  // a window's MMAs done
  uint64_t *flushed = win_done + 1;                                                 // its main sums flushed
  uint64_t *fin = flushed + 1;                                                      // every issued MMA done
  uint32_t *tslot = reinterpret_cast<uint32_t *>(fin + 1);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tslot + 1);
  volatile int *issued_any = abort_flag + 1;

  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  // tiles of the result: all mtiles x ntiles, or for a set with itself (sym) only those with nt >= mt
  const int tiles = sym ? mtiles * (mtiles + 1) / 2 : mtiles * ntiles;
  const int ti = blockIdx.x % tiles, ks = blockIdx.x / tiles;
  int mt = ti % mtiles, nt = ti / mtiles;
  if (sym) {
    mt = 0;
    int r = ti;
    while (r >= mtiles - mt) {
      r -= mtiles - mt;
      mt++;
    }
    nt = mt + r;
  }
  const int m0 = mt * TC_M, n0 = nt * N;
  const long long kbeg = (long long)ks * kper;
  const long long kend = kbeg + kper < npoints ? kbeg + kper : npoints;
  const int nchunks = kend > kbeg ? int((kend - kbeg + TC_KC - 1) / TC_KC) : 0;

  for (int i = t; i < 2 * TC_N * TC_M; i += TC_THREADS + 32) sums[i] = 0.f;
  if (t == 0) {
    for (int i = 0; i < NB; i++) {
      ptx::mbar_init(&full[i], TC_THREADS);
      ptx::mbar_init(&empty[i], 1);
    }
    ptx::mbar_init(win_done, 1);
    ptx::mbar_init(flushed, TC_THREADS);
    ptx::mbar_init(fin, 1);
    *abort_flag = 0;
    *issued_any = 0;
    ptx::mbar_init_fence();
  }
  if (warp == 0) ptx::tmem_alloc(tslot, 512);
  ptx::tc_fence_before();
  __syncthreads();
  ptx::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t id = ptx::idesc_bf16_f32(TC_M, N, false), idn = ptx::idesc_bf16_f32(TC_M, N, true);
  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };
  auto wait = [&](uint64_t *bar, uint32_t parity) -> bool {
    const uint64_t t0 = ptx::global_ns();
    while (!ptx::mbar_try_wait(bar, parity)) {
      if (*abort_flag) return false;
      if (ptx::global_ns() - t0 > WAIT_NS) {
        fail();
        return false;
      }
    }
    return true;
  };

  if (warp == TC_THREADS / 32) {
    // issuer warp: lane 0 issues every chunk's 16 MMAs once its planes are in shared memory
    if (lane == 0) {
      int issued = 0;
      for (int c = 0; c < nchunks; c++) {
        const int bsel = c % NB;
        if (!wait(&full[bsel], uint32_t(c / NB) & 1u)) break;
        if (c % WIN == 0 && c > 0 && !wait(flushed, uint32_t(c / WIN - 1) & 1u)) break;  // main restarts
        ptx::tc_fence_after();
        const uint32_t ab = ptx::smem_u32(smem + bsel * BUF_BYTES), bb = ab + 4 * PLANE;
        uint64_t da[4], db[4];
#pragma unroll
        for (int p = 0; p < 4; p++) {
          da[p] = ptx::smem_desc_kmajor(ab + p * PLANE, 128, 256);
          db[p] = ptx::smem_desc_kmajor(bb + p * PLANE, 128, 256);
        }
        const bool fresh_main = (c % WIN) == 0, fresh_corr = c == 0;
        const uint32_t mre = tmem + COL_MAIN_RE, mim = tmem + COL_MAIN_IM;
        const uint32_t cre = tmem + COL_CORR_RE, cim = tmem + COL_CORR_IM;
        // planes: 0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo
        ptx::mma_bf16(mre, da[0], db[0], id, !fresh_main);
        ptx::mma_bf16(mre, da[2], db[2], id, true);
        ptx::mma_bf16(mim, da[0], db[2], id, !fresh_main);
        ptx::mma_bf16(mim, da[2], db[0], idn, true);
        ptx::mma_bf16(cre, da[0], db[1], id, !fresh_corr);
        ptx::mma_bf16(cre, da[1], db[0], id, true);
        ptx::mma_bf16(cre, da[1], db[1], id, true);
        ptx::mma_bf16(cre, da[2], db[3], id, true);
        ptx::mma_bf16(cre, da[3], db[2], id, true);
        ptx::mma_bf16(cre, da[3], db[3], id, true);
        ptx::mma_bf16(cim, da[0], db[3], id, !fresh_corr);
        ptx::mma_bf16(cim, da[1], db[2], id, true);
        ptx::mma_bf16(cim, da[1], db[3], id, true);
        ptx::mma_bf16(cim, da[2], db[1], idn, true);
        ptx::mma_bf16(cim, da[3], db[0], idn, true);
        ptx::mma_bf16(cim, da[3], db[1], idn, true);
        ptx::mma_commit(&empty[bsel]);
        if ((c % WIN) == WIN - 1 || c == nchunks - 1) ptx::mma_commit(win_done);
        issued = c + 1;
        *issued_any = 1;
      }
      if (issued > 0) ptx::mma_commit(fin);
    }
  } else {
    // converter warps: load, split and store the chunks; flush the main sums at each window's end
    const int row = t & (TC_M - 1), kh = t >> 7;
    const int acol = m0 + row, bcol = n0 + row;
    const bool aok = acol < Sa, bok = row < N && bcol < Sb;
    const int q = warp & 3, h = warp >> 2;
    const int myrow = q * 32 + lane;
    float2 pa[LOOK][8], pb[LOOK][8];
#pragma unroll
    for (int d = 0; d < LOOK - 1; d++)
      if (d < nchunks) {
        load_unit(a, Sa, acol, aok, kbeg + (long long)d * TC_KC + kh * 8, kend, pa[d]);
        load_unit(b, Sb, bcol, bok, kbeg + (long long)d * TC_KC + kh * 8, kend, pb[d]);
      }
    bool ok = true;
    for (int c = 0; c < nchunks && ok; c++) {
      const int bsel = c % NB;
      if (c + LOOK - 1 < nchunks) {
        const long long kn = kbeg + (long long)(c + LOOK - 1) * TC_KC + kh * 8;
        load_unit(a, Sa, acol, aok, kn, kend, pa[LOOK - 1]);
        load_unit(b, Sb, bcol, bok, kn, kend, pb[LOOK - 1]);
      }
      // the MMAs of chunk c - NB read this buffer
      if (c >= NB && !wait(&empty[bsel], uint32_t(c / NB - 1) & 1u)) break;
      unsigned char *bufA = smem + bsel * BUF_BYTES;
      store_unit(bufA, row, kh, pa[0]);
      store_unit(bufA + 4 * PLANE, row, kh, pb[0]);
      ptx::fence_proxy_async();
      ptx::mbar_arrive(&full[bsel]);
#pragma unroll
      for (int d = 0; d < LOOK - 1; d++)
#pragma unroll
        for (int u = 0; u < 8; u++) {
          pa[d][u] = pa[d + 1][u];
          pb[d][u] = pb[d + 1][u];
        }
      if ((c % WIN) == WIN - 1 || c == nchunks - 1) {
        // end of a window: add the main accumulators into the shared-memory running sums
        if (!wait(win_done, uint32_t(c / WIN) & 1u)) break;
        ptx::tc_fence_after();
        float *sum = sums + size_t(h) * TC_N * TC_M;
        for (int j0 = 0; j0 < N; j0 += 16) {
          float v[16];
          ptx::tmem_ld16(tmem + (uint32_t(q * 32) << 16) + (h ? COL_MAIN_IM : COL_MAIN_RE) + uint32_t(j0), v);
#pragma unroll
          for (int u = 0; u < 16; u++) sum[(j0 + u) * TC_M + myrow] += v[u];
        }
        ptx::tc_fence_before();
        ptx::mbar_arrive(flushed);
      }
    }
    // epilogue: running sums plus the correction accumulators (complete once the last window is done)
    if (!*abort_flag) {
      ptx::tc_fence_after();
      const int ia = m0 + myrow;
      const float *sum = sums + size_t(h) * TC_N * TC_M;
      float *dst = partial + ((size_t(ks) * 2 + h) * size_t(Sa) + size_t(ia)) * size_t(Sb) + n0;
      for (int j0 = 0; j0 < N; j0 += 16) {
        float v[16];
        if (nchunks > 0) {
          ptx::tmem_ld16(tmem + (uint32_t(q * 32) << 16) + (h ? COL_CORR_IM : COL_CORR_RE) + uint32_t(j0), v);
        } else {
#pragma unroll
          for (int u = 0; u < 16; u++) v[u] = 0.f;
        }
        if (ia < Sa) {
#pragma unroll
          for (int u = 0; u < 16; u++)
            if (n0 + j0 + u < Sb) dst[j0 + u] = sum[(j0 + u) * TC_M + myrow] + v[u];
        }
      }
    }
  }
  // tensor memory is freed only after every issued MMA has completed (also after an abort)
  ptx::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    if (*issued_any) (void)ptx::mbar_wait_bounded(fin, 0u, WAIT_NS);
    ptx::tc_fence_after();
    ptx::tmem_dealloc(tmem, 512);
  }
}

// out[i][j] = dv * sum over the point splits, in split order, in FP64; for a set with itself (sym) the
// tiles below the diagonal were not computed and take the conjugate of their mirror
__global__ void overlap_tc_reduce(const float *__restrict__ partial, int nsplit, int Sa, int Sb, int sym, double dv,
                                  double2 *__restrict__ out) {
  const long long n = (long long)Sa * Sb;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int i = int(e / Sb), j = int(e % Sb);
    const bool mirror = sym && (i / TC_M) > (j / TC_M);
    const long long f = mirror ? (long long)j * Sb + i : e;
    double re = 0.0, im = 0.0;
    for (int z = 0; z < nsplit; z++) {
      re += double(partial[(2LL * z) * n + f]);
      im += double(partial[(2LL * z + 1) * n + f]);
    }
    out[e] = make_double2(dv * re, mirror ? -dv * im : dv * im);
  }
}

}  // namespace

void launch_overlap_tc(Ctx &ctx, const float2 *a, int Sa, const float2 *b, int Sb, long long npoints, double dv,
                       double2 *out) {
  INQB_REQUIRE(Sa > 0 && Sb > 0 && npoints > 0, INQB_ERR_ARG, "empty overlap");
  const int mtiles = (Sa + TC_M - 1) / TC_M;
  const int N = Sb < TC_N ? (Sb + 15) / 16 * 16 : TC_N;
  const int ntiles = (Sb + N - 1) / N;
  // a set with itself: S is Hermitian, so only the tiles on and above the diagonal are computed
  const int sym = (a == b && Sa == Sb && N == TC_M) ? 1 : 0;
  const int tiles = sym ? mtiles * (mtiles + 1) / 2 : mtiles * ntiles;
  int nsplit = ctx.device_sms / tiles;  // the split (and so the rounding) does not follow grid_sms
  if (nsplit < 1) nsplit = 1;
  long long kper = ((npoints + nsplit - 1) / nsplit + TC_KC - 1) / TC_KC * TC_KC;
  nsplit = int((npoints + kper - 1) / kper);  // every split holds at least one point
  float *partial = static_cast<float *>(dev_alloc(ctx, sizeof(float) * size_t(nsplit) * 2 * Sa * Sb));
  ensure_smem_attr(reinterpret_cast<const void *>(overlap_tc_kernel), TC_SMEM);
  overlap_tc_kernel<<<unsigned(tiles * nsplit), TC_THREADS + 32, TC_SMEM, ctx.stream>>>(
      a, Sa, b, Sb, npoints, mtiles, ntiles, N, kper, sym, partial, ctx.d_err);
  INQB_CUDA(cudaGetLastError());
  ctx.launches++;
  const long long n = (long long)Sa * Sb;
  long long blocks = (n + 255) / 256;
  if (blocks > 4L * ctx.num_sms) blocks = 4L * ctx.num_sms;
  overlap_tc_reduce<<<unsigned(blocks), 256, 0, ctx.stream>>>(partial, nsplit, Sa, Sb, sym, dv, out);
  INQB_CUDA(cudaGetLastError());
  ctx.launches++;
  dev_free(ctx, partial);
}

}  // namespace inqb
