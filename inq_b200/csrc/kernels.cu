// Nonlocal projector kernels and the orbital-set kernels around the FFT passes.
//
// Every reduction here has a fixed order (warp shuffles in a fixed tree, per-block
// partials summed in index order by a second kernel), so results are bitwise
// reproducible run to run; no floating-point atomics are used anywhere.

#include "inqb_internal.h"
#include "ptx.cuh"

#include <algorithm>
#include <mutex>

namespace inqb {

static inline unsigned grid_for(long long n, int threads, long long cap = 148LL * 64) {
  long long g = (n + threads - 1) / threads;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return unsigned(g);
}

#define LAUNCHED(ctx)                   \
  do {                                  \
    INQB_CUDA(cudaGetLastError());      \
    (ctx).launches++;                   \
  } while (0)

// ------------------------------------------------------------------ nonlocal tables
// gcoef[p][i][l] = dV * e^{+i kA.pos} * M[p][l][i]   (gather side, projector_all.hpp:120-128,156)
// hcoef[h][l]    = e^{-i kA.pos} * M[p][l][i]        (apply side, projector_all.hpp:281-287)
__global__ void nl_tables_kernel(int nproj, int maxsph, const int *__restrict__ pt, const float *__restrict__ pos,
                                 const double *__restrict__ mat, double dv, double k0, double k1, double k2,
                                 double2 *gcoef, float2 *gcoef32) {
  const long long total = (long long)nproj * maxsph;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int p = int(idx / maxsph), i = int(idx % maxsph);
    double2 ph = make_double2(0.0, 0.0);
    if (pt[idx] >= 0) {
      // dot(kpoint, pos) of the reference: covariant double times float contravariant
      double arg = k0 * double(pos[idx * 3 + 0]) + k1 * double(pos[idx * 3 + 1]) + k2 * double(pos[idx * 3 + 2]);
      double sn, cs;
      sincos(arg, &sn, &cs);
      ph = make_double2(cs, sn);
    }
    for (int l = 0; l < 4; l++) {
      double m = mat[((long long)p * 4 + l) * maxsph + i];
      double2 g = make_double2(dv * m * ph.x, dv * m * ph.y);
      gcoef[idx * 4 + l] = g;
      gcoef32[idx * 4 + l] = make_float2(float(g.x), float(g.y));
    }
  }
}

__global__ void nl_hit_kernel(long long total, const int *__restrict__ hit, int maxsph, const float *__restrict__ pos,
                              const double *__restrict__ mat, double k0, double k1, double k2, double2 *hcoef,
                              float2 *hcoef32) {
  for (long long h = blockIdx.x * (long long)blockDim.x + threadIdx.x; h < total;
       h += (long long)gridDim.x * blockDim.x) {
    const long long idx = hit[h];
    const int p = int(idx / maxsph), i = int(idx % maxsph);
    double arg = k0 * double(pos[idx * 3 + 0]) + k1 * double(pos[idx * 3 + 1]) + k2 * double(pos[idx * 3 + 2]);
    double sn, cs;
    sincos(arg, &sn, &cs);
    for (int l = 0; l < 4; l++) {
      double m = mat[((long long)p * 4 + l) * maxsph + i];
      double2 c = make_double2(m * cs, -m * sn);
      hcoef[h * 4 + l] = c;
      hcoef32[h * 4 + l] = make_float2(float(c.x), float(c.y));
    }
  }
}

void launch_nl_tables(Ctx &ctx, const Basis &b, Hamiltonian &h, const double kA[3]) {
  Projectors &P = h.proj;
  if (P.nproj == 0 || P.maxsph == 0) return;
  const double dv = b.volume / double(b.npoints);
  const long long total = (long long)P.nproj * P.maxsph;
  nl_tables_kernel<<<grid_for(total, 256), 256, 0, ctx.stream>>>(P.nproj, P.maxsph, P.d_pt, P.d_pos, P.d_mat, dv,
                                                                 kA[0], kA[1], kA[2], P.d_gcoef, P.d_gcoef32);
  LAUNCHED(ctx);
  if (P.total > 0) {
    nl_hit_kernel<<<grid_for(P.total, 256), 256, 0, ctx.stream>>>(P.total, P.d_hit, P.maxsph, P.d_pos, P.d_mat, kA[0],
                                                                  kA[1], kA[2], P.d_hcoef, P.d_hcoef32);
    LAUNCHED(ctx);
  }
  for (int i = 0; i < 3; i++) P.kA[i] = kA[i];
}

// ------------------------------------------------------------------ bulk-copy kernels: shared pieces
// acc + a * b as four fused multiply-adds (one rounding per product term)
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
template <typename T> __device__ __forceinline__ T cmac(T acc, T a, T b) {
  acc.x = fma_rn(a.x, b.x, acc.x);
  acc.x = fma_rn(-a.y, b.y, acc.x);
  acc.y = fma_rn(a.x, b.y, acc.y);
  acc.y = fma_rn(a.y, b.x, acc.y);
  return acc;
}

// The bulk-copy forms of the projection and the apply run NLA_NT compute threads beside one producer
// warp that moves whole rows of states (contiguous in the state-fastest layout) with bulk
// asynchronous copies.  The compute threads synchronise among themselves on named barrier 1.
constexpr int NLA_NT = 128;

__device__ __forceinline__ void nla_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NLA_NT) : "memory"); }
// the same barrier, returning whether any compute thread passed a nonzero value (uniform result)
__device__ __forceinline__ bool nla_sync_or(int v) {
  uint32_t r;
  asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
               : "=r"(r)
               : "r"(v), "n"(NLA_NT)
               : "memory");
  return r != 0;
}
// bounded wait on an mbarrier phase (2 s); false, with the CTA's abort flag and the error flag raised,
// on expiry, and false as soon as another thread of the CTA has raised the abort flag
__device__ __forceinline__ bool nla_wait(uint64_t *b, uint32_t parity, volatile int *abort_flag, int *err) {
  const uint64_t t0 = ptx::global_ns();
  while (!ptx::mbar_try_wait(b, parity)) {
    if (*abort_flag) return false;
    if (ptx::global_ns() - t0 > 2000000000ull) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
  return true;
}

// ------------------------------------------------------------------ nonlocal projection
// proj[p][l][s] = sum_i gcoef[p][i][l] * psi[pt_i][s]; projD = coeff[p] . proj
// (projector_all.hpp:113-211).  Stage 1: CTA = (projector p, range rg of its sphere points, chunk of
// 32 K states); each of its 8 warps takes a contiguous run of the range, reads 32 point indices with
// one coalesced load and hands them out by shuffles, and keeps NP points in flight; a lane holds K
// states 32 apart, so each point costs K contiguous 256-byte segments of the state-fastest row.  The
// warp partials are summed in order into partial[p][rg][l][s].  Stage 2 sums the ranges in order and
// applies the KB coefficients.
constexpr int NLP_WARPS = 8, NLP_RANGES = 16;  // 16 ranges: the bulk projection 181 us against 218 with 8 (FP64, 96^3 x 256)

template <typename R, typename A, int K>
__global__ void __launch_bounds__(NLP_WARPS * 32) nl_project_kernel(const C2<R> *__restrict__ psi, int S,
                                                                    const int *__restrict__ pt,
                                                                    const C2<A> *__restrict__ gcoef,
                                                                    const int *__restrict__ npts, int maxsph,
                                                                    C2<A> *__restrict__ partial) {
  using T = C2<R>;
  using TA = C2<A>;
  constexpr int NP = 4;  // points in flight per warp
  __shared__ TA part[NLP_WARPS][4][32 * K];
  const int p = blockIdx.x, rg = blockIdx.y;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int sbase = blockIdx.z * 32 * K;
  const int np = npts[p];
  const int nr = int(gridDim.y);  // ranges of a sphere
  const int rper = (np + nr - 1) / nr;
  const int r0 = rg * rper, r1 = min(np, r0 + rper);
  const int per = (max(r1 - r0, 0) + NLP_WARPS - 1) / NLP_WARPS;
  const int i0 = r0 + wp * per, i1 = min(r1, i0 + per);
  TA acc[K][4];
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int l = 0; l < 4; l++) acc[k][l] = mk<TA>(A(0), A(0));
  const long long rowbase = (long long)p * maxsph;
  for (int base = i0; base < i1; base += 32) {
    const int cnt = min(32, i1 - base);
    const int qv = lane < cnt ? __ldg(&pt[rowbase + base + lane]) : 0;
    for (int j = 0; j < cnt; j += NP) {
      T x[NP][K];
#pragma unroll
      for (int u = 0; u < NP; u++) {
        const long long q = __shfl_sync(0xffffffffu, qv, (j + u) & 31);
#pragma unroll
        for (int k = 0; k < K; k++) {
          const int s = sbase + k * 32 + lane;
          x[u][k] = (j + u < cnt && s < S) ? psi[q * S + s] : mk<T>(R(0), R(0));
        }
      }
#pragma unroll
      for (int u = 0; u < NP; u++) {
        if (j + u < cnt) {
          const TA *g = gcoef + (rowbase + base + j + u) * 4;
          TA gl[4];
#pragma unroll
          for (int l = 0; l < 4; l++) gl[l] = g[l];
#pragma unroll
          for (int k = 0; k < K; k++) {
            const TA v = mk<TA>(A(x[u][k].x), A(x[u][k].y));
#pragma unroll
            for (int l = 0; l < 4; l++) acc[k][l] = cadd(acc[k][l], cmul(gl[l], v));
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < K; k++)
#pragma unroll
    for (int l = 0; l < 4; l++) part[wp][l][k * 32 + lane] = acc[k][l];
  __syncthreads();
  for (int e = threadIdx.x; e < 4 * 32 * K; e += blockDim.x) {
    const int l = e / (32 * K), sl = e % (32 * K);
    const int s = sbase + sl;
    TA t = part[0][l][sl];
    for (int w = 1; w < NLP_WARPS; w++) t = cadd(t, part[w][l][sl]);
    if (s < S) partial[(((long long)p * nr + rg) * 4 + l) * S + s] = t;
  }
}

// Bulk-copy form of the projection.  CTA = (projector p, range rg of its sphere points, chunk of up to
// NLA_NT * J states).  The producer warp copies the range's points in batches of KB -- each point's
// row of the chunk's states and the point's four gather coefficients -- into a ring of NLP_NS stages;
// each compute thread owns J states and sums over the range's points in order (a batch's points first,
// then the batch sums, so the chains stay as short as in nl_project_kernel).  No cross-warp reduction:
// the thread writes its states of partial[p][rg][l][s] directly.
constexpr int NLP_NS = 3;

template <typename R, typename A, int J>
__global__ void __launch_bounds__(NLA_NT + 32) nl_project_bulk_kernel(const C2<R> *psi, int S,
                                                                       const int *__restrict__ pt,
                                                                       const C2<A> *gcoef,
                                                                       const int *__restrict__ npts, int maxsph,
                                                                       int KB, C2<A> *__restrict__ partial, int *err) {
  using T = C2<R>;
  using TA = C2<A>;
  using namespace ptx;
  extern __shared__ __align__(128) unsigned char smem[];
  const int p = blockIdx.x, rg = blockIdx.y;
  const int s0 = blockIdx.z * NLA_NT * J;
  const int SCmax = min(NLA_NT * J, S);  // row stride of the stages
  const int SC = min(NLA_NT * J, S - s0);  // states of this chunk
  T *rows = reinterpret_cast<T *>(smem);                                     // [NS][KB][SCmax]
  TA *gs = reinterpret_cast<TA *>(rows + size_t(NLP_NS) * KB * SCmax);        // [NS][KB][4]
  uint64_t *full = reinterpret_cast<uint64_t *>(gs + size_t(NLP_NS) * KB * 4);  // stage loaded
  uint64_t *done = full + NLP_NS;                                            // stage consumed
  volatile int *abort_flag = reinterpret_cast<volatile int *>(done + NLP_NS);
  const int np = npts[p];
  const int nr = int(gridDim.y);  // ranges of a sphere
  const int rper = (np + nr - 1) / nr;
  const int r0 = rg * rper, r1 = min(np, r0 + rper);
  const int n = max(r1 - r0, 0);
  const int nbatch = (n + KB - 1) / KB;
  const long long rowbase = (long long)p * maxsph;
  const uint32_t row_bytes = uint32_t(SC) * uint32_t(sizeof(T));
  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int st = 0; st < NLP_NS; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&done[st], NLA_NT);
    }
    mbar_init_fence();
  }
  __syncthreads();

  if (threadIdx.x >= NLA_NT) {
    // producer warp: lane q copies point q of a batch, lane 0 also the batch's coefficients
    const int lane = threadIdx.x - NLA_NT;
    auto issue = [&](int st, int b) {
      const int base = r0 + b * KB;
      const int nb = min(KB, r1 - base);
      const long long q = lane < nb ? (long long)pt[rowbase + base + lane] : 0;
      if (lane == 0) mbar_expect_tx(&full[st], uint32_t(nb) * (row_bytes + 4 * uint32_t(sizeof(TA))));
      __syncwarp();
      if (lane < nb) bulk_load(rows + (size_t(st) * KB + lane) * SCmax, psi + q * S + s0, row_bytes, &full[st]);
      if (lane == 0)
        bulk_load(gs + size_t(st) * KB * 4, gcoef + (rowbase + base) * 4, uint32_t(nb) * 4 * uint32_t(sizeof(TA)),
                  &full[st]);
    };
    int issued = 0;  // batches whose copies were issued
    for (int b = 0; b < NLP_NS && b < nbatch; b++) issue(b, b), issued++;
    for (int b = 0; b + NLP_NS < nbatch; b++) {
      const int st = b % NLP_NS;
      if (!nla_wait(&done[st], uint32_t(b / NLP_NS) & 1u, abort_flag, err)) break;
      issue(st, b + NLP_NS);
      issued++;
    }
    // after an abort the compute threads may leave early: wait (bounded) for every issued copy to land
    // before the CTA's shared memory is released (on the normal path these phases are already complete)
    for (int b = issued - NLP_NS < 0 ? 0 : issued - NLP_NS; b < issued; b++)
      mbar_wait_bounded(&full[b % NLP_NS], uint32_t(b / NLP_NS) & 1u, 2000000000ull);
    return;
  }

  const int tid = threadIdx.x;
  TA acc[J][4];
#pragma unroll
  for (int j = 0; j < J; j++)
#pragma unroll
    for (int l = 0; l < 4; l++) acc[j][l] = mk<TA>(A(0), A(0));
  for (int b = 0; b < nbatch; b++) {
    const int st = b % NLP_NS;
    const bool ok = nla_wait(&full[st], uint32_t(b / NLP_NS) & 1u, abort_flag, err);
    if (nla_sync_or(!ok || *abort_flag)) break;
    const int nb = min(KB, r1 - (r0 + b * KB));
    const T *rw = rows + size_t(st) * KB * SCmax;
    const TA *g = gs + size_t(st) * KB * 4;
    TA bacc[J][4];
#pragma unroll
    for (int j = 0; j < J; j++)
#pragma unroll
      for (int l = 0; l < 4; l++) bacc[j][l] = mk<TA>(A(0), A(0));
    for (int q = 0; q < nb; q++) {
      TA gl[4];
#pragma unroll
      for (int l = 0; l < 4; l++) gl[l] = g[q * 4 + l];
#pragma unroll
      for (int j = 0; j < J; j++) {
        const int sl = tid + j * NLA_NT;
        if (sl < SC) {
          const T x = rw[(size_t)q * SCmax + sl];
          const TA v = mk<TA>(A(x.x), A(x.y));
          // fused products in single precision (0.10 against 0.11 ms at 96^3 x 256); separate ones in
          // double (0.18 against 0.19 ms)
          if constexpr (sizeof(A) == 4) {
#pragma unroll
            for (int l = 0; l < 4; l++) bacc[j][l] = cmac(bacc[j][l], gl[l], v);
          } else {
#pragma unroll
            for (int l = 0; l < 4; l++) bacc[j][l] = cadd(bacc[j][l], cmul(gl[l], v));
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < J; j++)
#pragma unroll
      for (int l = 0; l < 4; l++) acc[j][l] = cadd(acc[j][l], bacc[j][l]);
    mbar_arrive(&done[st]);  // the producer refills the stage
  }
#pragma unroll
  for (int j = 0; j < J; j++) {
    const int sl = tid + j * NLA_NT;
    if (sl < SC) {
#pragma unroll
      for (int l = 0; l < 4; l++) partial[(((long long)p * nr + rg) * 4 + l) * S + s0 + sl] = acc[j][l];
    }
  }
}

template <typename R, typename A>
__global__ void nl_project_finish_kernel(const C2<A> *__restrict__ partial, int nproj, int nr, int S,
                                         const A *__restrict__ coeff, C2<R> *projraw, C2<R> *projD) {
  using T = C2<R>;
  using TA = C2<A>;
  const long long n = (long long)nproj * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int p = int(e / S), s = int(e % S);
    TA pr[4];
#pragma unroll
    for (int l = 0; l < 4; l++) {
      TA t = partial[(((long long)p * nr) * 4 + l) * S + s];
      for (int rg = 1; rg < nr; rg++) t = cadd(t, partial[(((long long)p * nr + rg) * 4 + l) * S + s]);
      pr[l] = t;
      projraw[((long long)p * 4 + l) * S + s] = mk<T>(R(t.x), R(t.y));
    }
#pragma unroll
    for (int l = 0; l < 4; l++) {
      TA t = mk<TA>(A(0), A(0));
#pragma unroll
      for (int j = 0; j < 4; j++) t = cadd(t, cscale(pr[j], coeff[(p * 4 + l) * 4 + j]));
      projD[((long long)p * 4 + l) * S + s] = mk<T>(R(t.x), R(t.y));
    }
  }
}

template <typename R>
void launch_nl_project(Ctx &ctx, const Basis &b, const Hamiltonian &h, const C2<R> *psi, int S, C2<R> *projraw,
                       C2<R> *projD) {
  const Projectors &P = h.proj;
  if (P.nproj == 0) return;
  const bool dbl = sizeof(R) == 8 || ctx.mixed_compute != 0;  // double-precision coefficients and sums
  // ranges per sphere (option nl_project_ranges; the summation order follows it)
  const int NR = ctx.nl_project_ranges > 0 ? ctx.nl_project_ranges : NLP_RANGES;
  const size_t pbytes = size_t(P.nproj) * NR * 4 * S * (dbl ? sizeof(double2) : sizeof(float2));
  void *partial = dev_alloc(ctx, pbytes);
  const long long fin = (long long)P.nproj * S;
  // bulk form: rows of 16-byte multiples, and (automatic choice) enough CTAs to fill the device; the
  // choice (and so the summation order) follows the device's SM count, not the grid_sms option
  constexpr int JB = 2;
  const size_t row_bytes = size_t(S) * sizeof(C2<R>);
  const int nchunks = (S + NLA_NT * JB - 1) / (NLA_NT * JB);
  const bool bulk_ok = row_bytes % 16 == 0 && reinterpret_cast<uintptr_t>(psi) % 16 == 0;
  const bool bulk = bulk_ok && (ctx.nl_bulk > 0 ||
                                (ctx.nl_bulk == 0 && (long long)P.nproj * NR * nchunks >= 2LL * ctx.device_sms));
  if (bulk) {
    const int SCmax = std::min(NLA_NT * JB, S);
    const size_t srow = size_t(SCmax) * sizeof(C2<R>);
    int KB = ctx.nl_project_points > 0 ? ctx.nl_project_points : int(16384 / srow);  // about 16 KB of rows per stage
    KB = KB < 1 ? 1 : (KB > 32 ? 32 : KB);
    const size_t abytes = dbl ? sizeof(double2) : sizeof(float2);
    auto smem_of = [&](int kb) {
      return size_t(NLP_NS) * kb * srow + size_t(NLP_NS) * kb * 4 * abytes + 2 * NLP_NS * sizeof(uint64_t) + 16;
    };
    while (KB > 1 && smem_of(KB) > size_t(ctx.max_smem_optin)) KB--;  // an option asking for more than fits
    const size_t smem = smem_of(KB);
    const dim3 grid(P.nproj, NR, nchunks);
    if (dbl) {
      auto kern = nl_project_bulk_kernel<R, double, JB>;
      ensure_smem_attr(reinterpret_cast<const void *>(kern), smem);
      kern<<<grid, NLA_NT + 32, smem, ctx.stream>>>(psi, S, P.d_pt, P.d_gcoef, P.d_npts, P.maxsph, KB,
                                                    static_cast<double2 *>(partial), ctx.d_err);
      LAUNCHED(ctx);
      nl_project_finish_kernel<R, double><<<grid_for(fin, 256), 256, 0, ctx.stream>>>(
          static_cast<const double2 *>(partial), P.nproj, NR, S, P.d_coeff, projraw, projD);
    } else {
      auto kern = nl_project_bulk_kernel<R, float, JB>;
      ensure_smem_attr(reinterpret_cast<const void *>(kern), smem);
      kern<<<grid, NLA_NT + 32, smem, ctx.stream>>>(psi, S, P.d_pt, P.d_gcoef32, P.d_npts, P.maxsph, KB,
                                                    static_cast<float2 *>(partial), ctx.d_err);
      LAUNCHED(ctx);
      nl_project_finish_kernel<R, float><<<grid_for(fin, 256), 256, 0, ctx.stream>>>(
          static_cast<const float2 *>(partial), P.nproj, NR, S, P.d_coeff32, projraw, projD);
    }
    LAUNCHED(ctx);
    dev_free(ctx, partial);
    return;
  }
  if (dbl) {
    constexpr int K = 2;
    dim3 grid(P.nproj, NR, (S + 32 * K - 1) / (32 * K));
    nl_project_kernel<R, double, K><<<grid, NLP_WARPS * 32, 0, ctx.stream>>>(
        psi, S, P.d_pt, P.d_gcoef, P.d_npts, P.maxsph, static_cast<double2 *>(partial));
    LAUNCHED(ctx);
    nl_project_finish_kernel<R, double><<<grid_for(fin, 256), 256, 0, ctx.stream>>>(
        static_cast<const double2 *>(partial), P.nproj, NR, S, P.d_coeff, projraw, projD);
  } else {
    // two states per lane (64-state chunks) in single precision too: more CTAs with fewer registers
    // hide the gather latency better (measured 168 us against 202 us with four at 96^3 x 256)
    constexpr int K = 2;
    dim3 grid(P.nproj, NR, (S + 32 * K - 1) / (32 * K));
    nl_project_kernel<R, float, K><<<grid, NLP_WARPS * 32, 0, ctx.stream>>>(
        psi, S, P.d_pt, P.d_gcoef32, P.d_npts, P.maxsph, static_cast<float2 *>(partial));
    LAUNCHED(ctx);
    nl_project_finish_kernel<R, float><<<grid_for(fin, 256), 256, 0, ctx.stream>>>(
        static_cast<const float2 *>(partial), P.nproj, NR, S, P.d_coeff32, projraw, projD);
  }
  LAUNCHED(ctx);
  dev_free(ctx, partial);
}

// out[pt][s] = nonlocal term (ks_hamiltonian::non_local, ks_hamiltonian.hpp:106-120)
template <typename R>
__global__ void nl_scatter_kernel(long long npoints, int S, const int *__restrict__ offs, const int *__restrict__ hit,
                                  const C2<R> *__restrict__ hcoef, const C2<R> *__restrict__ projD, int maxsph,
                                  C2<R> *out) {
  using T = C2<R>;
  const long long total = npoints * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long pt = e / S;
    const int s = int(e % S);
    T acc = mk<T>(R(0), R(0));
    for (int hh = offs[pt]; hh < offs[pt + 1]; hh++) {
      const int p = hit[hh] / maxsph;
#pragma unroll
      for (int l = 0; l < 4; l++) acc = cadd(acc, cmul(hcoef[(long long)hh * 4 + l], projD[((long long)p * 4 + l) * S + s]));
    }
    out[e] = acc;
  }
}

template <typename R>
void launch_nl_scatter(Ctx &ctx, const Basis &b, const Hamiltonian &h, const C2<R> *projD, int S, C2<R> *out) {
  const Projectors &P = h.proj;
  const C2<R> *hc;
  if constexpr (sizeof(R) == 8) hc = P.d_hcoef;
  else hc = P.d_hcoef32;
  nl_scatter_kernel<R><<<grid_for(b.npoints * S, 256), 256, 0, ctx.stream>>>(b.npoints, S, P.d_offs, P.d_hit, hc,
                                                                             projD, P.maxsph, out);
  LAUNCHED(ctx);
}

// out[pt][s] += nonlocal term at the grid points that lie in a sphere (ks_hamiltonian.hpp:153,
// projector_all.hpp:276-288), hits of a point summed in projector order, no atomics; optionally scaled,
// out += scale * term (a Horner step of a Taylor exponential).
// Owner computes: one warp per (grid point with sphere hits, chunk of 32 * U states), lanes over states.
// The point's record gives its first hit and projector in one load, so the coefficient, projection and
// output reads are all issued together (a two-level dependency instead of point -> CSR -> hit ->
// projection); splitting the states into chunks keeps the registers low and many warps resident.
template <typename R>
__global__ void __launch_bounds__(128) nl_apply_kernel(long long nitems, int nchunks, int S,
                                                          const int4 *__restrict__ hrec, const int *__restrict__ hitp,
                                                          const C2<R> *__restrict__ hcoef,
                                                          const C2<R> *__restrict__ projD, C2<R> *__restrict__ out,
                                                          bool scaled, C2<R> scale) {
  using T = C2<R>;
  constexpr int U = 16 / sizeof(R);  // states per lane: 4 single, 2 double
  const int lane = threadIdx.x & 31;
  const long long warp = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  // the record of the warp's next item is requested while the current one is processed
  int4 next = warp < nitems ? hrec[warp / nchunks] : make_int4(0, 0, 0, 0);
  for (long long it = warp; it < nitems; it += nwarps) {
    const int s0 = int(it % nchunks) * (32 * U);
    const int4 rec = next;
    if (it + nwarps < nitems) next = hrec[(it + nwarps) / nchunks];
    const long long pt = rec.x;
    const int h0 = rec.y, nh = rec.z, p0 = rec.w;
    T hc[4], o[U], pd[4][U];
#pragma unroll
    for (int l = 0; l < 4; l++) hc[l] = hcoef[(long long)h0 * 4 + l];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int s = s0 + u * 32 + lane;
      if (s < S) {
        o[u] = out[pt * S + s];
#pragma unroll
        for (int l = 0; l < 4; l++) pd[l][u] = projD[((long long)p0 * 4 + l) * S + s];
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int s = s0 + u * 32 + lane;
      if (s >= S) continue;
      T accv = mk<T>(R(0), R(0));
#pragma unroll
      for (int l = 0; l < 4; l++) accv = cadd(accv, cmul(hc[l], pd[l][u]));
      for (int k = 1; k < nh; k++) {
        const int h = h0 + k;
        const int p = hitp[h];
#pragma unroll
        for (int l = 0; l < 4; l++)
          accv = cadd(accv, cmul(hcoef[(long long)h * 4 + l], projD[((long long)p * 4 + l) * S + s]));
      }
      const long long e = pt * S + s;
      out[e] = cadd(o[u], scaled ? cmul(scale, accv) : accv);
    }
  }
}

// Bulk-copy form of the apply.  A CTA takes batches of KB consecutive hit points: a producer warp
// copies the points' output rows (S contiguous states each) into shared memory with bulk asynchronous
// copies, the compute threads add the nonlocal term to them there, and the producer writes the rows
// back with bulk copies.  Two stages overlap one batch's copies with the next batch's arithmetic, and
// the copy engine keeps the bytes in flight that the register-held form could not.  The terms are
// summed in nl_apply_kernel's order, with fused multiply-adds (single precision: 0.19 against 0.20 ms
// at 96^3 x 256, and six CTAs per SM, 0.18 ms; double: 0.31 against 0.32 ms).
constexpr int NLA_NS = 2;     // stages
constexpr int NLA_KMAX = 32;  // largest batch (one producer lane per row)

template <typename R, int J>
__global__ void __launch_bounds__(NLA_NT + 32, sizeof(R) == 4 ? 6 : 3) nl_apply_bulk_kernel(long long nrec, int KB, int S,
                                                                     const int4 *__restrict__ hrec,
                                                                     const int *__restrict__ hitp,
                                                                     const C2<R> *__restrict__ hcoef,
                                                                     const C2<R> *__restrict__ projD, C2<R> *out,
                                                                     bool scaled, C2<R> scale, int *err) {
  using T = C2<R>;
  using namespace ptx;
  extern __shared__ __align__(128) unsigned char smem[];
  T *rows = reinterpret_cast<T *>(smem);                                 // [NS][KB][S]
  T *hcs = rows + size_t(NLA_NS) * KB * S;                               // [KB][4] first-hit coefficients
  int4 *recs = reinterpret_cast<int4 *>(hcs + NLA_KMAX * 4);             // [NS][KMAX]
  uint64_t *full = reinterpret_cast<uint64_t *>(recs + NLA_NS * NLA_KMAX);  // rows and records loaded
  uint64_t *done = full + NLA_NS;                                        // rows computed
  volatile int *abort_flag = reinterpret_cast<volatile int *>(done + NLA_NS);
  const long long nbatch = (nrec + KB - 1) / KB;
  const uint32_t row_bytes = uint32_t(S) * uint32_t(sizeof(T));
  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int st = 0; st < NLA_NS; st++) {
      mbar_init(&full[st], 1);
      mbar_init(&done[st], NLA_NT);
    }
    mbar_init_fence();
  }
  __syncthreads();
  auto wait_bar = [&](uint64_t *b, uint32_t parity) { return nla_wait(b, parity, abort_flag, err); };

  if (threadIdx.x >= NLA_NT) {
    // producer warp: lane q copies row q of a batch in and out
    const int lane = threadIdx.x - NLA_NT;
    auto issue = [&](int st, long long b) {
      const long long k0 = b * KB;
      const int nb = int(min((long long)KB, nrec - k0));
      int4 rec = make_int4(0, 0, 0, 0);
      if (lane < nb) {
        rec = hrec[k0 + lane];
        recs[st * NLA_KMAX + lane] = rec;
      }
      __threadfence_block();
      __syncwarp();
      if (lane == 0) mbar_expect_tx(&full[st], uint32_t(nb) * row_bytes);
      __syncwarp();
      if (lane < nb) bulk_load(rows + (size_t(st) * KB + lane) * S, out + (long long)rec.x * S, row_bytes, &full[st]);
    };
    int issued = 0;  // batches whose loads were issued, in order
    for (int st = 0; st < NLA_NS; st++) {
      const long long b = blockIdx.x + (long long)st * gridDim.x;
      if (b < nbatch) issue(st, b), issued++;
    }
    int k = 0;
    for (long long b = blockIdx.x; b < nbatch; b += gridDim.x, k++) {
      const int st = k % NLA_NS;
      if (!wait_bar(&done[st], uint32_t(k / NLA_NS) & 1u)) break;
      const int nb = int(min((long long)KB, nrec - b * KB));
      if (lane < nb)
        bulk_store(out + (long long)recs[st * NLA_KMAX + lane].x * S, rows + (size_t(st) * KB + lane) * S, row_bytes);
      bulk_commit();
      bulk_wait_read0();  // the stage may be refilled once its rows are read out
      __syncwarp();
      const long long bn = b + (long long)NLA_NS * gridDim.x;
      if (bn < nbatch) issue(st, bn), issued++;
    }
    // after an abort the compute threads may leave early: wait (bounded) for every issued load to land
    // before the CTA's shared memory is released (on the normal path these phases are already complete)
    for (int i = issued - NLA_NS < 0 ? 0 : issued - NLA_NS; i < issued; i++)
      mbar_wait_bounded(&full[i % NLA_NS], uint32_t(i / NLA_NS) & 1u, 2000000000ull);
    bulk_wait0();
    return;
  }

  const int tid = threadIdx.x;
  T pd[J][4];
  int pprev = -1;
  int i = 0;
  for (long long b = blockIdx.x; b < nbatch; b += gridDim.x, i++) {
    const int st = i % NLA_NS;
    const bool ok = wait_bar(&full[st], uint32_t(i / NLA_NS) & 1u);
    if (nla_sync_or(!ok || *abort_flag)) break;
    const int nb = int(min((long long)KB, nrec - b * KB));
    const int4 *rc = recs + st * NLA_KMAX;
    T *rw = rows + size_t(st) * KB * S;
    // the batch's first-hit coefficients, requested together
    for (int t = tid; t < nb * 4; t += NLA_NT) hcs[t] = hcoef[(long long)rc[t >> 2].y * 4 + (t & 3)];
    nla_sync();
    for (int q = 0; q < nb; q++) {
      const int4 rec = rc[q];
      const int h0 = rec.y, nh = rec.z, p0 = rec.w;
      if (p0 != pprev) {
#pragma unroll
        for (int j = 0; j < J; j++) {
          const int s = tid + j * NLA_NT;
          if (s < S) {
#pragma unroll
            for (int l = 0; l < 4; l++) pd[j][l] = projD[((long long)p0 * 4 + l) * S + s];
          }
        }
        pprev = p0;
      }
      T hc[4];
#pragma unroll
      for (int l = 0; l < 4; l++) hc[l] = hcs[q * 4 + l];
#pragma unroll
      for (int j = 0; j < J; j++) {
        const int s = tid + j * NLA_NT;
        if (s >= S) continue;
        T accv = mk<T>(R(0), R(0));
#pragma unroll
        for (int l = 0; l < 4; l++) accv = cmac(accv, hc[l], pd[j][l]);
        for (int k = 1; k < nh; k++) {
          const int h = h0 + k;
          const int p = hitp[h];
#pragma unroll
          for (int l = 0; l < 4; l++)
            accv = cadd(accv, cmul(hcoef[(long long)h * 4 + l], projD[((long long)p * 4 + l) * S + s]));
        }
        T *o = rw + (size_t)q * S + s;
        *o = cadd(*o, scaled ? cmul(scale, accv) : accv);
      }
    }
    fence_proxy_async();
    mbar_arrive(&done[st]);  // the producer writes the rows back and refills the stage
  }
}

template <typename R>
void launch_nl_apply(Ctx &ctx, const Hamiltonian &h, const C2<R> *projD, int S, C2<R> *out, bool scaled, C2<R> scale) {
  const Projectors &P = h.proj;
  if (P.nhitpts == 0) return;
  const C2<R> *hc;
  if constexpr (sizeof(R) == 8) hc = P.d_hcoef;
  else hc = P.d_hcoef32;
  // bulk form: rows of 16-byte multiples (and 16-byte aligned starts), up to 4 states per compute thread
  const size_t row_bytes = size_t(S) * sizeof(C2<R>);
  if (ctx.nl_bulk >= 0 && row_bytes % 16 == 0 && S <= 4 * NLA_NT && reinterpret_cast<uintptr_t>(out) % 16 == 0) {
    // 8 points per batch (measured at 96^3 x 256: 211 us FP32 / 318 us FP64, against 229 / 357 with
    // 16 / 4 points and 466 / 562 with 32 / 16), fewer when a stage would pass 48 KB
    int KB = int(49152 / row_bytes);
    KB = KB < 1 ? 1 : (KB > 8 ? 8 : KB);
    if (ctx.nl_apply_points > 0) KB = ctx.nl_apply_points;
    const size_t smem = size_t(NLA_NS) * KB * row_bytes + NLA_KMAX * 4 * sizeof(C2<R>) + NLA_NS * NLA_KMAX * sizeof(int4) +
                        2 * NLA_NS * sizeof(uint64_t) + 16;
    if (smem <= size_t(ctx.max_smem_optin)) {
      auto kern = S <= 2 * NLA_NT ? nl_apply_bulk_kernel<R, 2> : nl_apply_bulk_kernel<R, 4>;
      ensure_smem_attr(reinterpret_cast<const void *>(kern), smem);
      // CTAs per SM for this kernel and shared-memory size, computed once under a lock
      static std::mutex mtx;
      static const void *occ_kern[2] = {nullptr, nullptr};
      static size_t occ_smem[2] = {0, 0};
      static int occ_per_sm[2] = {1, 1};
      const int slot = S <= 2 * NLA_NT ? 0 : 1;
      int per_sm;
      {
        std::lock_guard<std::mutex> lock(mtx);
        if (occ_kern[slot] != reinterpret_cast<const void *>(kern) || occ_smem[slot] != smem) {
          INQB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_per_sm[slot], kern, NLA_NT + 32, smem));
          occ_kern[slot] = reinterpret_cast<const void *>(kern);
          occ_smem[slot] = smem;
        }
        per_sm = occ_per_sm[slot];
      }
      const long long nbatch = (P.nhitpts + KB - 1) / KB;
      long long grid = (long long)(per_sm < 1 ? 1 : per_sm) * ctx.num_sms;
      if (grid > nbatch) grid = nbatch;
      kern<<<unsigned(grid), NLA_NT + 32, smem, ctx.stream>>>(P.nhitpts, KB, S, P.d_hrec, P.d_hitp, hc, projD, out,
                                                             scaled, scale, ctx.d_err);
      LAUNCHED(ctx);
      return;
    }
  }
  const int chunk = 32 * int(16 / sizeof(R));
  const int nchunks = (S + chunk - 1) / chunk;
  const long long nitems = P.nhitpts * nchunks;
  long long blocks = (nitems + 3) / 4;
  if (blocks > 148LL * 48) blocks = 148LL * 48;
  nl_apply_kernel<R><<<unsigned(blocks), 128, 0, ctx.stream>>>(nitems, nchunks, S, P.d_hrec, P.d_hitp, hc, projD, out,
                                                               scaled, scale);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ bounded-wait self-test
// One thread waits on an mbarrier phase that nothing completes; the wait is bounded by `limit_ns` of
// %globaltimer, after which the context's error flag is raised exactly as by an expired wait of the
// FFT ring, the tensor-core overlap or the bulk-copy nonlocal kernels.
__global__ void wait_timeout_kernel(int *err, long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&bar, 1);
    ptx::mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !ptx::mbar_wait_bounded(&bar, 0, uint64_t(limit_ns))) atomicExch(err, 1);
}

void launch_wait_timeout(Ctx &ctx, long long limit_ns) {
  wait_timeout_kernel<<<1, 32, 0, ctx.stream>>>(ctx.d_err, limit_ns);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ elementwise
template <typename R> __global__ void fill_kernel(C2<R> *p, long long n, R re, R im) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    p[i] = mk<C2<R>>(re, im);
}
template <typename R> void launch_fill(Ctx &ctx, C2<R> *p, long long n, double re, double im) {
  fill_kernel<R><<<grid_for(n, 256), 256, 0, ctx.stream>>>(p, n, R(re), R(im));
  LAUNCHED(ctx);
}

template <typename R> __global__ void axpy_kernel(C2<R> *y, const C2<R> *x, long long n, R re, R im) {
  const C2<R> c = mk<C2<R>>(re, im);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = cadd(y[i], cmul(c, x[i]));
}
template <typename R> void launch_axpy(Ctx &ctx, C2<R> *y, const C2<R> *x, long long n, double re, double im) {
  axpy_kernel<R><<<grid_for(n, 256), 256, 0, ctx.stream>>>(y, x, n, R(re), R(im));
  LAUNCHED(ctx);
}

// y[pt][s] += scale * coef[s] * x[pt][s]   (operations::shift with a per-state factor, shift.hpp:19-31)
template <typename R>
__global__ void shift_vec_kernel(C2<R> *y, const C2<R> *x, int S, long long n, const double *coef, double scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const R c = R(scale * coef[i % S]);
    y[i] = cadd(y[i], cscale(x[i], c));
  }
}
template <typename R>
void launch_shift_vec(Ctx &ctx, C2<R> *y, const C2<R> *x, int S, long long npoints, const double *coef_dev,
                      double scale) {
  shift_vec_kernel<R><<<grid_for(npoints * S, 256), 256, 0, ctx.stream>>>(y, x, S, npoints * S, coef_dev, scale);
  LAUNCHED(ctx);
}

struct Metric {
  int n[3];
  double rlat[3][3];
  double lat[3][3];
};

__device__ __forceinline__ int symi(int i, int n) { return i >= (n + 1) / 2 ? i - n : i; }

__device__ __forceinline__ double lapl_at(const Metric &m, long long pt, double factor, const double *gc, double k2) {
  const int iz = int(pt % m.n[2]);
  const int iy = int((pt / m.n[2]) % m.n[1]);
  const int ix = int(pt / ((long long)m.n[2] * m.n[1]));
  const double tp = 6.283185307179586476925286766559;
  double G0 = tp * symi(ix, m.n[0]), G1 = tp * symi(iy, m.n[1]), G2 = tp * symi(iz, m.n[2]);
  double c0 = (m.rlat[0][0] * G0 + m.rlat[1][0] * G1) + m.rlat[2][0] * G2;
  double c1 = (m.rlat[0][1] * G0 + m.rlat[1][1] * G1) + m.rlat[2][1] * G2;
  double c2 = (m.rlat[0][2] * G0 + m.rlat[1][2] * G1) + m.rlat[2][2] * G2;
  double g2 = c0 * c0 + c1 * c1 + c2 * c2;
  return factor * (-g2 + (gc[0] * G0 + gc[1] * G1 + gc[2] * G2) + k2);
}

static Metric metric_of(const Basis &b) {
  Metric m;
  for (int i = 0; i < 3; i++) {
    m.n[i] = b.n[i];
    for (int j = 0; j < 3; j++) {
      m.rlat[i][j] = b.rlat[i][j];
      m.lat[i][j] = b.lat[i][j];
    }
  }
  return m;
}

struct Vec3 {
  double v[3];
};

template <typename R>
__global__ void laplacian_kernel(Metric m, const C2<R> *in, C2<R> *out, int S, long long n, double factor, Vec3 gc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const R f = R(lapl_at(m, i / S, factor, gc.v, 0.0));
    out[i] = cscale(in[i], f);
  }
}
template <typename R>
void launch_laplacian(Ctx &ctx, const Basis &b, const C2<R> *in, C2<R> *out, int S, double factor, const double gc[3]) {
  Vec3 g{{gc[0], gc[1], gc[2]}};
  laplacian_kernel<R><<<grid_for(b.npoints * S, 256), 256, 0, ctx.stream>>>(metric_of(b), in, out, S, b.npoints * S,
                                                                            factor, g);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ per-state reductions
// Stage 1: block b handles a contiguous point range; thread t owns state s = t (blockDim >= S handled by loop)
// and accumulates over its points in a fixed order: U running sums over the points p = 0 .. U-1 mod U of the
// range (U independent loads of each operand in flight per thread; U = 8 for single precision, whose 8-byte
// elements need twice the loads in flight to cover the same bytes), added pairwise at the end.  Stage 2
// sums the block partials in order.  592 blocks of 256 threads are resident at once (4 per SM).
constexpr int RED_BLOCKS = 592;

// MODE 0: conj(a) b; 1: conj(a) lapl a; 2: |b - e_s a|^2 (the residual norm of energy.hpp:86-89 without
// forming the residual); 3: (|a|^2, Re conj(a) b), the two sums of one eigenvalue in one pass
template <typename R, int MODE>
__device__ __forceinline__ double2 state_term(const C2<R> *__restrict__ a, const C2<R> *__restrict__ b, int S,
                                              long long p, int s, const Metric &m, double factor, const Vec3 &gc,
                                              double k2, double es) {
  const C2<R> x = a[p * S + s];
  if (MODE == 0) {
    const C2<R> y = b[p * S + s];
    return make_double2(double(x.x) * double(y.x) + double(x.y) * double(y.y),
                        double(x.x) * double(y.y) - double(x.y) * double(y.x));
  } else if (MODE == 1) {
    const double f = lapl_at(m, p, factor, gc.v, k2);
    return make_double2(f * (double(x.x) * double(x.x) + double(x.y) * double(x.y)), 0.0);
  } else if (MODE == 2) {
    const C2<R> y = b[p * S + s];
    const double rx = double(y.x) - es * double(x.x), ry = double(y.y) - es * double(x.y);
    return make_double2(rx * rx + ry * ry, 0.0);
  } else {
    const C2<R> y = b[p * S + s];
    return make_double2(double(x.x) * double(x.x) + double(x.y) * double(x.y),
                        double(x.x) * double(y.x) + double(x.y) * double(y.y));
  }
}

template <typename R, int MODE>
__global__ void state_reduce_kernel(const C2<R> *__restrict__ a, const C2<R> *__restrict__ b, int S, long long npoints,
                                    Metric m, double factor, Vec3 gc, double k2, const double2 *__restrict__ ne,
                                    double2 *partial) {
  const long long chunk = (npoints + gridDim.x - 1) / gridDim.x;
  const long long p0 = blockIdx.x * chunk;
  const long long p1 = min(npoints, p0 + chunk);
  constexpr int U = sizeof(R) == 4 ? 8 : 4;
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    // MODE 2: the eigenvalue Re<a|b>/<a|a> from the MODE 3 sums (the same division the host does)
    const double es = MODE == 2 ? ne[s].y / ne[s].x : 0.0;
    double2 acc[U];
#pragma unroll
    for (int u = 0; u < U; u++) acc[u] = make_double2(0.0, 0.0);
    long long p = p0;
    for (; p + U - 1 < p1; p += U) {
#pragma unroll
      for (int u = 0; u < U; u++) {
        const double2 t = state_term<R, MODE>(a, b, S, p + u, s, m, factor, gc, k2, es);
        acc[u].x += t.x;
        acc[u].y += t.y;
      }
    }
#pragma unroll
    for (int u = 0; u < U - 1; u++)
      if (p + u < p1) {
        const double2 t = state_term<R, MODE>(a, b, S, p + u, s, m, factor, gc, k2, es);
        acc[u].x += t.x;
        acc[u].y += t.y;
      }
#pragma unroll
    for (int w = U / 2; w >= 1; w /= 2)
#pragma unroll
      for (int u = 0; u < w; u++) {
        acc[u].x += acc[u + w].x;
        acc[u].y += acc[u + w].y;
      }
    partial[(long long)blockIdx.x * S + s] = acc[0];
  }
}

__global__ void sum_partials_kernel(const double2 *partial, int nblk, int S, double scale, double2 *out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nblk; k++) {
      re += partial[(long long)k * S + s].x;
      im += partial[(long long)k * S + s].y;
    }
    out[s] = make_double2(scale * re, scale * im);
  }
}

template <typename R>
void launch_overlap_diag(Ctx &ctx, const C2<R> *a, const C2<R> *b, int S, long long npoints, double dv, double2 *out) {
  double2 *partial = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * RED_BLOCKS * S));
  Metric m{};
  Vec3 g{{0, 0, 0}};
  state_reduce_kernel<R, 0><<<RED_BLOCKS, 256, 0, ctx.stream>>>(a, b, S, npoints, m, 0.0, g, 0.0, nullptr, partial);
  LAUNCHED(ctx);
  sum_partials_kernel<<<(S + 255) / 256, 256, 0, ctx.stream>>>(partial, RED_BLOCKS, S, dv, out);
  LAUNCHED(ctx);
  dev_free(ctx, partial);
}

// Eigenvalues and residual norms of energy.hpp:80-89 in two passes over a and b = H a:
// ne[s] = dv (<a|a>, Re<a|b>); when res is given, res[s].x = dv sum_p |b - e_s a|^2 with e_s = ne[s].y / ne[s].x
template <typename R>
void launch_eigen_sums(Ctx &ctx, const C2<R> *a, const C2<R> *b, int S, long long npoints, double dv, double2 *ne,
                       double2 *res) {
  double2 *partial = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * RED_BLOCKS * S));
  Metric m{};
  Vec3 g{{0, 0, 0}};
  state_reduce_kernel<R, 3><<<RED_BLOCKS, 256, 0, ctx.stream>>>(a, b, S, npoints, m, 0.0, g, 0.0, nullptr, partial);
  LAUNCHED(ctx);
  sum_partials_kernel<<<(S + 255) / 256, 256, 0, ctx.stream>>>(partial, RED_BLOCKS, S, dv, ne);
  LAUNCHED(ctx);
  if (res) {
    state_reduce_kernel<R, 2><<<RED_BLOCKS, 256, 0, ctx.stream>>>(a, b, S, npoints, m, 0.0, g, 0.0, ne, partial);
    LAUNCHED(ctx);
    sum_partials_kernel<<<(S + 255) / 256, 256, 0, ctx.stream>>>(partial, RED_BLOCKS, S, dv, res);
    LAUNCHED(ctx);
  }
  dev_free(ctx, partial);
}

template <typename R>
void launch_kinetic_ev(Ctx &ctx, const Basis &b, const C2<R> *fphi, int S, double factor, const double gc[3], double k2,
                       double *out_dev) {
  double2 *partial = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * (RED_BLOCKS * S + S)));
  Vec3 g{{gc[0], gc[1], gc[2]}};
  state_reduce_kernel<R, 1><<<RED_BLOCKS, 256, 0, ctx.stream>>>(fphi, fphi, S, b.npoints, metric_of(b), factor, g, k2, nullptr,
                                                                partial);
  LAUNCHED(ctx);
  double2 *sums = partial + RED_BLOCKS * S;
  sum_partials_kernel<<<(S + 255) / 256, 256, 0, ctx.stream>>>(partial, RED_BLOCKS, S, 1.0, sums);
  LAUNCHED(ctx);
  INQB_CUDA(cudaMemcpy2DAsync(out_dev, sizeof(double), sums, sizeof(double2), sizeof(double), S,
                              cudaMemcpyDeviceToDevice, ctx.stream));
  dev_free(ctx, partial);
}

// ------------------------------------------------------------------ overlap (complex GEMM, K = npoints)
// S[i][j] = dv * sum_p conj(a[p][i]) b[p][j].  64x64 output tile per CTA, split-K over point chunks,
// 256 threads with a 4x4 register tile each, two CTAs per SM (128 registers: 24.5 ms against 31.6 ms with
// 130 registers and one CTA per SM, 96^3 x 256 with itself); partial tiles summed in chunk order.
template <typename R>
__global__ void __launch_bounds__(256, 2) overlap_kernel(const C2<R> *__restrict__ a, int Sa, const C2<R> *__restrict__ b,
                                                      int Sb, long long npoints, long long chunk, int sym,
                                                      double2 *partial) {
  constexpr int TB = 64, KT = 16;
  __shared__ double2 As[KT][TB];
  __shared__ double2 Bs[KT][TB];
  // sym: blockIdx.x enumerates the tiles on and above the diagonal, column by column
  int bi = blockIdx.x, bj = blockIdx.y;
  if (sym) {
    bj = 0;
    while ((bj + 1) * (bj + 2) / 2 <= bi) bj++;
    bi -= bj * (bj + 1) / 2;
  }
  const int ti = bi * TB, tj = bj * TB;
  const long long p0 = blockIdx.z * chunk;
  const long long p1 = min(npoints, p0 + chunk);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double2 acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) acc[u][v] = make_double2(0.0, 0.0);
  for (long long k0 = p0; k0 < p1; k0 += KT) {
    for (int e = threadIdx.x; e < KT * TB; e += 256) {
      const int kk = e / TB, c = e % TB;
      const long long p = k0 + kk;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (p < p1) {
        if (ti + c < Sa) {
          C2<R> x = a[p * Sa + ti + c];
          va = make_double2(double(x.x), double(x.y));
        }
        if (tj + c < Sb) {
          C2<R> y = b[p * Sb + tj + c];
          vb = make_double2(double(y.x), double(y.y));
        }
      }
      As[kk][c] = va;
      Bs[kk][c] = vb;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < KT; kk++) {
      double2 av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) av[u] = As[kk][ty + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; v++) bv[v] = Bs[kk][tx + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          acc[u][v].x += av[u].x * bv[v].x + av[u].y * bv[v].y;
          acc[u][v].y += av[u].x * bv[v].y - av[u].y * bv[v].x;
        }
    }
    __syncthreads();
  }
  const long long base = (long long)blockIdx.z * Sa * Sb;
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int i = ti + ty + 16 * u, j = tj + tx + 16 * v;
      if (i < Sa && j < Sb) partial[base + (long long)i * Sb + j] = acc[u][v];
    }
}

// With sym (a set against itself, S x S) only tiles with i/64 <= j/64 were computed: an element below
// them is the conjugate of its mirror, since <a_j|a_i> = conj(<a_i|a_j>).
// The FP64 form of overlap_kernel with its operand tiles double-buffered in shared memory: the next
// 16 points of a and b are copied with cp.async while the current ones are multiplied, so the global
// latency no longer stalls the tile.  Same tiles, order and arithmetic: bitwise the same result.
__global__ void __launch_bounds__(256, 2) overlap64_kernel(const double2 *__restrict__ a, int Sa,
                                                        const double2 *__restrict__ b, int Sb, long long npoints,
                                                        long long chunk, int sym, double2 *partial) {
  constexpr int TB = 64, KT = 16;
  extern __shared__ __align__(16) double2 osm[];  // [2 buffers][a, b][KT][TB]
  int bi = blockIdx.x, bj = blockIdx.y;
  if (sym) {
    bj = 0;
    while ((bj + 1) * (bj + 2) / 2 <= bi) bj++;
    bi -= bj * (bj + 1) / 2;
  }
  const int ti = bi * TB, tj = bj * TB;
  const long long p0 = blockIdx.z * chunk;
  const long long p1 = min(npoints, p0 + chunk);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  auto tile = [&](int buf, int ab) { return osm + (size_t(buf) * 2 + ab) * KT * TB; };
  auto issue = [&](int buf, long long k0) {
    double2 *As = tile(buf, 0), *Bs = tile(buf, 1);
    for (int e = threadIdx.x; e < KT * TB; e += 256) {
      const int kk = e / TB, c = e % TB;
      const long long p = k0 + kk;
      const bool va = p < p1 && ti + c < Sa, vb = p < p1 && tj + c < Sb;
      ptx::cp_async16(As + e, va ? a + p * Sa + ti + c : a, va ? 16u : 0u);
      ptx::cp_async16(Bs + e, vb ? b + p * Sb + tj + c : b, vb ? 16u : 0u);
    }
    ptx::cp_async_commit();
  };
  double2 acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) acc[u][v] = make_double2(0.0, 0.0);
  if (p0 < p1) issue(0, p0);
  int cur = 0;
  for (long long k0 = p0; k0 < p1; k0 += KT, cur ^= 1) {
    if (k0 + KT < p1) {
      issue(cur ^ 1, k0 + KT);  // the other buffer was released by the barrier closing the last step
      ptx::cp_async_wait<1>();
    } else {
      ptx::cp_async_wait<0>();
    }
    __syncthreads();
    const double2 *As = tile(cur, 0), *Bs = tile(cur, 1);
#pragma unroll 4
    for (int kk = 0; kk < KT; kk++) {
      double2 av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) av[u] = As[kk * TB + ty + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; v++) bv[v] = Bs[kk * TB + tx + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          acc[u][v].x += av[u].x * bv[v].x + av[u].y * bv[v].y;
          acc[u][v].y += av[u].x * bv[v].y - av[u].y * bv[v].x;
        }
    }
    __syncthreads();
  }
  const long long base = (long long)blockIdx.z * Sa * Sb;
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int i = ti + ty + 16 * u, j = tj + tx + 16 * v;
      if (i < Sa && j < Sb) partial[base + (long long)i * Sb + j] = acc[u][v];
    }
}

// The same 64 x 64 tiles of a^H b on the FP64 tensor-core path: mma.sync m8n8k4 (DMMA), four per pair
// of complex operand fragments (re.re + im.im into the real part, re.im - im.re into the imaginary).
// 128 threads: each warp owns a 32 x 32 block of the tile, 4 x 4 fragments of 8 x 8, and steps through
// the point chunk four points at a time; operand tiles double-buffered by cp.async as above, rows padded
// to 66 complex numbers so that the fragment loads of a quarter-warp hit distinct banks.
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128) overlap64_mma_kernel(const double2 *__restrict__ a, int Sa,
                                                            const double2 *__restrict__ b, int Sb, long long npoints,
                                                            long long chunk, int sym, double2 *partial) {
  constexpr int TB = 64, KT = 16, LD = TB + 2;
  extern __shared__ __align__(16) double2 osm[];  // [2 buffers][a, b][KT][LD]
  int bi = blockIdx.x, bj = blockIdx.y;
  if (sym) {
    bj = 0;
    while ((bj + 1) * (bj + 2) / 2 <= bi) bj++;
    bi -= bj * (bj + 1) / 2;
  }
  const int ti = bi * TB, tj = bj * TB;
  const long long p0 = blockIdx.z * chunk;
  const long long p1 = min(npoints, p0 + chunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;  // the warp's block of the tile
  auto tile = [&](int buf, int ab) { return osm + (size_t(buf) * 2 + ab) * KT * LD; };
  auto issue = [&](int buf, long long k0) {
    double2 *As = tile(buf, 0), *Bs = tile(buf, 1);
    for (int e = threadIdx.x; e < KT * TB; e += 128) {
      const int kk = e / TB, c = e % TB;
      const long long p = k0 + kk;
      const bool va = p < p1 && ti + c < Sa, vb = p < p1 && tj + c < Sb;
      ptx::cp_async16(As + kk * LD + c, va ? a + p * Sa + ti + c : a, va ? 16u : 0u);
      ptx::cp_async16(Bs + kk * LD + c, vb ? b + p * Sb + tj + c : b, vb ? 16u : 0u);
    }
    ptx::cp_async_commit();
  };
  double cre[4][4][2], cim[4][4][2];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) cre[u][v][0] = cre[u][v][1] = cim[u][v][0] = cim[u][v][1] = 0.0;
  if (p0 < p1) issue(0, p0);
  int cur = 0;
  // fragment coordinates: A (8 x 4, row-major) element (row lane / 4, col lane % 4), B (4 x 8,
  // col-major) element (row lane % 4, col lane / 4); here the row of A and the col of B are states and
  // the k index is the point
  const int fk = lane & 3, fs = lane >> 2;
  for (long long k0 = p0; k0 < p1; k0 += KT, cur ^= 1) {
    if (k0 + KT < p1) {
      issue(cur ^ 1, k0 + KT);
      ptx::cp_async_wait<1>();
    } else {
      ptx::cp_async_wait<0>();
    }
    __syncthreads();
    const double2 *As = tile(cur, 0), *Bs = tile(cur, 1);
#pragma unroll
    for (int ks = 0; ks < KT; ks += 4) {
      double2 af[4], bf[4];
#pragma unroll
      for (int u = 0; u < 4; u++) af[u] = As[(ks + fk) * LD + wm + 8 * u + fs];
#pragma unroll
      for (int v = 0; v < 4; v++) bf[v] = Bs[(ks + fk) * LD + wn + 8 * v + fs];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          dmma_8x8x4(cre[u][v], af[u].x, bf[v].x);
          dmma_8x8x4(cre[u][v], af[u].y, bf[v].y);
          dmma_8x8x4(cim[u][v], af[u].x, bf[v].y);
          dmma_8x8x4(cim[u][v], -af[u].y, bf[v].x);
        }
    }
    __syncthreads();
  }
  // accumulator fragment: element (row lane / 4, col 2 (lane % 4) + {0, 1}) of each 8 x 8 block
  const long long base = (long long)blockIdx.z * Sa * Sb;
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int i = ti + wm + 8 * u + fs, j = tj + wn + 8 * v + 2 * fk + h;
        if (i < Sa && j < Sb) partial[base + (long long)i * Sb + j] = make_double2(cre[u][v][h], cim[u][v][h]);
      }
}

__global__ void sum_tiles_kernel(const double2 *partial, int nz, long long n, int S, int sym, double scale,
                                 double2 *out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    long long src = e;
    bool mirror = false;
    if (sym) {
      const int i = int(e / S), j = int(e % S);
      if (i / 64 > j / 64) {
        src = (long long)j * S + i;
        mirror = true;
      }
    }
    double re = 0.0, im = 0.0;
    for (int z = 0; z < nz; z++) {
      re += partial[z * n + src].x;
      im += partial[z * n + src].y;
    }
    out[e] = make_double2(scale * re, mirror ? -scale * im : scale * im);
  }
}

template <typename R>
void launch_overlap(Ctx &ctx, const C2<R> *a, int Sa, const C2<R> *b, int Sb, long long npoints, double dv,
                    double2 *out) {
  const int gi = (Sa + 63) / 64, gj = (Sb + 63) / 64;
  const int sym = (a == b && Sa == Sb) ? 1 : 0;
  const int tiles = sym ? gi * (gi + 1) / 2 : gi * gj;
  // CTAs in flight: two per SM of the 256-thread SIMT kernel, four of the 128-thread tensor-core one
  const int per_sm = (sizeof(R) == 8 && ctx.fp64_mma) ? 4 : 2;
  int nz = int((long long)per_sm * ctx.device_sms + tiles - 1) / tiles;  // independent of grid_sms
  if (nz < 1) nz = 1;
  if (nz > 256) nz = 256;
  long long chunk = (npoints + nz - 1) / nz;
  chunk = ((chunk + 15) / 16) * 16;
  nz = int((npoints + chunk - 1) / chunk);
  double2 *partial = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * (size_t)nz * Sa * Sb));
  const dim3 grid = sym ? dim3(tiles, 1, nz) : dim3(gi, gj, nz);
  if constexpr (sizeof(R) == 8) {
    if (ctx.fp64_mma) {
      const size_t smem = 2 * 2 * 16 * 66 * sizeof(double2);
      ensure_smem_attr(reinterpret_cast<const void *>(overlap64_mma_kernel), smem);
      overlap64_mma_kernel<<<grid, 128, smem, ctx.stream>>>(a, Sa, b, Sb, npoints, chunk, sym, partial);
    } else {
      const size_t smem = 2 * 2 * 16 * 64 * sizeof(double2);
      ensure_smem_attr(reinterpret_cast<const void *>(overlap64_kernel), smem);
      overlap64_kernel<<<grid, 256, smem, ctx.stream>>>(a, Sa, b, Sb, npoints, chunk, sym, partial);
    }
  } else {
    overlap_kernel<R><<<grid, 256, 0, ctx.stream>>>(a, Sa, b, Sb, npoints, chunk, sym, partial);
  }
  LAUNCHED(ctx);
  const long long n = (long long)Sa * Sb;
  sum_tiles_kernel<<<grid_for(n, 256), 256, 0, ctx.stream>>>(partial, nz, n, Sb, sym, dv, out);
  LAUNCHED(ctx);
  dev_free(ctx, partial);
}

// ------------------------------------------------------------------ rotate: out[p][:] <- alpha in[p][:] R + beta out[p][:]
template <typename R>
__global__ void __launch_bounds__(256) rotate_kernel(const C2<R> *in, int Sin, C2<R> *out, int Sout, long long npoints,
                                                     const double2 *__restrict__ Rm, double2 alpha, double2 beta,
                                                     int scaled, int use_beta) {
  constexpr int ROWS = 8;
  extern __shared__ __align__(16) unsigned char sm[];
  double2 *rows = reinterpret_cast<double2 *>(sm);  // [ROWS][Sin]
  for (long long p0 = (long long)blockIdx.x * ROWS; p0 < npoints; p0 += (long long)gridDim.x * ROWS) {
    const int nr = int(min((long long)ROWS, npoints - p0));
    for (int e = threadIdx.x; e < ROWS * Sin; e += blockDim.x) {
      const int r = e / Sin, k = e % Sin;
      double2 v = make_double2(0.0, 0.0);
      if (r < nr) {
        C2<R> x = in[(p0 + r) * Sin + k];
        v = make_double2(double(x.x), double(x.y));
      }
      rows[e] = v;
    }
    __syncthreads();  // in place (in == out): every row is staged before any is overwritten
    for (int j = threadIdx.x; j < Sout; j += blockDim.x) {
      double2 acc[ROWS];
#pragma unroll
      for (int r = 0; r < ROWS; r++) acc[r] = make_double2(0.0, 0.0);
      for (int k = 0; k < Sin; k++) {
        const double2 rk = Rm[(long long)k * Sout + j];
#pragma unroll
        for (int r = 0; r < ROWS; r++) {
          const double2 x = rows[r * Sin + k];
          acc[r].x += x.x * rk.x - x.y * rk.y;
          acc[r].y += x.x * rk.y + x.y * rk.x;
        }
      }
#pragma unroll
      for (int r = 0; r < ROWS; r++) {  // constant trip count: acc stays in registers
        if (r >= nr) break;
        double2 v = acc[r];
        if (scaled) v = make_double2(alpha.x * v.x - alpha.y * v.y, alpha.x * v.y + alpha.y * v.x);
        C2<R> *o = out + (p0 + r) * Sout + j;
        if (use_beta) {
          const double2 y = make_double2(double(o->x), double(o->y));
          v.x += beta.x * y.x - beta.y * y.y;
          v.y += beta.x * y.y + beta.y * y.x;
        }
        *o = mk<C2<R>>(R(v.x), R(v.y));
      }
    }
    __syncthreads();
  }
}

// Tiled form of the rotation for distinct in and out: CTA = 64 points x 64 output states, 4 x 4 per
// thread, the states k in steps of 16 with both operand tiles (rows of in, rows of Rm) double-buffered
// in shared memory by cp.async.  Each CTA reads Rm's 64 columns once for 64 points (the row form reads
// all of Rm for every 8 points: 116 GB of cache traffic at 96^3 x 256).  Rows of in must be 16-byte
// multiples (an even state count in single precision).
template <typename R>
__global__ void __launch_bounds__(256, 2) rotate_tiled_kernel(const C2<R> *__restrict__ in, int Sin,
                                                           C2<R> *__restrict__ out, int Sout, long long npoints,
                                                           const double2 *__restrict__ Rm, double2 alpha,
                                                           double2 beta, int scaled, int use_beta) {
  using T = C2<R>;
  constexpr int TP = 64, TJ = 64, KT = 16;
  constexpr int EPC = 16 / int(sizeof(T));  // elements of in per 16-byte copy
  extern __shared__ __align__(16) unsigned char rsm[];
  T *Abuf = reinterpret_cast<T *>(rsm);                                   // [2][TP][KT]
  double2 *Bbuf = reinterpret_cast<double2 *>(Abuf + 2 * TP * KT);        // [2][KT][TJ]
  // blockIdx.x enumerates (point tile, output tile) with the output tiles fastest, so the CTAs that
  // read one tile of points run together
  const int njt = (Sout + TJ - 1) / TJ;
  const int j0 = int(blockIdx.x % njt) * TJ;
  const long long p0 = (long long)(blockIdx.x / njt) * TP;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  auto issue = [&](int buf, int k0) {
    T *As = Abuf + buf * TP * KT;
    double2 *Bs = Bbuf + buf * KT * TJ;
    for (int e = threadIdx.x; e < TP * KT / EPC; e += 256) {
      const int r = e / (KT / EPC), kk = (e % (KT / EPC)) * EPC;
      const long long p = p0 + r;
      const bool v = p < npoints && k0 + kk < Sin;
      ptx::cp_async16(As + r * KT + kk, v ? in + p * Sin + k0 + kk : in, v ? 16u : 0u);
    }
    for (int e = threadIdx.x; e < KT * TJ; e += 256) {
      const int kk = e / TJ, c = e % TJ;
      const bool v = k0 + kk < Sin && j0 + c < Sout;
      ptx::cp_async16(Bs + e, v ? Rm + (long long)(k0 + kk) * Sout + j0 + c : Rm, v ? 16u : 0u);
    }
    ptx::cp_async_commit();
  };
  double2 acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) acc[u][v] = make_double2(0.0, 0.0);
  issue(0, 0);
  int cur = 0;
  for (int k0 = 0; k0 < Sin; k0 += KT, cur ^= 1) {
    if (k0 + KT < Sin) {
      issue(cur ^ 1, k0 + KT);  // the other buffer was released by the barrier closing the last step
      ptx::cp_async_wait<1>();
    } else {
      ptx::cp_async_wait<0>();
    }
    __syncthreads();
    const T *As = Abuf + cur * TP * KT;
    const double2 *Bs = Bbuf + cur * KT * TJ;
#pragma unroll 4
    for (int kk = 0; kk < KT; kk++) {
      double2 av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const T x = As[(ty + 16 * u) * KT + kk];
        av[u] = make_double2(double(x.x), double(x.y));
      }
#pragma unroll
      for (int v = 0; v < 4; v++) bv[v] = Bs[kk * TJ + tx + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          acc[u][v].x += av[u].x * bv[v].x - av[u].y * bv[v].y;
          acc[u][v].y += av[u].x * bv[v].y + av[u].y * bv[v].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const long long p = p0 + ty + 16 * u;
      const int j = j0 + tx + 16 * v;
      if (p < npoints && j < Sout) {
        double2 w = acc[u][v];
        if (scaled) w = make_double2(alpha.x * w.x - alpha.y * w.y, alpha.x * w.y + alpha.y * w.x);
        T *o = out + p * Sout + j;
        if (use_beta) {
          const double2 y = make_double2(double(o->x), double(o->y));
          w.x += beta.x * y.x - beta.y * y.y;
          w.y += beta.x * y.y + beta.y * y.x;
        }
        *o = mk<T>(R(w.x), R(w.y));
      }
    }
}

// The tiled rotation on the FP64 tensor-core path (mma.sync m8n8k4, four per pair of complex fragments:
// re.re - im.im into the real part, re.im + im.re into the imaginary): 64 points x 64 output states per
// CTA of 128 threads, each warp a 32 x 32 block of 8 x 8 fragments; operand tiles double-buffered by
// cp.async, rows padded (20 elements of in, 66 of R) so that the fragment loads hit distinct banks.
template <typename R>
__global__ void __launch_bounds__(128) rotate_mma_kernel(const C2<R> *__restrict__ in, int Sin, C2<R> *__restrict__ out,
                                                         int Sout, long long npoints, const double2 *__restrict__ Rm,
                                                         double2 alpha, double2 beta, int scaled, int use_beta) {
  using T = C2<R>;
  constexpr int TP = 64, TJ = 64, KT = 16, LDA = 20, LDB = TJ + 2;
  constexpr int EPC = 16 / int(sizeof(T));  // elements of in per 16-byte copy
  extern __shared__ __align__(16) unsigned char rsm[];
  T *Abuf = reinterpret_cast<T *>(rsm);                                   // [2][TP][LDA]
  double2 *Bbuf = reinterpret_cast<double2 *>(Abuf + 2 * TP * LDA);       // [2][KT][LDB]
  const int njt = (Sout + TJ - 1) / TJ;
  const int j0 = int(blockIdx.x % njt) * TJ;
  const long long p0 = (long long)(blockIdx.x / njt) * TP;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int fk = lane & 3, fs = lane >> 2;
  auto issue = [&](int buf, int k0) {
    T *As = Abuf + buf * TP * LDA;
    double2 *Bs = Bbuf + buf * KT * LDB;
    for (int e = threadIdx.x; e < TP * KT / EPC; e += 128) {
      const int r = e / (KT / EPC), kk = (e % (KT / EPC)) * EPC;
      const long long p = p0 + r;
      const bool v = p < npoints && k0 + kk < Sin;
      ptx::cp_async16(As + r * LDA + kk, v ? in + p * Sin + k0 + kk : in, v ? 16u : 0u);
    }
    for (int e = threadIdx.x; e < KT * TJ; e += 128) {
      const int kk = e / TJ, c = e % TJ;
      const bool v = k0 + kk < Sin && j0 + c < Sout;
      ptx::cp_async16(Bs + kk * LDB + c, v ? Rm + (long long)(k0 + kk) * Sout + j0 + c : Rm, v ? 16u : 0u);
    }
    ptx::cp_async_commit();
  };
  double cre[4][4][2], cim[4][4][2];
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) cre[u][v][0] = cre[u][v][1] = cim[u][v][0] = cim[u][v][1] = 0.0;
  issue(0, 0);
  int cur = 0;
  for (int k0 = 0; k0 < Sin; k0 += KT, cur ^= 1) {
    if (k0 + KT < Sin) {
      issue(cur ^ 1, k0 + KT);
      ptx::cp_async_wait<1>();
    } else {
      ptx::cp_async_wait<0>();
    }
    __syncthreads();
    const T *As = Abuf + cur * TP * LDA;
    const double2 *Bs = Bbuf + cur * KT * LDB;
#pragma unroll
    for (int ks = 0; ks < KT; ks += 4) {
      double2 af[4], bf[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const T x = As[(wm + 8 * u + fs) * LDA + ks + fk];  // A (8 x 4, row-major): (point, input state)
        af[u] = make_double2(double(x.x), double(x.y));
      }
#pragma unroll
      for (int v = 0; v < 4; v++) bf[v] = Bs[(ks + fk) * LDB + wn + 8 * v + fs];  // B (4 x 8): (input, output)
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) {
          dmma_8x8x4(cre[u][v], af[u].x, bf[v].x);
          dmma_8x8x4(cre[u][v], -af[u].y, bf[v].y);
          dmma_8x8x4(cim[u][v], af[u].x, bf[v].y);
          dmma_8x8x4(cim[u][v], af[u].y, bf[v].x);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const long long p = p0 + wm + 8 * u + fs;
        const int j = j0 + wn + 8 * v + 2 * fk + h;
        if (p < npoints && j < Sout) {
          double2 w = make_double2(cre[u][v][h], cim[u][v][h]);
          if (scaled) w = make_double2(alpha.x * w.x - alpha.y * w.y, alpha.x * w.y + alpha.y * w.x);
          T *o = out + p * Sout + j;
          if (use_beta) {
            const double2 y = make_double2(double(o->x), double(o->y));
            w.x += beta.x * y.x - beta.y * y.y;
            w.y += beta.x * y.y + beta.y * y.x;
          }
          *o = mk<T>(R(w.x), R(w.y));
        }
      }
}

// out <- alpha (in Rm) + beta out, Rm [Sin][Sout]; in == out (Sin == Sout) rotates in place
template <typename R>
void launch_rotate_to(Ctx &ctx, const C2<R> *in, int Sin, C2<R> *out, int Sout, long long npoints, const double2 *Rdev,
                      double2 alpha, double2 beta) {
  const int scaled = !(alpha.x == 1.0 && alpha.y == 0.0);
  const int use_beta = !(beta.x == 0.0 && beta.y == 0.0);
  const bool aligned = (size_t(Sin) * sizeof(C2<R>)) % 16 == 0 && reinterpret_cast<uintptr_t>(in) % 16 == 0 &&
                       reinterpret_cast<uintptr_t>(Rdev) % 16 == 0;
  if (aligned) {
    // tiled kernel, out of place; in place, chunks of 32768 points go through a scratch block and are
    // copied back (the kernel's CTAs for one tile of points read all of its states)
    const size_t tsmem = 2 * 64 * 16 * sizeof(C2<R>) + 2 * 16 * 64 * sizeof(double2);
    const size_t msmem = 2 * 64 * 20 * sizeof(C2<R>) + 2 * 16 * 66 * sizeof(double2);
    if (ctx.fp64_mma) ensure_smem_attr(reinterpret_cast<const void *>(rotate_mma_kernel<R>), msmem);
    else ensure_smem_attr(reinterpret_cast<const void *>(rotate_tiled_kernel<R>), tsmem);
    auto launch = [&](const C2<R> *src, C2<R> *dst, long long n) {
      const long long nblk = (long long)((Sout + 63) / 64) * ((n + 63) / 64);
      INQB_REQUIRE(nblk < (1LL << 31), INQB_ERR_UNSUPPORTED, "set too large for the rotation grid");
      if (ctx.fp64_mma)
        rotate_mma_kernel<R><<<unsigned(nblk), 128, msmem, ctx.stream>>>(src, Sin, dst, Sout, n, Rdev, alpha, beta,
                                                                         scaled, use_beta);
      else
        rotate_tiled_kernel<R><<<unsigned(nblk), 256, tsmem, ctx.stream>>>(src, Sin, dst, Sout, n, Rdev, alpha, beta,
                                                                          scaled, use_beta);
      LAUNCHED(ctx);
    };
    if (in != out) {
      launch(in, out, npoints);
      return;
    }
    INQB_REQUIRE(Sin == Sout && !use_beta, INQB_ERR_ARG, "an in-place rotation is square and has no beta term");
    constexpr long long CH = 32768;
    const long long ch = npoints < CH ? npoints : CH;
    C2<R> *scratch = static_cast<C2<R> *>(dev_alloc(ctx, sizeof(C2<R>) * size_t(ch) * Sout));
    for (long long c0 = 0; c0 < npoints; c0 += CH) {
      const long long n = npoints - c0 < CH ? npoints - c0 : CH;
      launch(in + c0 * Sin, scratch, n);
      INQB_CUDA(cudaMemcpyAsync(out + c0 * Sout, scratch, sizeof(C2<R>) * size_t(n) * Sout, cudaMemcpyDeviceToDevice,
                                ctx.stream));
    }
    dev_free(ctx, scratch);
    return;
  }
  const size_t smem = sizeof(double2) * 8 * Sin;
  INQB_REQUIRE(smem <= ctx.max_smem_optin, INQB_ERR_UNSUPPORTED, "too many states for rotate");
  ensure_smem_attr(reinterpret_cast<const void *>(rotate_kernel<R>), smem);
  rotate_kernel<R><<<grid_for(npoints, 8, 148LL * 16), 256, smem, ctx.stream>>>(in, Sin, out, Sout, npoints, Rdev, alpha,
                                                                              beta, scaled, use_beta);
  LAUNCHED(ctx);
}

template <typename R> void launch_rotate(Ctx &ctx, C2<R> *phi, int S, long long npoints, const double2 *Rdev) {
  launch_rotate_to<R>(ctx, phi, S, phi, S, npoints, Rdev, make_double2(1.0, 0.0), make_double2(0.0, 0.0));
}

// ------------------------------------------------------------------ density n[p] (+)= sum_s occ_s |phi[p][s]|^2
// one warp per point, lanes stride over states, fixed shuffle tree (density.hpp:24-36)
template <typename R>
__global__ void density_kernel(const C2<R> *__restrict__ phi, int S, long long npoints, const double *__restrict__ occ,
                               double *dens, int accumulate) {
  const int lane = threadIdx.x & 31;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long p = warp; p < npoints; p += nwarps) {
    double acc = 0.0;
    for (int s = lane; s < S; s += 32) {
      C2<R> x = phi[p * S + s];
      acc += occ[s] * (double(x.x) * double(x.x) + double(x.y) * double(x.y));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) dens[p] = accumulate ? dens[p] + acc : acc;
  }
}
template <typename R>
void launch_density(Ctx &ctx, const C2<R> *phi, int S, long long npoints, const double *occ_dev, double *dens,
                    int accumulate) {
  density_kernel<R><<<grid_for(npoints * 32, 256), 256, 0, ctx.stream>>>(phi, S, npoints, occ_dev, dens, accumulate);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ kick: phi *= exp(i E_cov . r_contra)
template <typename R>
__global__ void kick_kernel(Metric m, C2<R> *phi, int S, long long npoints, Vec3 ecov) {
  const long long n = npoints * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long pt = e / S;
    const int iz = int(pt % m.n[2]);
    const int iy = int((pt / m.n[2]) % m.n[1]);
    const int ix = int(pt / ((long long)m.n[2] * m.n[1]));
    // rvector: symmetric index times contravariant spacing 1/n (real_space.hpp:127-130)
    const double r0 = symi(ix, m.n[0]) * (1.0 / m.n[0]);
    const double r1 = symi(iy, m.n[1]) * (1.0 / m.n[1]);
    const double r2 = symi(iz, m.n[2]) * (1.0 / m.n[2]);
    const double arg = ecov.v[0] * r0 + ecov.v[1] * r1 + ecov.v[2] * r2;
    double sn, cs;
    sincos(arg, &sn, &cs);
    C2<R> x = phi[e];
    double re = double(x.x) * cs - double(x.y) * sn;
    double im = double(x.x) * sn + double(x.y) * cs;
    phi[e] = mk<C2<R>>(R(re), R(im));
  }
}
template <typename R> void launch_kick(Ctx &ctx, const Basis &b, C2<R> *phi, int S, const double ecov[3]) {
  Vec3 e{{ecov[0], ecov[1], ecov[2]}};
  kick_kernel<R><<<grid_for(b.npoints * S, 256), 256, 0, ctx.stream>>>(metric_of(b), phi, S, b.npoints, e);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ sum |a - b| (integral_sum_absdiff)
__global__ void absdiff_kernel(const double *a, const double *b, long long n, double *partial) {
  __shared__ double red[256];
  const long long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long long p0 = blockIdx.x * chunk, p1 = min(n, p0 + chunk);
  double acc = 0.0;
  for (long long i = p0 + threadIdx.x; i < p1; i += blockDim.x) acc += fabs(a[i] - b[i]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}
__global__ void absdiff_final_kernel(const double *partial, int nb, double *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nb; i++) s += partial[i];
    *out = s;
  }
}
void launch_absdiff_sum(Ctx &ctx, const double *a, const double *b, long long n, double *out_dev) {
  double *partial = static_cast<double *>(dev_alloc(ctx, sizeof(double) * RED_BLOCKS));
  absdiff_kernel<<<RED_BLOCKS, 256, 0, ctx.stream>>>(a, b, n, partial);
  LAUNCHED(ctx);
  absdiff_final_kernel<<<1, 32, 0, ctx.stream>>>(partial, RED_BLOCKS, out_dev);
  LAUNCHED(ctx);
  dev_free(ctx, partial);
}

// dipole = dV sum_r n(r) r (observables::dipole, dipole.hpp:24-60) of a device density: r from the
// symmetric grid index of each point (cell-centred coordinates), contravariant -> cartesian.  Block b
// sums a contiguous point range, threads strided, then a shared-memory tree; the partials are added in
// block order.
__global__ void dipole_kernel(const double *__restrict__ dens, int nx, int ny, int nz, long long n, Vec3 a0, Vec3 a1,
                              Vec3 a2, double *partial) {
  __shared__ double red[3][256];
  const long long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long long p0 = blockIdx.x * chunk, p1 = min(n, p0 + chunk);
  double acc[3] = {0.0, 0.0, 0.0};
  for (long long p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    const int iz = int(p % nz), iy = int((p / nz) % ny), ix = int(p / ((long long)ny * nz));
    const double c0 = (ix >= (nx + 1) / 2 ? ix - nx : ix) * (1.0 / nx);
    const double c1 = (iy >= (ny + 1) / 2 ? iy - ny : iy) * (1.0 / ny);
    const double c2 = (iz >= (nz + 1) / 2 ? iz - nz : iz) * (1.0 / nz);
    const double d = dens[p];
#pragma unroll
    for (int j = 0; j < 3; j++) acc[j] += ((a0.v[j] * c0 + a1.v[j] * c1) + a2.v[j] * c2) * d;
  }
  for (int j = 0; j < 3; j++) red[j][threadIdx.x] = acc[j];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int j = 0; j < 3; j++) red[j][threadIdx.x] += red[j][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) partial[blockIdx.x * 3 + threadIdx.x] = red[threadIdx.x][0];
}
__global__ void dipole_final_kernel(const double *partial, int nb, double scale, double *out) {
  if (blockIdx.x == 0 && threadIdx.x < 3) {
    double s = 0.0;
    for (int i = 0; i < nb; i++) s += partial[i * 3 + threadIdx.x];
    out[threadIdx.x] = scale * s;
  }
}
void launch_dipole(Ctx &ctx, const Basis &b, const double *dens, double *out3_dev) {
  double *partial = static_cast<double *>(dev_alloc(ctx, sizeof(double) * 3 * RED_BLOCKS));
  Vec3 a[3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a[i].v[j] = b.lat[i][j];
  dipole_kernel<<<RED_BLOCKS, 256, 0, ctx.stream>>>(dens, b.n[0], b.n[1], b.n[2], b.npoints, a[0], a[1], a[2], partial);
  LAUNCHED(ctx);
  dipole_final_kernel<<<1, 32, 0, ctx.stream>>>(partial, RED_BLOCKS, b.volume / double(b.npoints), out3_dev);
  LAUNCHED(ctx);
  dev_free(ctx, partial);
}

// ------------------------------------------------------------------ eigensolver pieces
// y[pt][s] += scale * (coef[s] * x[pt][s]) with complex per-state factors (operations::shift, shift.hpp:19-31)
template <typename R>
__global__ void shift_cvec_kernel(C2<R> *__restrict__ y, const C2<R> *__restrict__ x, int S, long long n,
                                  const double2 *__restrict__ coef, double scale) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double2 c = coef[i % S];
    const C2<R> xv = x[i];
    const double tr = c.x * double(xv.x) - c.y * double(xv.y), ti = c.x * double(xv.y) + c.y * double(xv.x);
    y[i] = mk<C2<R>>(R(double(y[i].x) + scale * tr), R(double(y[i].y) + scale * ti));
  }
}
template <typename R>
void launch_shift_cvec(Ctx &ctx, C2<R> *y, const C2<R> *x, int S, long long npoints, const double2 *coef_dev,
                       double scale) {
  shift_cvec_kernel<R><<<grid_for(npoints * S, 256), 256, 0, ctx.stream>>>(y, x, S, npoints * S, coef_dev, scale);
  LAUNCHED(ctx);
}

// Teter-Payne-Allan preconditioner on a Fourier-space set (preconditioner.hpp:24-46):
// x[G][s] *= K(0.5 |G|^2 / kin[s]), K(t) = (((8t + 12)t + 18)t + 27) / ((((16t + 8)t + 12)t + 18)t + 27)
template <typename R>
__global__ void tpa_precondition_kernel(Metric m, C2<R> *__restrict__ x, int S, long long n,
                                        const double *__restrict__ kin) {
  const double zero[3] = {0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double lapl = -0.5 * lapl_at(m, i / S, 1.0, zero, 0.0);  // -0.5 * (-|G|^2)
    const double t = lapl / kin[i % S];
    const double num = ((8.0 * t + 12.0) * t + 18.0) * t + 27.0;
    const double den = (((16.0 * t + 8.0) * t + 12.0) * t + 18.0) * t + 27.0;
    const double k = num / den;
    x[i] = mk<C2<R>>(R(double(x[i].x) * k), R(double(x[i].y) * k));
  }
}
template <typename R> void launch_tpa_precondition(Ctx &ctx, const Basis &b, C2<R> *x, int S, const double *kin_dev) {
  tpa_precondition_kernel<R><<<grid_for(b.npoints * S, 256), 256, 0, ctx.stream>>>(metric_of(b), x, S,
                                                                                   b.npoints * S, kin_dev);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ restart files
// out[k][pt] = (complex<double>) in[pt][s0 + k], k < ns: states [s0, s0 + ns) as contiguous rows
template <typename R>
__global__ void extract_states_kernel(const C2<R> *__restrict__ in, int S, long long np, int s0, int ns,
                                      double2 *__restrict__ out) {
  const long long n = np * ns;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / np, pt = i % np;
    const C2<R> v = in[pt * S + s0 + k];
    out[i] = make_double2(double(v.x), double(v.y));
  }
}
// the reverse: out[pt][s0 + k] = in[k][pt]
template <typename R>
__global__ void insert_states_kernel(const double2 *__restrict__ in, int S, long long np, int s0, int ns,
                                     C2<R> *__restrict__ out) {
  const long long n = np * ns;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / np, pt = i % np;
    const double2 v = in[i];
    out[pt * S + s0 + k] = mk<C2<R>>(R(v.x), R(v.y));
  }
}
template <typename R>
void launch_extract_states(Ctx &ctx, const C2<R> *in, int S, long long np, int s0, int ns, double2 *out) {
  extract_states_kernel<R><<<grid_for(np * ns, 256), 256, 0, ctx.stream>>>(in, S, np, s0, ns, out);
  LAUNCHED(ctx);
}
template <typename R>
void launch_insert_states(Ctx &ctx, const double2 *in, int S, long long np, int s0, int ns, C2<R> *out) {
  insert_states_kernel<R><<<grid_for(np * ns, 256), 256, 0, ctx.stream>>>(in, S, np, s0, ns, out);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ interacting potential
// (solvers/poisson.hpp, hamiltonian/xc_term.hpp, hamiltonian/self_consistency.hpp)

__global__ void real_to_complex_kernel(const double *__restrict__ in, double2 *__restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = make_double2(in[i], 0.0);
}

// poisson_apply_kernel with poisson_kernel_3d (poisson.hpp:29-35, 72-87): times scal * kern,
// scal = -4 pi / N, kern = -1/|G|^2 (cartesian), 0 for |G|^2 < 1e-6
__global__ void poisson_factor_kernel(Metric m, double2 *__restrict__ f, long long n, double scal) {
  const double zero[3] = {0.0, 0.0, 0.0};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double g2 = lapl_at(m, i, -1.0, zero, 0.0);
    const double k = g2 < 1e-6 ? 0.0 : -1.0 / g2;
    const double c = scal * k;
    f[i] = make_double2(f[i].x * c, f[i].y * c);
  }
}

// Slater exchange and Perdew-Zunger 1981 correlation of an unpolarised density (the published
// parametrisation, libxc's XC_LDA_X and XC_LDA_C_PZ): energy per particle and potential.
__device__ __forceinline__ void lda_xc(double n, double &eps, double &v) {
  if (!(n > 1e-15)) {
    eps = 0.0;
    v = 0.0;
    return;
  }
  const double pi = 3.14159265358979323846;
  const double cx = -0.75 * cbrt(3.0 / pi);
  const double ex = cx * cbrt(n);
  const double rs = cbrt(3.0 / (4.0 * pi * n));
  double ec, vc;
  if (rs >= 1.0) {
    const double sq = sqrt(rs);
    const double den = 1.0 + 1.0529 * sq + 0.3334 * rs;
    ec = -0.1423 / den;
    vc = ec * (1.0 + 7.0 / 6.0 * 1.0529 * sq + 4.0 / 3.0 * 0.3334 * rs) / den;
  } else {
    const double lr = log(rs);
    ec = 0.0311 * lr - 0.048 + 0.0020 * rs * lr - 0.0116 * rs;
    vc = 0.0311 * lr + (-0.048 - 0.0311 / 3.0) + 2.0 / 3.0 * 0.0020 * rs * lr + (2.0 * -0.0116 - 0.0020) / 3.0 * rs;
  }
  eps = ex + ec;
  v = 4.0 / 3.0 * ex + vc;
}

// V = V_ion + Re V_H + V_xc (double and single copies) and the block sums, in a fixed order, of
// n V_ion, n V_H, n eps_xc, n v_xc
__global__ void ks_potential_kernel(const double *__restrict__ n, const double *__restrict__ vion,
                                    const double2 *__restrict__ vh, int xc, long long np, double *__restrict__ V,
                                    float *__restrict__ V32, double *__restrict__ partial) {
  __shared__ double red[4][256];
  const long long chunk = (np + gridDim.x - 1) / gridDim.x;
  const long long p0 = blockIdx.x * chunk, p1 = min(np, p0 + chunk);
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
    const double d = n[i];
    const double h = vh ? vh[i].x : 0.0;
    double eps = 0.0, vx = 0.0;
    if (xc) lda_xc(d, eps, vx);
    const double v = (vion[i] + h) + vx;
    V[i] = v;
    V32[i] = float(v);
    s[0] += d * vion[i];
    s[1] += d * h;
    s[2] += d * eps;
    s[3] += d * vx;
  }
  for (int k = 0; k < 4; k++) red[k][threadIdx.x] = s[k];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; k++) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) partial[blockIdx.x * 4 + k] = red[k][0];
}

void launch_real_to_complex(Ctx &ctx, const double *in, double2 *out, long long n) {
  real_to_complex_kernel<<<grid_for(n, 256), 256, 0, ctx.stream>>>(in, out, n);
  LAUNCHED(ctx);
}

void launch_poisson_factor(Ctx &ctx, const Basis &b, double2 *f) {
  poisson_factor_kernel<<<grid_for(b.npoints, 256), 256, 0, ctx.stream>>>(metric_of(b), f, b.npoints,
                                                                         -4.0 * 3.14159265358979323846 / double(b.npoints));
  LAUNCHED(ctx);
}

void launch_ks_potential(Ctx &ctx, const double *n, const double *vion, const double2 *vh, int xc, long long np,
                         double *V, float *V32, double *partial_dev) {
  ks_potential_kernel<<<KS_BLOCKS, 256, 0, ctx.stream>>>(n, vion, vh, xc, np, V, V32, partial_dev);
  LAUNCHED(ctx);
}

// ------------------------------------------------------------------ instantiations
// ------------------------------------------------------------------ Taylor terms combined

struct TaylorCoefs {
  double2 c1[8], c2[8];
};
struct TaylorTerms {
  const void *u[8];
};

// e1 = x + sum_n c1[n] u[n], e2 = x + sum_n c2[n] u[n], element-wise, terms added in order n = 0, 1, ...
// (the order in which exponential.hpp:56-69 adds them); complex products in double
template <typename R>
__global__ void taylor_combine_kernel(const C2<R> *__restrict__ x, TaylorTerms u, int nterms, TaylorCoefs c,
                                      C2<R> *e1, C2<R> *e2, long long n) {
  using T = C2<R>;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const T xv = x[i];
    double2 a1 = make_double2(double(xv.x), double(xv.y)), a2 = a1;
    for (int k = 0; k < nterms; k++) {
      const T t = static_cast<const T *>(u.u[k])[i];
      const double2 tv = make_double2(double(t.x), double(t.y));
      if (e1) a1 = cadd(a1, cmul(c.c1[k], tv));
      a2 = cadd(a2, cmul(c.c2[k], tv));
    }
    if (e1) e1[i] = mk<T>(R(a1.x), R(a1.y));
    e2[i] = mk<T>(R(a2.x), R(a2.y));
  }
}

template <typename R>
void launch_taylor_combine(Ctx &ctx, const C2<R> *x, const C2<R> *const *u, int nterms, const double2 *c1,
                           const double2 *c2, C2<R> *e1, C2<R> *e2, long long n) {
  INQB_REQUIRE(nterms >= 1 && nterms <= 8, INQB_ERR_UNSUPPORTED, "Taylor order must be 1..8");
  TaylorTerms t{};
  TaylorCoefs c{};
  for (int k = 0; k < nterms; k++) {
    t.u[k] = u[k];
    c.c1[k] = c1 ? c1[k] : make_double2(0.0, 0.0);
    c.c2[k] = c2[k];
  }
  long long blocks = (n + 255) / 256;
  if (blocks > 16LL * ctx.num_sms) blocks = 16LL * ctx.num_sms;
  taylor_combine_kernel<R><<<unsigned(blocks), 256, 0, ctx.stream>>>(x, t, nterms, c, e1, e2, n);
  LAUNCHED(ctx);
}

#define INST(R)                                                                                                   \
  template void launch_nl_project<R>(Ctx &, const Basis &, const Hamiltonian &, const C2<R> *, int, C2<R> *,       \
                                     C2<R> *);                                                                    \
  template void launch_nl_scatter<R>(Ctx &, const Basis &, const Hamiltonian &, const C2<R> *, int, C2<R> *);     \
  template void launch_nl_apply<R>(Ctx &, const Hamiltonian &, const C2<R> *, int, C2<R> *, bool, C2<R>);        \
  template void launch_taylor_combine<R>(Ctx &, const C2<R> *, const C2<R> *const *, int, const double2 *,         \
                                         const double2 *, C2<R> *, C2<R> *, long long);                           \
  template void launch_fill<R>(Ctx &, C2<R> *, long long, double, double);                                         \
  template void launch_axpy<R>(Ctx &, C2<R> *, const C2<R> *, long long, double, double);                          \
  template void launch_shift_vec<R>(Ctx &, C2<R> *, const C2<R> *, int, long long, const double *, double);        \
  template void launch_shift_cvec<R>(Ctx &, C2<R> *, const C2<R> *, int, long long, const double2 *, double);      \
  template void launch_extract_states<R>(Ctx &, const C2<R> *, int, long long, int, int, double2 *);               \
  template void launch_insert_states<R>(Ctx &, const double2 *, int, long long, int, int, C2<R> *);                \
  template void launch_tpa_precondition<R>(Ctx &, const Basis &, C2<R> *, int, const double *);                    \
  template void launch_laplacian<R>(Ctx &, const Basis &, const C2<R> *, C2<R> *, int, double, const double *);    \
  template void launch_overlap_diag<R>(Ctx &, const C2<R> *, const C2<R> *, int, long long, double, double2 *);    \
  template void launch_eigen_sums<R>(Ctx &, const C2<R> *, const C2<R> *, int, long long, double, double2 *,      \
                                     double2 *);                                                                   \
  template void launch_kinetic_ev<R>(Ctx &, const Basis &, const C2<R> *, int, double, const double *, double,     \
                                     double *);                                                                   \
  template void launch_overlap<R>(Ctx &, const C2<R> *, int, const C2<R> *, int, long long, double, double2 *);   \
  template void launch_rotate<R>(Ctx &, C2<R> *, int, long long, const double2 *);                                 \
  template void launch_rotate_to<R>(Ctx &, const C2<R> *, int, C2<R> *, int, long long, const double2 *, double2,     \
                                    double2);                                                                      \
  template void launch_density<R>(Ctx &, const C2<R> *, int, long long, const double *, double *, int);            \
  template void launch_kick<R>(Ctx &, const Basis &, C2<R> *, int, const double *);

INST(double)
INST(float)

}  // namespace inqb

namespace inqb {

// ------------------------------------------------------------------ synthetic orbitals
// SplitMix64 (Steele, Lea & Flood 2014) counter stream and the Box-Muller transform.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long seed, unsigned long long counter) {
  unsigned long long z = seed + (counter + 1ULL) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double u01(unsigned long long x) { return double(x >> 11) * (1.0 / 9007199254740992.0); }

template <typename R>
__global__ void randomize_gsphere_kernel(Metric m, C2<R> *phi, int S, long long npoints, unsigned long long seed,
                                         double ecut) {
  const long long n = npoints * S;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const long long pt = e / S;
    const int s = int(e % S);
    const double half_g2 = -0.5 * lapl_at(m, pt, 1.0, Vec3{{0, 0, 0}}.v, 0.0);
    C2<R> v = mk<C2<R>>(R(0), R(0));
    if (half_g2 < ecut) {
      const unsigned long long c = (unsigned long long)s * (unsigned long long)npoints + (unsigned long long)pt;
      const double a = u01(splitmix64(seed, 2 * c)), b = u01(splitmix64(seed, 2 * c + 1));
      const double r = sqrt(-2.0 * log(1.0 - a));
      double sn, cs;
      sincospi(2.0 * b, &sn, &cs);
      v = mk<C2<R>>(R(r * cs), R(r * sn));
    }
    phi[e] = v;
  }
}

template <typename R>
void launch_randomize_gsphere(Ctx &ctx, const Basis &b, C2<R> *phi, int S, unsigned long long seed, double ecut) {
  randomize_gsphere_kernel<R><<<grid_for(b.npoints * S, 256), 256, 0, ctx.stream>>>(metric_of(b), phi, S, b.npoints,
                                                                                     seed, ecut);
  LAUNCHED(ctx);
}

template <typename RI, typename RO> __global__ void convert_kernel(const C2<RI> *in, C2<RO> *out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    C2<RI> x = in[i];
    out[i] = mk<C2<RO>>(RO(x.x), RO(x.y));
  }
}

void launch_convert(Ctx &ctx, const void *in, int in_prec, void *out, int out_prec, long long n) {
  if (in_prec == INQB_F64 && out_prec == INQB_F32)
    convert_kernel<double, float><<<grid_for(n, 256), 256, 0, ctx.stream>>>(static_cast<const double2 *>(in),
                                                                            static_cast<float2 *>(out), n);
  else if (in_prec == INQB_F32 && out_prec == INQB_F64)
    convert_kernel<float, double><<<grid_for(n, 256), 256, 0, ctx.stream>>>(static_cast<const float2 *>(in),
                                                                            static_cast<double2 *>(out), n);
  else
    throw Error(INQB_ERR_ARG, "conversion needs two different precisions");
  LAUNCHED(ctx);
}

template void launch_randomize_gsphere<double>(Ctx &, const Basis &, double2 *, int, unsigned long long, double);
template void launch_randomize_gsphere<float>(Ctx &, const Basis &, float2 *, int, unsigned long long, double);

}  // namespace inqb
