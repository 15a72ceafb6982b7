// Persistent, TMA-pipelined batched FFT pass for compile-time line lengths.
//
// Same tile as fft.cu -- one grid line of N points times W consecutive states,
// 256-byte rows -- but:
//   * tiles stream through an NS-stage shared-memory ring: one elected thread
//     issues cp.async.bulk.tensor (TMA) loads NS tiles ahead and a TMA store per
//     finished tile, so HBM traffic overlaps the arithmetic of the other stages;
//   * the line DFT is a two-level Cooley-Tukey N = N1 x N2 done in registers
//     (N1- and N2-point codelets, composite ones from radix 2,3,4,5,8 with
//     twiddles from a shared-memory copy of the line's table), with one
//     shared-memory exchange instead of one per radix;
//   * all index arithmetic is compile-time except the per-tile line decomposition.
// Every mbarrier wait is bounded (about 2 s by %globaltimer); on expiry the CTA
// raises the context's error flag and leaves its tile loop.

#pragma once

#include <cuda.h>

#include "fft_common.cuh"
#include "ptx.cuh"

namespace inqb {
namespace v2 {

enum Variant {
  FWD_STORE = 0, INV_STORE = 1, MID_KIN = 2, INV_FINAL = 3, FWD_VPSI = 4, FWD_LAPLADD = 5,
  // the same passes with the frequencies along the pass axis in digit-reversed order (position
  // k2 + N2 k1 holds frequency k1 + N1 k2): forward output, inverse input
  FWD_PERM = 6, INV_PERM = 7, INV_FINAL_PERM = 8
};

constexpr int base_var(int v) { return v == FWD_PERM ? FWD_STORE : (v == INV_PERM ? INV_STORE : (v == INV_FINAL_PERM ? INV_FINAL : v)); }
constexpr bool is_perm(int v) { return v >= FWD_PERM; }
constexpr bool has_aux(int v) { return base_var(v) == INV_FINAL || v == FWD_LAPLADD; }

template <int N> struct Split { static constexpr int N1 = 0, N2 = 0; };
template <> struct Split<24> { static constexpr int N1 = 8, N2 = 3; };
template <> struct Split<32> { static constexpr int N1 = 8, N2 = 4; };
template <> struct Split<40> { static constexpr int N1 = 8, N2 = 5; };
template <> struct Split<48> { static constexpr int N1 = 8, N2 = 6; };
template <> struct Split<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct Split<72> { static constexpr int N1 = 8, N2 = 9; };
template <> struct Split<96> { static constexpr int N1 = 8, N2 = 12; };
template <> struct Split<120> { static constexpr int N1 = 8, N2 = 15; };
template <> struct Split<128> { static constexpr int N1 = 8, N2 = 16; };

constexpr int first_factor(int M) {
  const int f[6] = {8, 4, 2, 3, 5, 7};
  for (int i = 0; i < 6; i++)
    if (M % f[i] == 0 && M != f[i]) return f[i];
  return M;
}

// ------------------------------------------------------------------ PTX helpers

using ptx::global_ns;
using ptx::mbar_init;
using ptx::mbar_init_fence;
using ptx::mbar_try_wait;
using ptx::smem_u32;
using ptx::mbar_expect_tx;
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, const void *src, int c0, int c1, int c2, int c3) {
  asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
               : "memory");
}
using ptx::bulk_commit;
using ptx::bulk_wait0;
using ptx::bulk_wait_read0;
using ptx::fence_proxy_async;

// ------------------------------------------------------------------ register codelets (compile-time size)

template <int DIR, typename T> __device__ __forceinline__ T mmi(T a) {  // a * (-i * DIR)
  if constexpr (DIR > 0) return mk<T>(a.y, -a.x);
  else return mk<T>(-a.y, a.x);
}
template <int DIR, typename T> __device__ __forceinline__ T twid(T t) {
  if constexpr (DIR < 0) t.y = -t.y;
  return t;
}

// cos(2 pi m / r) and sin(2 pi m / r), m = 1..(r-1)/2, for the odd prime codelets
// Single-precision products by a constant or a twiddle factor.  The float roundings of sqrt(1/2),
// sin(pi/3) and of many table twiddles fall on the same side often enough to shrink every transform
// by ~2e-8 (an energy bias that reaches ~1e-6 Ha in <psi|H|psi>).  With c = c_hi + c_lo (c_lo the
// float rounding remainder), fma(x, c_hi, x * c_lo) leaves only an unbiased rounding; double products
// need no correction.
template <typename T> __device__ __forceinline__ T kscale(T a, double c) {
  using R = decltype(T::x);
  if constexpr (sizeof(R) == 4) {
    const float hi = float(c), lo = float(c - double(float(c)));
    if (lo == 0.0f) return mk<T>(a.x * hi, a.y * hi);
    return mk<T>(__fmaf_rn(a.x, hi, a.x * lo), __fmaf_rn(a.y, hi, a.y * lo));
  } else {
    return mk<T>(a.x * R(c), a.y * R(c));
  }
}
// a times twiddle `idx` of the line table; single-precision tables interleave each twiddle's float
// part and float remainder (one 16-byte load).
template <int DIR, int N, typename T> __device__ __forceinline__ T twmul(T a, const T *__restrict__ tw, int idx) {
  using R = decltype(T::x);
  if constexpr (sizeof(R) == 4) {
    const float4 q = reinterpret_cast<const float4 *>(tw)[idx];
    const T h = twid<DIR>(mk<T>(q.x, q.y)), l = twid<DIR>(mk<T>(q.z, q.w));
    const R lr = __fmaf_rn(-a.y, l.y, a.x * l.x), li = __fmaf_rn(a.y, l.x, a.x * l.y);
    return mk<T>(__fmaf_rn(a.x, h.x, __fmaf_rn(-a.y, h.y, lr)), __fmaf_rn(a.x, h.y, __fmaf_rn(a.y, h.x, li)));
  } else {
    return cmul(a, twid<DIR>(tw[idx]));
  }
}
// entries of the line's twiddle table in shared memory: N, or 2N for single precision
template <typename R> constexpr int tw_entries(int N) { return sizeof(R) == 4 ? 2 * N : N; }

template <int RR> __host__ __device__ constexpr double odd_cos(int m) {
  if (RR == 3) return -0.5;
  if (RR == 5) return m == 1 ? 0.30901699437494742410229341718281905886 : -0.80901699437494742410229341718281905886;
  return m == 1 ? 0.62348980185873353052500488400423981063
                : (m == 2 ? -0.22252093395631440428890256449679475947 : -0.90096886790241912623610231950744505117);
}
template <int RR> __host__ __device__ constexpr double odd_sin(int m) {
  if (RR == 3) return 0.86602540378443864676372317075293618347;
  if (RR == 5) return m == 1 ? 0.95105651629515357211643933337938214341 : 0.58778525229247312916870595463907276860;
  return m == 1 ? 0.78183148246802980870844452667405775023
                : (m == 2 ? 0.97492791218182360701813168299393121723 : 0.43388373911755812047576833284835875461);
}

// cos and sin of 2 pi p / q, evaluated at compile time: the angle is folded into [0, pi/4] by exact
// integer reflections, multiples of 30 and 45 degrees take exact values, the rest a Taylor series
// (x <= pi/4, terms to x^27).
struct CosSin {
  double c, s;
};
__host__ __device__ constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int n = 1; n < 14; n++) {
    term = -term * x * x / double((2 * n) * (2 * n + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; n++) {
    term = -term * x * x / double((2 * n - 1) * (2 * n));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr CosSin cos_sin_turn(long long p, long long q) {
  p %= q;
  if (p < 0) p += q;
  bool neg_s = false, neg_c = false, swap = false;
  if (2 * p > q) { p = q - p; neg_s = true; }              // 2 pi - theta
  if (4 * p > q) { p = q - 2 * p; q = 2 * q; neg_c = true; }  // pi - theta
  if (8 * p > q) { p = q - 4 * p; q = 4 * q; swap = true; }   // pi / 2 - theta
  double c = taylor_cos(6.283185307179586476925286766559 * double(p) / double(q));
  double s = taylor_sin(6.283185307179586476925286766559 * double(p) / double(q));
  if (p == 0) { c = 1.0; s = 0.0; }
  if (8 * p == q) c = s = 0.70710678118654752440084436210484903928;
  if (12 * p == q) { c = 0.86602540378443864676372317075293618347; s = 0.5; }
  if (swap) { const double t = c; c = s; s = t; }
  if (neg_c) c = -c;
  if (neg_s) s = -s;
  return CosSin{c, s};
}

// a times the compile-time twiddle W_M^TT = exp(-2 pi i TT DIR / M).  Single precision: the same
// compensated product as twmul (twiddle = float part + float remainder), with the terms of exact
// parts dropped; unit twiddles are sign changes and swaps.
template <int DIR, int M, int TT, typename T> __device__ __forceinline__ T tw_const(T a) {
  using R = decltype(T::x);
  constexpr CosSin cs = cos_sin_turn(TT, M);
  constexpr double tx = cs.c, ty = -double(DIR) * cs.s;
  if constexpr (ty == 0.0) {
    if constexpr (tx > 0.0) return a;
    else return mk<T>(-a.x, -a.y);
  } else if constexpr (tx == 0.0) {
    if constexpr (ty > 0.0) return mk<T>(-a.y, a.x);
    else return mk<T>(a.y, -a.x);
  } else if constexpr (sizeof(R) == 4) {
    constexpr float hx = float(tx), hy = float(ty);
    constexpr float lx = float(tx - double(hx)), ly = float(ty - double(hy));
    R lr, li;
    if constexpr (lx == 0.0f && ly == 0.0f) {
      lr = R(0);
      li = R(0);
      return mk<T>(__fmaf_rn(a.x, hx, -a.y * hy), __fmaf_rn(a.x, hy, a.y * hx));
    } else if constexpr (ly == 0.0f) {
      lr = a.x * lx;
      li = a.y * lx;
    } else if constexpr (lx == 0.0f) {
      lr = -a.y * ly;
      li = a.x * ly;
    } else {
      lr = __fmaf_rn(-a.y, ly, a.x * lx);
      li = __fmaf_rn(a.y, lx, a.x * ly);
    }
    return mk<T>(__fmaf_rn(a.x, hx, __fmaf_rn(-a.y, hy, lr)), __fmaf_rn(a.x, hy, __fmaf_rn(a.y, hx, li)));
  } else {
    return mk<T>(a.x * R(tx) - a.y * R(ty), a.x * R(ty) + a.y * R(tx));
  }
}
// tw_const with the exponent known only after unrolling (folds to one product once t is constant)
template <int DIR, int M, int TT = 1, typename T> __device__ __forceinline__ T tw_const_at(T a, int t) {
  if constexpr (TT >= M) return a;
  else return t == TT ? tw_const<DIR, M, TT>(a) : tw_const_at<DIR, M, TT + 1>(a, t);
}

// M-point DFT in registers.  Composite sizes take their inner twiddles as compile-time constants, or
// from the line's table when TABLE is set (the faster choice measured for the single-precision
// forward streaming passes; the constants win everywhere else).
template <int M, int DIR, int N, bool TABLE = false, typename T>
__device__ __forceinline__ void dft(T (&v)[M], const T *__restrict__ tw) {
  using R = decltype(T::x);
  if constexpr (M == 1) {
  } else if constexpr (M == 2) {
    T a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if constexpr (M == 4) {
    T t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    T t2 = cadd(v[1], v[3]), t3 = mmi<DIR>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  } else if constexpr (M == 8) {
    constexpr double h = 0.70710678118654752440084436210484903928;
    T e[4] = {v[0], v[2], v[4], v[6]};
    T o[4] = {v[1], v[3], v[5], v[7]};
    dft<4, DIR, N>(e, tw);
    dft<4, DIR, N>(o, tw);
    T w1, w3;
    if constexpr (DIR > 0) {
      w1 = kscale(mk<T>(o[1].x + o[1].y, o[1].y - o[1].x), h);
      w3 = kscale(mk<T>(o[3].y - o[3].x, -o[3].x - o[3].y), h);
    } else {
      w1 = kscale(mk<T>(o[1].x - o[1].y, o[1].y + o[1].x), h);
      w3 = kscale(mk<T>(-o[3].x - o[3].y, o[3].x - o[3].y), h);
    }
    T w2 = mmi<DIR>(o[2]);
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], w1);
    v[5] = csub(e[1], w1);
    v[2] = cadd(e[2], w2);
    v[6] = csub(e[2], w2);
    v[3] = cadd(e[3], w3);
    v[7] = csub(e[3], w3);
  } else if constexpr (M == 3 || M == 5 || M == 7) {
    constexpr int H = (M - 1) / 2;
    T a[H], b[H];
#pragma unroll
    for (int m = 1; m <= H; m++) {
      a[m - 1] = cadd(v[m], v[M - m]);
      b[m - 1] = csub(v[m], v[M - m]);
    }
    const T x0 = v[0];
    T s = x0;
#pragma unroll
    for (int m = 0; m < H; m++) s = cadd(s, a[m]);
    T y[M];
    y[0] = s;
#pragma unroll
    for (int k = 1; k <= H; k++) {
      T re = x0, im = mk<T>(R(0), R(0));
#pragma unroll
      for (int m = 1; m <= H; m++) {
        const int idx = (m * k) % M;
        const double c = idx <= H ? odd_cos<M>(idx) : odd_cos<M>(M - idx);
        const double sn = idx <= H ? odd_sin<M>(idx) : -odd_sin<M>(M - idx);
        re = cadd(re, kscale(a[m - 1], c));
        im = cadd(im, kscale(b[m - 1], sn));
      }
      const T t = mmi<DIR>(im);
      y[k] = cadd(re, t);
      y[M - k] = csub(re, t);
    }
#pragma unroll
    for (int k = 0; k < M; k++) v[k] = y[k];
  } else {
    // composite: Cooley-Tukey M = A * B, twiddles W_M^t = constants or tw[t * N / M]
    constexpr int A = first_factor(M);
    constexpr int B = M / A;
    T tmp[M];
#pragma unroll
    for (int j2 = 0; j2 < B; j2++) {
      T s[A];
#pragma unroll
      for (int j1 = 0; j1 < A; j1++) s[j1] = v[j2 + B * j1];
      dft<A, DIR, N, TABLE>(s, tw);
#pragma unroll
      for (int k1 = 0; k1 < A; k1++) {
        if (j2 * k1 == 0) tmp[k1 * B + j2] = s[k1];
        else if constexpr (TABLE) tmp[k1 * B + j2] = twmul<DIR, N>(s[k1], tw, (j2 * k1) * (N / M));
        else tmp[k1 * B + j2] = tw_const_at<DIR, M>(s[k1], j2 * k1);
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; k1++) {
      T s[B];
#pragma unroll
      for (int j2 = 0; j2 < B; j2++) s[j2] = tmp[k1 * B + j2];
      dft<B, DIR, N, TABLE>(s, tw);
#pragma unroll
      for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = s[k2];
    }
  }
}

// Two-level in-place transform of a [N][W] tile (rows = points, natural order in and out).
template <typename TO, typename TI> __device__ __forceinline__ TO conv(TI x) { return mk<TO>(decltype(TO::x)(x.x), decltype(TO::x)(x.y)); }

// Barrier of the CTA's NT compute threads (named barrier 1).  A kernel with a producer warp runs it
// after the NT compute threads; that warp never joins, so the compute threads synchronise among
// themselves.  Without a producer warp NT is the whole CTA.
template <int NT> __device__ __forceinline__ void csync() { asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); }
// the same barrier, returning whether any compute thread passed a nonzero value (uniform result)
template <int NT> __device__ __forceinline__ bool csync_or(int v) {
  uint32_t r;
  asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
               : "=r"(r)
               : "r"(v), "n"(NT)
               : "memory");
  return r != 0;
}
using ptx::mbar_arrive;

// The tile transforms below end without a barrier: their last step writes only addresses the
// writing thread owns in that step, and the kernel's fence + barrier before the TMA store (or an
// explicit barrier before another sweep) orders those writes for the other threads.

// Two-level transform of one [N][W] tile.
//   step A: N1-point DFTs down the columns j2 (points j2 + N2 j1), twiddle W_N^{j2 k1};
//   step B: N2-point DFTs along the rows k1, outputs in natural order m = k1 + N1 k2.
// Step A reads `asrc` (times an optional per-point factor `pre`, applied on load) and writes
// `adst`; step B reads `adst` and hands every output value to `put(m, w, value)`.  When
// HOLD is set (step B writes into the buffer it reads), all step-B inputs are read into
// registers before a barrier and only then stored.
template <int N, int DIR, int W, int NT, bool HOLD, typename TC, typename SA, typename DA, typename Put>
__device__ __forceinline__ void tile_dft(const SA *asrc, DA *adst, const TC *__restrict__ tw,
                                         const decltype(TC::x) *pre, Put put) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int it = threadIdx.x; it < W * N2; it += NT) {
    const int w = it % W, j2 = it / W;
    TC s[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) {
      s[j1] = conv<TC>(asrc[(j2 + N2 * j1) * W + w]);
      if (pre) s[j1] = cscale(s[j1], pre[j2 + N2 * j1]);
    }
    dft<N1, DIR, N>(s, tw);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++) s[k1] = twmul<DIR, N>(s[k1], tw, j2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) adst[(j2 + N2 * k1) * W + w] = conv<DA>(s[k1]);
  }
  csync<NT>();
  if constexpr (HOLD) {
    constexpr int IB = (W * N1 + NT - 1) / NT;
    TC r[IB][N2];
#pragma unroll
    for (int b = 0; b < IB; b++) {
      const int it = threadIdx.x + b * NT;
      if (it < W * N1) {
        const int w = it % W, k1 = it / W;
#pragma unroll
        for (int j2 = 0; j2 < N2; j2++) r[b][j2] = conv<TC>(adst[(j2 + N2 * k1) * W + w]);
        dft<N2, DIR, N>(r[b], tw);
      }
    }
    csync<NT>();
#pragma unroll
    for (int b = 0; b < IB; b++) {
      const int it = threadIdx.x + b * NT;
      if (it < W * N1) {
        const int w = it % W, k1 = it / W;
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) put(k1 + N1 * k2, w, r[b][k2]);
      }
    }
  } else {
    for (int it = threadIdx.x; it < W * N1; it += NT) {
      const int w = it % W, k1 = it / W;
      TC r[N2];
#pragma unroll
      for (int j2 = 0; j2 < N2; j2++) r[j2] = conv<TC>(adst[(j2 + N2 * k1) * W + w]);
      dft<N2, DIR, N>(r, tw);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) put(k1 + N1 * k2, w, r[k2]);
    }
  }
}

// The in-place transforms below take the tile through one restrict-qualified pointer, so the compiler
// may overlap one item's shared-memory loads with the previous item's stores, and hand every output
// value to epi(m, w, value), which returns what is stored at row m (scaling, epilogue terms, Taylor
// accumulators; the identity for a plain pass).  None ends with a barrier: the last step writes only
// rows its thread read in that step, and the kernel's fence + barrier before the TMA store orders them.

struct Identity {
  template <typename T> __device__ __forceinline__ T operator()(int, int, T v) const { return v; }
};

// Natural order in and out: step A (N1-point DFTs down the columns j2, twiddle W_N^{j2 k1}), step B
// (N2-point DFTs along the rows k1, outputs m = k1 + N1 k2).  Step B reads all its inputs before a
// barrier and stores after it (it writes other rows than it reads).
template <int N, int DIR, int W, int NT, typename T, typename Epi>
__device__ __forceinline__ void tile_dft_inplace(T *__restrict__ buf, const T *__restrict__ tw, Epi epi) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int it = threadIdx.x; it < W * N2; it += NT) {
    const int w = it % W, j2 = it / W;
    T s[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) s[j1] = buf[(j2 + N2 * j1) * W + w];
    dft<N1, DIR, N>(s, tw);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++) s[k1] = twmul<DIR, N>(s[k1], tw, j2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) buf[(j2 + N2 * k1) * W + w] = s[k1];
  }
  csync<NT>();
  constexpr int IB = (W * N1 + NT - 1) / NT;
  T r[IB][N2];
#pragma unroll
  for (int b = 0; b < IB; b++) {
    const int it = threadIdx.x + b * NT;
    if (it < W * N1) {
      const int w = it % W, k1 = it / W;
#pragma unroll
      for (int j2 = 0; j2 < N2; j2++) r[b][j2] = buf[(j2 + N2 * k1) * W + w];
      dft<N2, DIR, N, (sizeof(decltype(T::x)) == 4 && DIR > 0)>(r[b], tw);
    }
  }
  csync<NT>();
#pragma unroll
  for (int b = 0; b < IB; b++) {
    const int it = threadIdx.x + b * NT;
    if (it < W * N1) {
      const int w = it % W, k1 = it / W;
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) buf[(k1 + N1 * k2) * W + w] = epi(k1 + N1 * k2, w, r[b][k2]);
    }
  }
}

// forward column step in place: N1-point DFT down column j2, twiddle W_N^{j2 k1}
template <int N, int W, int NT, typename T>
__device__ __forceinline__ void col_forward_inplace(T *__restrict__ buf, const T *__restrict__ tw) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int it = threadIdx.x; it < W * N2; it += NT) {
    const int w = it % W, j2 = it / W;
    T s[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) s[j1] = buf[(j2 + N2 * j1) * W + w];
    dft<N1, +1, N>(s, tw);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++) s[k1] = twmul<+1, N>(s[k1], tw, j2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) buf[(j2 + N2 * k1) * W + w] = s[k1];
  }
}

// inverse column step in place: inverse N1-point DFT down column j2, x[j2 + N2 j1] in natural order
template <int N, int W, int NT, typename T, typename Epi>
__device__ __forceinline__ void col_inverse_inplace(T *__restrict__ buf, const T *__restrict__ tw, Epi epi) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int it = threadIdx.x; it < W * N2; it += NT) {
    const int w = it % W, j2 = it / W;
    T s[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) s[k1] = buf[(j2 + N2 * k1) * W + w];
    dft<N1, -1, N>(s, tw);
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) buf[(j2 + N2 * j1) * W + w] = epi(j2 + N2 * j1, w, s[j1]);
  }
}

// The x pass of the real-space operator in place: forward transform, per-frequency factor fac[m],
// inverse transform.  The inverse runs the forward's two steps transposed (step B first, with
// conjugate twiddles, then step A), so it starts from the forward's k1-major output and every step
// writes the rows it read: three shared-memory sweeps and two barriers, no transposition.
//   forward A: N1-point DFTs down the columns j2, twiddle W_N^{j2 k1}
//   forward B, factor, inverse B: N2-point DFT along row k1, times fac[k1 + N1 k2], inverse
//     N2-point DFT, twiddle W_N^{-j2 k1} (rows of up to 12 points batched two items at a time)
//   inverse A: inverse N1-point DFTs down the columns j2, natural order
template <int N, int W, int NT, typename T, typename Epi>
__device__ __forceinline__ void tile_kin_inplace(T *__restrict__ buf, const T *__restrict__ tw,
                                                 const decltype(T::x) *__restrict__ fac, int wsplit, Epi epi) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  constexpr int IB = N2 <= 12 ? (W * N1 + NT - 1) / NT : 1;
  col_forward_inplace<N, W, NT, T>(buf, tw);
  csync<NT>();
  for (int it0 = threadIdx.x; it0 < W * N1; it0 += IB * NT) {
    T r[IB][N2];
#pragma unroll
    for (int b = 0; b < IB; b++) {
      const int it = it0 + b * NT;
      if (it < W * N1) {
        const int w = it % W, k1 = it / W;
#pragma unroll
        for (int j2 = 0; j2 < N2; j2++) r[b][j2] = buf[(j2 + N2 * k1) * W + w];
      }
    }
#pragma unroll
    for (int b = 0; b < IB; b++) {
      const int it = it0 + b * NT;
      if (it < W * N1) {
        const int w = it % W, k1 = it / W;
        const auto *f = fac + (w >= wsplit ? N : 0);  // the column's line
        dft<N2, +1, N>(r[b], tw);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) r[b][k2] = cscale(r[b][k2], f[k1 + N1 * k2]);
        dft<N2, -1, N>(r[b], tw);
        if (k1 > 0) {
#pragma unroll
          for (int j2 = 1; j2 < N2; j2++) r[b][j2] = twmul<-1, N>(r[b][j2], tw, j2 * k1);
        }
#pragma unroll
        for (int j2 = 0; j2 < N2; j2++) buf[(j2 + N2 * k1) * W + w] = r[b][j2];
      }
    }
  }
  csync<NT>();
  col_inverse_inplace<N, W, NT, T>(buf, tw, epi);
}

// Forward transform in place with the output in digit-reversed order: row k2 + N2 k1 receives
// frequency k1 + N1 k2.  Step B writes the rows it read, so no second barrier is needed.
template <int N, int W, int NT, typename T, typename Epi>
__device__ __forceinline__ void tile_fwd_perm_inplace(T *__restrict__ buf, const T *__restrict__ tw, Epi epi) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, IB = (W * N1 + NT - 1) / NT;
  col_forward_inplace<N, W, NT, T>(buf, tw);
  csync<NT>();
  T r[IB][N2];
#pragma unroll
  for (int b = 0; b < IB; b++) {
    const int it = threadIdx.x + b * NT;
    if (it < W * N1) {
      const int w = it % W, k1 = it / W;
#pragma unroll
      for (int j2 = 0; j2 < N2; j2++) r[b][j2] = buf[(j2 + N2 * k1) * W + w];
    }
  }
#pragma unroll
  for (int b = 0; b < IB; b++) {
    const int it = threadIdx.x + b * NT;
    if (it < W * N1) {
      const int w = it % W, k1 = it / W;
      dft<N2, +1, N, (sizeof(decltype(T::x)) == 4)>(r[b], tw);
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) buf[(k2 + N2 * k1) * W + w] = epi(k2 + N2 * k1, w, r[b][k2]);
    }
  }
}

// Inverse transform in place of a tile whose rows are in digit-reversed order (row k2 + N2 k1 holds
// frequency k1 + N1 k2): the forward's steps transposed, conjugate twiddles; natural order out.
template <int N, int W, int NT, typename T, typename Epi>
__device__ __forceinline__ void tile_inv_perm_inplace(T *__restrict__ buf, const T *__restrict__ tw, Epi epi) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2, IB = (W * N1 + NT - 1) / NT;
  T r[IB][N2];
#pragma unroll
  for (int b = 0; b < IB; b++) {
    const int it = threadIdx.x + b * NT;
    if (it < W * N1) {
      const int w = it % W, k1 = it / W;
#pragma unroll
      for (int k2 = 0; k2 < N2; k2++) r[b][k2] = buf[(k2 + N2 * k1) * W + w];
    }
  }
#pragma unroll
  for (int b = 0; b < IB; b++) {
    const int it = threadIdx.x + b * NT;
    if (it < W * N1) {
      const int w = it % W, k1 = it / W;
      dft<N2, -1, N>(r[b], tw);
      if (k1 > 0) {
#pragma unroll
        for (int j2 = 1; j2 < N2; j2++) r[b][j2] = twmul<-1, N>(r[b][j2], tw, j2 * k1);
      }
#pragma unroll
      for (int j2 = 0; j2 < N2; j2++) buf[(j2 + N2 * k1) * W + w] = r[b][j2];
    }
  }
  csync<NT>();
  col_inverse_inplace<N, W, NT, T>(buf, tw, epi);
}

// Column and row steps of the two-level transforms below.
//   column step: item (j2, w), N1 values at rows j2 + N2 j1; a runtime loop over the thread's items
//   row step:    item (k1, w), N2 values at rows j2 + N2 k1; the thread's IB items are batched (all
//                loads first, then the arithmetic, then the stores) so their loads are in flight
//                together and their arithmetic interleaves
// Both write only the rows they read, so no barrier separates a step's loads from its stores.

// forward column step: N1-point DFT down column j2, twiddle W_N^{j2 k1}  (asrc -> work)
template <int N, int W, int NT, typename TC, typename SA>
__device__ __forceinline__ void col_forward(const SA *asrc, TC *work, const TC *__restrict__ tw) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int it = threadIdx.x; it < W * N2; it += NT) {
    const int w = it % W, j2 = it / W;
    TC s[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) s[j1] = conv<TC>(asrc[(j2 + N2 * j1) * W + w]);
    dft<N1, +1, N>(s, tw);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++) s[k1] = twmul<+1, N>(s[k1], tw, j2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) work[(j2 + N2 * k1) * W + w] = s[k1];
  }
}

// inverse column step: inverse N1-point DFT down column j2; x[j2 + N2 j1] to put (natural order)
template <int N, int W, int NT, typename TC, typename Put>
__device__ __forceinline__ void col_inverse(const TC *work, const TC *__restrict__ tw, Put put) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  for (int it = threadIdx.x; it < W * N2; it += NT) {
    const int w = it % W, j2 = it / W;
    TC s[N1];
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) s[k1] = work[(j2 + N2 * k1) * W + w];
    dft<N1, -1, N>(s, tw);
#pragma unroll
    for (int j1 = 0; j1 < N1; j1++) put(j2 + N2 * j1, w, s[j1]);
  }
}

// Forward transform, per-frequency factor fac[m], inverse transform of one [N][W] tile (the x pass of
// the real-space operator), with the arithmetic in a separate buffer `work` (wider type than the
// tile); the in-place form for equal types is tile_kin_inplace.  The inverse runs the forward's two steps transposed (step B first, with
// conjugate twiddles, then step A), so it starts from the forward's k1-major output and every step
// writes the addresses it read: three shared-memory sweeps and two barriers, no transposition.
//   forward A: N1-point DFTs down the columns j2, twiddle W_N^{j2 k1}           (asrc -> work)
//   forward B, factor, inverse B: N2-point DFT along row k1, times fac[k1 + N1 k2], inverse
//     N2-point DFT, twiddle W_N^{-j2 k1}                                      (work, in place)
//   inverse A: inverse N1-point DFTs down the columns j2; x[j2 + N2 j1] goes to put(m, w, value)
// `asrc` may be `work` itself.  No barrier follows the last step.
template <int N, int W, int NT, typename TC, typename SA, typename Put>
__device__ __forceinline__ void tile_dft_kin(const SA *asrc, TC *work, const TC *__restrict__ tw,
                                             const decltype(TC::x) *fac, int wsplit, Put put) {
  constexpr int N1 = Split<N>::N1, N2 = Split<N>::N2;
  // rows of up to 12 points are batched (two transforms per row keep longer rows one at a time)
  constexpr int IB = N2 <= 12 ? (W * N1 + NT - 1) / NT : 1;
  col_forward<N, W, NT, TC>(asrc, work, tw);
  csync<NT>();
  for (int it0 = threadIdx.x; it0 < W * N1; it0 += IB * NT) {
    TC r[IB][N2];
#pragma unroll
    for (int b = 0; b < IB; b++) {
      const int it = it0 + b * NT;
      if (it < W * N1) {
        const int w = it % W, k1 = it / W;
#pragma unroll
        for (int j2 = 0; j2 < N2; j2++) r[b][j2] = work[(j2 + N2 * k1) * W + w];
      }
    }
#pragma unroll
    for (int b = 0; b < IB; b++) {
      const int it = it0 + b * NT;
      if (it < W * N1) {
        const int w = it % W, k1 = it / W;
        const auto *f = fac + (w >= wsplit ? N : 0);  // the column's line
        dft<N2, +1, N>(r[b], tw);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) r[b][k2] = cscale(r[b][k2], f[k1 + N1 * k2]);
        dft<N2, -1, N>(r[b], tw);
        if (k1 > 0) {
#pragma unroll
          for (int j2 = 1; j2 < N2; j2++) r[b][j2] = twmul<-1, N>(r[b][j2], tw, j2 * k1);
        }
#pragma unroll
        for (int j2 = 0; j2 < N2; j2++) work[(j2 + N2 * k1) * W + w] = r[b][j2];
      }
    }
  }
  csync<NT>();
  col_inverse<N, W, NT, TC>(work, tw, put);
}

struct Geom2 {
  Geom g;           // grid and line decomposition (point strides)
  int axis;
  int nsb;          // state blocks per line
  long long ntiles;
  int stages;
  int cwords;       // 32-bit words per complex element
  int aux_single;   // second input tiles single-buffered (1) or one set per ring stage (0)
  int cpa;          // rows that are not 16-byte multiples: the compute threads move tiles with 8-byte
                    // cp.async loads and plain stores instead of TMA (two stages, second tiles per stage)
  int flat;         // y and x passes over flattened columns (below); nsb is then the column blocks per row
  long long ncols;  // flat: columns per row, nz*S (y pass) or ny*nz*S (x pass)
};

// Flattened columns.  A y (x) transform acts on every column of the [nx][ny][nz*S] ([nx][ny*nz*S]) view
// of the set alike, so a tile may take any W consecutive columns of that view: the (z, state) or
// (y, z, state) pairs follow one another in memory.  Rows are then W full elements for every state count
// (odd counts too, whose point rows are not 16-byte multiples, and counts that leave the last state block
// of a line part-empty), and only the last tile of each row runs past its end (TMA fills the loads with
// zeros and clips the stores).  With S a multiple of W the tiles, and their order, are those of the
// (line, state block) decomposition.  The kinetic factor of a column depends on its (y, z) line; with
// S >= W a tile's columns lie on at most two lines.

template <int VAR> constexpr int dir_first() { return (base_var(VAR) == INV_STORE || base_var(VAR) == INV_FINAL) ? -1 : +1; }

// Tiles of 256-byte rows, or 128-byte rows when the butterflies run in a wider type than the storage
// (the tile then also needs an exchange buffer of that type, and smaller tiles let several CTAs share
// an SM to cover the double-precision latency).
template <typename R, typename CR, int WIDE = 0> constexpr int tile_w() {
  return WIDE ? 512 / int(2 * sizeof(R)) : (sizeof(CR) > sizeof(R) ? 128 : 256) / int(2 * sizeof(R));
}
// Threads per CTA.  The two steps of a tile transform have W*N2 and W*N1 independent line pieces; with
// 128 threads and 16-state tiles (N1 = 8) the first step of N = 72, 96, 120, 128 takes two rounds in
// which part of the CTA idles at the next barrier, so those tiles get one thread per first-step piece.
// The kinetic pass (two transforms, the second with two idle thirds in its second step either way)
// keeps 128 threads and more CTAs per SM.  The single-precision final passes of 96- to 128-point
// lines (two tiles per stage: two stages, and 8 warps per SM at 128 threads for 96 points, 4 for
// 120) run one thread per column item: 384 threads for 96 points (measured: 1.06 ms against 1.15 ms
// at 96^3 x 256), 480 for 120.
template <typename R, typename CR, int N, int VAR, int WIDE = 0> constexpr int threads_of() {
  constexpr int W = tile_w<R, CR, WIDE>();
  constexpr int A = W * Split<N>::N2, B = W * Split<N>::N1;
  constexpr int M = A > B ? A : B;
  if constexpr (WIDE) return 256;
  if constexpr (base_var(VAR) == INV_FINAL && W == 32 && N >= 96 && sizeof(CR) == 4) return (A + 31) / 32 * 32;
  return (VAR != MID_KIN && W == 16 && M > 128 && M <= 256) ? (M + 31) / 32 * 32 : 128;
}

// Whether the kernel runs a producer warp: one extra warp whose lane 0 issues every TMA load and
// store and waits for the stores to drain, so no compute thread stalls on the copies.  Measured at
// 96^3 x 256: the single-precision passes gain 8-15 % (final pass 0.80 ms against 0.93, kinetic pass
// 0.68 against 0.73); the FP64 passes, already at the HBM limit, lose (forward 1.29 against 1.11).
template <typename R, typename CR, int N, int VAR> constexpr bool ws_of() {
  return sizeof(R) == 4 && sizeof(CR) == 4;
}
template <typename R, typename CR, int N, int VAR, int WIDE = 0> constexpr int block_threads_of() {
  return threads_of<R, CR, N, VAR, WIDE>() + (ws_of<R, CR, N, VAR>() ? 32 : 0);
}

// CTAs per SM the register allocation must allow: four for the single-precision kinetic pass of lines
// up to 96 points (two transforms per tile, latency-bound with fewer warps; longer lines would spill);
// 0 (no constraint: the compiler's own register choice) otherwise.
template <typename R, typename CR, int N, int VAR, int WIDE = 0> constexpr int min_ctas_of() {
  if constexpr (WIDE) return 0;
  return (VAR == MID_KIN && sizeof(R) == 4 && sizeof(CR) == 4 && N <= 96) ? 4 : 0;
}

template <typename R, typename CR, int N, int VAR, int WIDE>
__global__ void __launch_bounds__(block_threads_of<R, CR, N, VAR, WIDE>(), min_ctas_of<R, CR, N, VAR, WIDE>()) fft2_kernel(const __grid_constant__ CUtensorMap map_in,
                                                   const __grid_constant__ CUtensorMap map_out,
                                                   const __grid_constant__ CUtensorMap map_aux,
                                                   const __grid_constant__ CUtensorMap map_base, PassArgs<R> a, Geom2 gg,
                                                   const C2<CR> *__restrict__ twg, int *err) {
  using T = C2<R>;
  using TC = C2<CR>;
  constexpr int NT = threads_of<R, CR, N, VAR, WIDE>();   // compute threads
  constexpr bool WS = ws_of<R, CR, N, VAR>();             // plus a producer warp
  constexpr int NTT = block_threads_of<R, CR, N, VAR, WIDE>();
  constexpr bool SPLIT = sizeof(CR) > sizeof(R);          // exchange buffer in the arithmetic type
  constexpr int W = tile_w<R, CR, WIDE>();
  constexpr int TILE = N * W;                       // complex elements per tile
  constexpr uint32_t TILE_BYTES = TILE * sizeof(T);
  constexpr bool AUX = has_aux(VAR);
  const int NS = gg.stages;
  // a Horner step (final pass of the real-space operator): a third tile per stage holds the base
  const bool horner = AUX && a.hbase != nullptr;

  // The second input tile (psi of V psi or of the Laplacian term) and the Horner base are needed only in
  // the last step of a tile's transform.  Either every ring stage holds them beside its tile (loaded with
  // it), or, when that would leave one CTA per SM (gg.aux_single), they are single-buffered: loaded for
  // the CTA's next tile as soon as its current one is computed, so that they land during the next tile's
  // first steps, while the ring stages hold one tile each.
  const int naux = AUX ? (horner ? 2 : 1) : 0;
  const bool aux1 = AUX && gg.aux_single;

  extern __shared__ __align__(1024) unsigned char smem[];
  T *stage_in = reinterpret_cast<T *>(smem);                         // NS tiles
  T *aux_ring = stage_in + size_t(NS) * TILE;                        // naux tiles, or NS x naux
  TC *exch = reinterpret_cast<TC *>(aux_ring + size_t(aux1 ? 1 : NS) * naux * TILE);  // one tile when SPLIT
  constexpr int TWN = tw_entries<CR>(N);
  TC *tw = exch + (SPLIT ? TILE : 0);                                // twiddles (high, then low parts)
  CR *linev = reinterpret_cast<CR *>(tw + TWN);                      // N per-point factors of the current line
  uint64_t *bar = reinterpret_cast<uint64_t *>(tw + TWN + N);        // NS "tile loaded" barriers (8-byte aligned)
  uint64_t *done = bar + NS;                                         // NS "tile computed" barriers (producer warp)
  uint64_t *abar = done + NS;                                        // "second input tiles loaded"
  volatile int *abort_flag = reinterpret_cast<volatile int *>(abar + 1);

  const Geom &g = gg.g;
  for (int i = threadIdx.x; i < TWN; i += NTT) tw[i] = twg[i];
  if (threadIdx.x == 0) {
    *abort_flag = 0;
    for (int s = 0; s < NS; s++) {
      mbar_init(&bar[s], 1);
      if constexpr (WS) mbar_init(&done[s], NT);
    }
    mbar_init(abar, 1);
    mbar_init_fence();
  }
  __syncthreads();

  auto coords = [&](long long t, int &c0, int &c1, int &c2, int &c3) {
    if (gg.flat) {
      c0 = int((t % gg.nsb) * W) * gg.cwords;
      c1 = 0;
      c2 = gg.axis == 1 ? int(t / gg.nsb) : 0;
      c3 = 0;
      return;
    }
    const long long L = t / gg.nsb;
    const int s0 = int(t % gg.nsb) * W;
    const int la = int(L / g.nb), lb = int(L % g.nb);
    c0 = s0 * gg.cwords;
    if (gg.axis == 2) { c1 = 0; c2 = lb; c3 = la; }        // z-lines: (x, y) fixed
    else if (gg.axis == 1) { c1 = lb; c2 = 0; c3 = la; }   // y-lines: (x, z) fixed
    else { c1 = lb; c2 = la; c3 = 0; }                     // x-lines: (y, z) fixed
  };
  auto issue = [&](int st, long long t) {
    int c0, c1, c2, c3;
    coords(t, c0, c1, c2, c3);
    mbar_expect_tx(&bar[st], uint32_t(aux1 ? 1 : 1 + naux) * TILE_BYTES);
    tma_load_4d(stage_in + size_t(st) * TILE, &map_in, &bar[st], c0, c1, c2, c3);
    if (AUX && !aux1) {
      T *ax = aux_ring + size_t(st) * naux * TILE;
      tma_load_4d(ax, &map_aux, &bar[st], c0, c1, c2, c3);
      if (horner) tma_load_4d(ax + TILE, &map_base, &bar[st], c0, c1, c2, c3);
    }
  };
  // single-buffered: the second input tile (and the Horner base) of tile t; the k-th such load completes
  // phase k of abar
  auto issue_aux = [&](long long t) {
    int c0, c1, c2, c3;
    coords(t, c0, c1, c2, c3);
    mbar_expect_tx(abar, uint32_t(naux) * TILE_BYTES);
    tma_load_4d(aux_ring, &map_aux, abar, c0, c1, c2, c3);
    if (horner) tma_load_4d(aux_ring + TILE, &map_base, abar, c0, c1, c2, c3);
  };

  // bounded wait on an mbarrier phase; false (and the error flag raised) on expiry or abort
  auto wait_bar = [&](uint64_t *b, uint32_t parity) -> bool {
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(b, parity)) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > 2000000000ull) {
        *abort_flag = 1;
        atomicExch(err, 1);
        return false;
      }
    }
    return true;
  };

  // tiles whose loads the issuing thread has started (the i-th goes to stage i % NS, phase i / NS);
  // before the CTA ends, that thread waits (bounded) for the last NS of them, so that after an aborted
  // wait no load still lands in shared memory (on the normal path those phases are complete already)
  int nissued = 0, naux_issued = 0;
  auto drain = [&]() {
    for (int i = nissued - NS < 0 ? 0 : nissued - NS; i < nissued; i++)
      ptx::mbar_wait_bounded(&bar[i % NS], uint32_t(i / NS) & 1u, 2000000000ull);
    if (naux_issued > 0) ptx::mbar_wait_bounded(abar, uint32_t(naux_issued - 1) & 1u, 2000000000ull);
  };
  if (threadIdx.x == (WS ? NT : 0) && !gg.cpa) {
    for (int s = 0; s < NS; s++) {
      const long long t = blockIdx.x + (long long)s * gridDim.x;
      if (t < gg.ntiles) issue(s, t), nissued++;
    }
    if (aux1 && blockIdx.x < gg.ntiles) issue_aux(blockIdx.x), naux_issued++;
  }
  if constexpr (WS) {
    // rows that TMA cannot move: the compute threads copy them (below); the producer warp has no work
    if (threadIdx.x >= NT && gg.cpa) return;
    if (threadIdx.x >= NT) {
      // producer warp: lane 0 stores every computed tile, waits for the store to read the stage and
      // refills it with the tile NS steps ahead
      if (threadIdx.x == NT) {
        int k = 0;
        for (long long t = blockIdx.x; t < gg.ntiles; t += gridDim.x, k++) {
          const int st = k % NS;
          if (!wait_bar(&done[st], uint32_t(k / NS) & 1u)) break;
          int c0, c1, c2, c3;
          coords(t, c0, c1, c2, c3);
          tma_store_4d(&map_out, stage_in + size_t(st) * TILE, c0, c1, c2, c3);
          bulk_commit();
          // the second input tiles were read by the finished tile's epilogue: load the next tile's
          if (aux1 && t + gridDim.x < gg.ntiles) issue_aux(t + gridDim.x), naux_issued++;
          bulk_wait_read0();
          const long long tn = t + (long long)NS * gridDim.x;
          if (tn < gg.ntiles) issue(st, tn), nissued++;
        }
        drain();
        bulk_wait0();
      }
      return;
    }
  }

  const bool scaled = a.scale != 1.0;
  // 8-byte copies by the compute threads (rows that are not 16-byte multiples, gg.cpa): tile t's rows of
  // `src` into dst, consecutive threads on consecutive states; with the second input tiles of the stage
  auto cpa_rows = [&](long long t, long long &pbase, int &s0, int &ws) {
    const long long L = t / gg.nsb;
    s0 = int(t % gg.nsb) * W;
    ws = a.S - s0 < W ? a.S - s0 : W;
    pbase = (L / g.nb) * g.sa + (L % g.nb) * g.sb;
  };
  auto cpa_load = [&](T *dst, const T *src, long long t) {
    long long pbase;
    int s0, ws;
    cpa_rows(t, pbase, s0, ws);
    for (int e = threadIdx.x; e < TILE; e += NT) {
      const int r = e / W, c = e % W;
      if (c < ws) ptx::cp_async8(dst + e, src + (pbase + r * g.sp) * a.S + s0 + c);
    }
  };
  auto cpa_load_stage = [&](int st, long long t) {
    cpa_load(stage_in + size_t(st) * TILE, a.in, t);
    if constexpr (AUX) {
      cpa_load(aux_ring + size_t(st) * naux * TILE, a.psi, t);
      if (horner) cpa_load(aux_ring + size_t(st) * naux * TILE + TILE, a.hbase, t);
    }
  };
  if (gg.cpa) {
    if (blockIdx.x < gg.ntiles) cpa_load_stage(0, blockIdx.x);
    ptx::cp_async_commit();
  }
  int i = 0;
  for (long long t = blockIdx.x; t < gg.ntiles; t += gridDim.x, i++) {
    const int st = i % NS;
    const uint32_t par = uint32_t(i / NS) & 1u;
    if (gg.cpa) {
      // two stages: the next tile's copies are issued before this tile's are awaited
      if (t + gridDim.x < gg.ntiles) cpa_load_stage((i + 1) % NS, t + gridDim.x);
      ptx::cp_async_commit();
      ptx::cp_async_wait<1>();
      csync<NT>();
    } else {
      // bounded wait for this stage's TMA load; every compute thread takes the same decision
      const bool ok = wait_bar(&bar[st], par);
      if (csync_or<NT>(!ok || *abort_flag)) break;
    }

    T *buf = stage_in + size_t(st) * TILE;
    const T *aux = aux_ring + (aux1 ? 0 : size_t(st) * naux * TILE);
    const T *base = aux + TILE;
    bool aux_ready = !aux1;  // this thread has waited for the tile's second input (phase i of abar)
    long long L;
    int s0, la, lb;
    if constexpr (VAR == MID_KIN) {
      // the issue-bound kinetic pass: 32-bit divisions (the host keeps the tile count below 2^31)
      const int ti = int(t), Li = ti / gg.nsb;
      L = Li;
      s0 = (ti - Li * gg.nsb) * W;
      la = Li / g.nb;
      lb = Li - la * g.nb;
    } else {
      L = t / gg.nsb;
      s0 = int(t % gg.nsb) * W;
      la = int(L / g.nb);
      lb = int(L % g.nb);
    }
    const long long pbase = la * g.sa + lb * g.sb;

    // per-point factors of this line (consumed after the first barrier of the transform); flattened
    // columns: of the tile's first line at linev[0, N) and, from column wsplit on, of the next at [N, 2N)
    int wsplit = W;
    if constexpr (VAR == MID_KIN || VAR == FWD_LAPLADD) {
      if (gg.flat) {
        // 32-bit divisions: a view row has fewer than 2^31 words (the host checks it)
        const int col0 = int(t % gg.nsb) * W, l0 = col0 / a.S, nlines = g.n[1] * g.n[2];
        wsplit = (l0 + 1) * a.S - col0 < W ? (l0 + 1) * a.S - col0 : W;
        const int nl = (wsplit < W && l0 + 1 < nlines) ? 2 : 1;
        for (int e = threadIdx.x; e < nl * N; e += NT) {
          const int l = l0 + e / N;  // x-line (y, z) = (l / nz, l % nz)
          const int ly = l / g.n[2];
          int ix, iy, iz;
          line_coords(gg.axis, ly, l - ly * g.n[2], e % N, ix, iy, iz);
          if (a.perm_n2[1]) iy = iy / a.perm_n2[1] + (g.n[1] / a.perm_n2[1]) * (iy % a.perm_n2[1]);
          if (a.perm_n2[2]) iz = iz / a.perm_n2[2] + (g.n[2] / a.perm_n2[2]) * (iz % a.perm_n2[2]);
          linev[e] = CR(lapl_value(g, ix, iy, iz, a.lap_factor, a.gc));
        }
      } else
      for (int m = threadIdx.x; m < N; m += NT) {
        int ix, iy, iz;
        line_coords(gg.axis, la, lb, m, ix, iy, iz);
        // axes held in digit-reversed frequency order: position k2 + N2 k1 is frequency k1 + N1 k2
        if (a.perm_n2[1]) iy = iy / a.perm_n2[1] + (g.n[1] / a.perm_n2[1]) * (iy % a.perm_n2[1]);
        if (a.perm_n2[2]) iz = iz / a.perm_n2[2] + (g.n[2] / a.perm_n2[2]) * (iz % a.perm_n2[2]);
        linev[m] = CR(lapl_value(g, ix, iy, iz, a.lap_factor, a.gc));
      }
    } else if constexpr (base_var(VAR) == INV_FINAL || VAR == FWD_VPSI) {
      for (int m = threadIdx.x; m < N; m += NT)
        linev[m] = CR(a.V[(pbase + m * g.sp) * a.nspin + a.spin]) + CR(a.vshift);
    }
    if constexpr (VAR == FWD_VPSI) {
      csync<NT>();
      if (a.nl_offs) {
        // Fourier-form operator: (V + shift) psi + nonlocal(psi) formed in shared memory before the transform
        for (int e = threadIdx.x; e < TILE; e += NT) {
          const int m = e / W, w = e % W, s = s0 + w;
          if (s < a.S) {
            const long long pt = pbase + m * g.sp;
            T v = conv<T>(cscale(conv<TC>(buf[e]), linev[m]));
            buf[e] = cadd(v, nl_term<R>(a, pt, s));
          }
        }
        csync<NT>();
      }
    }

    // final value of one output element: scaling, epilogue term, Horner step (base + c * value, the
    // value rounded to the storage type first, as the operator's output would be)
    auto epi_out = [&](int m, int w, TC v) -> T {
      if constexpr (AUX) {
        if (!aux_ready) {
          wait_bar(abar, uint32_t(i) & 1u);  // on expiry the error flag is raised and the tile loop ends
          aux_ready = true;
        }
      }
      if (scaled) v = kscale(v, a.scale);
      if constexpr (base_var(VAR) == INV_FINAL || VAR == FWD_LAPLADD) v = cadd(v, cscale(conv<TC>(aux[m * W + w]), linev[m]));
      if constexpr (AUX) {
        if (horner) return cadd(base[m * W + w], cmul(a.hc, conv<T>(v)));
      }
      return conv<T>(v);
    };
    auto put_out = [&](int m, int w, TC v) { buf[m * W + w] = epi_out(m, w, v); };
    const CR *pre = (VAR == FWD_VPSI && !a.nl_offs) ? linev : nullptr;
    constexpr int D = dir_first<VAR>();
    const T *twt = reinterpret_cast<const T *>(tw);

    if constexpr (SPLIT) {
      static_assert(!is_perm(VAR), "digit-reversed passes run with equal storage and arithmetic types");
      if constexpr (VAR == MID_KIN) {
        // forward, multiply by the kinetic factor, backward
        tile_dft_kin<N, W, NT, TC>(buf, exch, tw, linev, wsplit, put_out);
      } else {
        tile_dft<N, D, W, NT, false, TC>(buf, exch, tw, pre, put_out);
      }
    } else {
      if constexpr (VAR == FWD_VPSI) {
        if (!a.nl_offs) {
          for (int e = threadIdx.x; e < TILE; e += NT) buf[e] = cscale(buf[e], linev[e / W]);
          csync<NT>();
        }
      }
      // plain passes (no scaling, no accumulators) store the transform's values as they are
      const bool plain = !AUX && !scaled;
      if constexpr (VAR == MID_KIN) {
        if (plain) tile_kin_inplace<N, W, NT, T>(buf, twt, linev, wsplit, Identity());
        else tile_kin_inplace<N, W, NT, T>(buf, twt, linev, wsplit, epi_out);
      } else if constexpr (VAR == INV_FINAL_PERM) {
        tile_inv_perm_inplace<N, W, NT, T>(buf, twt, epi_out);
      } else if constexpr (VAR == FWD_PERM || VAR == INV_PERM) {
        if constexpr (VAR == FWD_PERM) tile_fwd_perm_inplace<N, W, NT, T>(buf, twt, Identity());
        else tile_inv_perm_inplace<N, W, NT, T>(buf, twt, Identity());
        if (!plain) {
          csync<NT>();
          for (int e = threadIdx.x; e < TILE; e += NT) put_out(e / W, e % W, buf[e]);
        }
      } else if constexpr (AUX) {
        // the epilogue (V psi or the Laplacian term, Taylor accumulators) in the transform's last step
        tile_dft_inplace<N, D, W, NT, T>(buf, twt, epi_out);
      } else {
        tile_dft_inplace<N, D, W, NT, T>(buf, twt, Identity());
        if (!plain) {
          csync<NT>();
          for (int e = threadIdx.x; e < TILE; e += NT) put_out(e / W, e % W, buf[e]);
        }
      }
    }

    if (gg.cpa) {
      // plain stores of the computed tile; the barrier after them frees the stage for the copies of the
      // tile two steps ahead
      csync<NT>();
      long long pbase;
      int s0, ws;
      cpa_rows(t, pbase, s0, ws);
      for (int e = threadIdx.x; e < TILE; e += NT) {
        const int r = e / W, c = e % W;
        if (c < ws) a.out[(pbase + r * g.sp) * a.S + s0 + c] = buf[e];
      }
      csync<NT>();
      continue;
    }
    fence_proxy_async();
    if constexpr (WS) {
      mbar_arrive(&done[st]);  // the producer warp stores the tile and refills the stage
    } else {
      csync<NT>();
      if (threadIdx.x == 0) {
        int c0, c1, c2, c3;
        coords(t, c0, c1, c2, c3);
        tma_store_4d(&map_out, buf, c0, c1, c2, c3);
        bulk_commit();
        if (aux1 && t + gridDim.x < gg.ntiles) issue_aux(t + gridDim.x), naux_issued++;
        bulk_wait_read0();  // the stage may be refilled once the store has read it
        const long long tn = t + (long long)NS * gridDim.x;
        if (tn < gg.ntiles) issue(st, tn), nissued++;
      }
    }
  }
  if (gg.cpa) ptx::cp_async_wait_all();
  if (!WS && threadIdx.x == 0) {
    drain();
    bulk_wait0();
  }
}

}  // namespace v2
}  // namespace inqb

// ------------------------------------------------------------------ host side
#include <cudaTypedefs.h>

#include <mutex>

namespace inqb {
namespace v2 {

inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  INQB_REQUIRE(fn != nullptr, INQB_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  return fn;
}

// 4-D map of a [nx][ny][nz][S] complex array as 32-bit words; box = W states x N points along `axis`.
inline CUtensorMap orbital_map(const void *base, const Basis &b, int S, int cwords, int axis, int W) {
  CUtensorMap m;
  const cuuint64_t row = cuuint64_t(S) * cwords * 4;
  cuuint64_t dims[4] = {cuuint64_t(S) * cwords, cuuint64_t(b.n[2]), cuuint64_t(b.n[1]), cuuint64_t(b.n[0])};
  cuuint64_t strides[3] = {row, row * b.n[2], row * b.n[2] * b.n[1]};
  cuuint32_t box[4] = {cuuint32_t(W * cwords), cuuint32_t(axis == 2 ? b.n[2] : 1), cuuint32_t(axis == 1 ? b.n[1] : 1),
                       cuuint32_t(axis == 0 ? b.n[0] : 1)};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, const_cast<void *>(base), dims, strides, box,
                                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  INQB_REQUIRE(r == CUDA_SUCCESS, INQB_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return m;
}

// 4-D map of the flattened-column view of a [nx][ny][nz][S] complex array as 32-bit words: y pass
// [nx][ny][nz*S], x pass [nx][ny*nz*S]; box = W columns x N points along `axis`.
inline CUtensorMap flat_map(const void *base, const Basis &b, long long ncols, int cwords, int axis, int W) {
  CUtensorMap m;
  const cuuint64_t roww = cuuint64_t(ncols) * cwords;
  const cuuint64_t d1 = cuuint64_t(axis == 1 ? b.n[1] : b.n[0]), d2 = cuuint64_t(axis == 1 ? b.n[0] : 1);
  cuuint64_t dims[4] = {roww, d1, d2, 1};
  cuuint64_t strides[3] = {roww * 4, roww * 4 * d1, roww * 4 * d1 * d2};
  cuuint32_t box[4] = {cuuint32_t(W * cwords), cuuint32_t(d1), 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, const_cast<void *>(base), dims, strides, box,
                                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  INQB_REQUIRE(r == CUDA_SUCCESS, INQB_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
  return m;
}

template <typename R, typename CR, int N, int VAR, int WIDE = 0>
void launch_kernel(Ctx &ctx, const Basis &b, const PassArgs<R> &a, Geom2 gg) {
  using T = C2<R>;
  using TC = C2<CR>;
  constexpr int W = tile_w<R, CR, WIDE>();
  constexpr size_t TILE_BYTES = size_t(N) * W * sizeof(T);
  const int naux = has_aux(VAR) ? (a.hbase ? 2 : 1) : 0;
  constexpr bool SPLIT = sizeof(CR) > sizeof(R);
  constexpr int NT = block_threads_of<R, CR, N, VAR, WIDE>();
  const size_t fixed = (SPLIT ? size_t(N) * W * sizeof(TC) : 0) + size_t(tw_entries<CR>(N) + N) * sizeof(TC) + 64 + 16 * 8;
  // shared memory per CTA: ~113 KB (two CTAs per SM) for the FP64 streaming passes; ~56 KB (four per SM)
  // for the wide-arithmetic, the kinetic and the producer-warp (single-precision) passes, whose
  // arithmetic needs more warps to hide latency (96^3 x 256 single: 3.81 ms per H against 3.89 with
  // four stages of 113 KB)
  size_t budget = (SPLIT || VAR == MID_KIN || ws_of<R, CR, N, VAR>()) ? 56 * 1024 : 113 * 1024;
  // 512-byte-row streaming passes: three stages, one CTA per SM
  if (WIDE) budget = 150 * 1024;
  // second input tiles beside every ring stage when two stages of them leave room for two CTAs per SM,
  // else single-buffered (96^3 x 256: 0.80 against 0.92 ms for the single-precision final pass beside
  // every stage; 120^3 x 256 double: 3.1 against 5.35 ms single-buffered, at two CTAs per SM against one)
  gg.cpa = !gg.flat && (size_t(a.S) * sizeof(T)) % 16 != 0;
  gg.aux_single = !gg.cpa && naux > 0 && size_t(2) * (1 + naux) * TILE_BYTES + fixed > 113 * 1024;
  const size_t per_stage = TILE_BYTES * (gg.aux_single ? 1 : 1 + naux);
  const size_t fixed_aux = gg.aux_single ? naux * TILE_BYTES : 0;
  int ns = budget > fixed + fixed_aux ? int((budget - fixed - fixed_aux) / per_stage) : 0;
  ns = ns < 2 ? 2 : (ns > 6 ? 6 : ns);
  if (ctx.fft_stages > 0) ns = ctx.fft_stages < 2 ? 2 : ctx.fft_stages;
  if (gg.cpa) ns = 2;
  gg.stages = ns;
  if (gg.flat) {
    INQB_REQUIRE(VAR != MID_KIN || a.S >= W, INQB_ERR_UNSUPPORTED, "flattened kinetic tiles span more than two lines");
    gg.nsb = (gg.ncols + W - 1) / W;
    gg.ntiles = gg.axis == 1 ? (long long)b.n[0] * gg.nsb : gg.nsb;
  } else {
    gg.nsb = (a.S + W - 1) / W;
    gg.ntiles = (b.npoints / b.n[gg.axis]) * gg.nsb;
  }
  const size_t smem = per_stage * ns + fixed_aux + fixed;
  INQB_REQUIRE(smem <= ctx.max_smem_optin, INQB_ERR_UNSUPPORTED, "FFT tile does not fit in shared memory");
  INQB_REQUIRE(gg.ntiles < (1LL << 31), INQB_ERR_UNSUPPORTED, "FFT pass has more than 2^31 tiles");
  auto kern = fft2_kernel<R, CR, N, VAR, WIDE>;
  // per instantiation: shared-memory attribute and occupancy, computed under a lock (several host
  // threads may drive contexts at once); the attribute only ever grows
  static std::mutex mtx;
  static int occ_smem = -1, occ_per_sm = 1;
  int per_sm;
  ensure_smem_attr(reinterpret_cast<const void *>(kern), smem);
  {
    std::lock_guard<std::mutex> lock(mtx);
    if (occ_smem != int(smem)) {
      INQB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_per_sm, kern, NT, smem));
      occ_smem = int(smem);
    }
    per_sm = occ_per_sm;
  }
  long long grid = (long long)(per_sm < 1 ? 1 : per_sm) * ctx.num_sms;
  if (grid > gg.ntiles) grid = gg.ntiles;
  const int cwords = int(sizeof(T) / 4);
  // rows that are not 16-byte multiples have no tensor map; the compute threads copy them (gg.cpa)
  constexpr bool has_producer = ws_of<R, CR, N, VAR>();
  INQB_REQUIRE(!gg.cpa || has_producer, INQB_ERR_UNSUPPORTED,
               "FFT pass rows that are not 16-byte multiples need the producer-warp kernel");
  CUtensorMap mi{}, mo{}, mx{}, mb{};
  if (gg.flat) {
    mi = flat_map(a.in, b, gg.ncols, cwords, gg.axis, W);
    mo = flat_map(a.out, b, gg.ncols, cwords, gg.axis, W);
    mx = mb = mi;
  } else if (!gg.cpa) {
    mi = orbital_map(a.in, b, a.S, cwords, gg.axis, W);
    mo = orbital_map(a.out, b, a.S, cwords, gg.axis, W);
    mx = has_aux(VAR) ? orbital_map(a.psi, b, a.S, cwords, gg.axis, W) : mi;
    mb = (has_aux(VAR) && a.hbase) ? orbital_map(a.hbase, b, a.S, cwords, gg.axis, W) : mi;
  }
  const TC *tw = reinterpret_cast<const TC *>(sizeof(CR) == 8 ? b.tw64[gg.axis] : b.tw32[gg.axis]);
  kern<<<unsigned(grid), NT, smem, ctx.stream>>>(mi, mo, mx, mb, a, gg, tw, ctx.d_err);
  INQB_CUDA(cudaGetLastError());
  ctx.launches++;
}

// The plain streaming passes of single-precision sets of at least 64 states run with 512-byte rows
// (64 states) in three stages, one CTA per SM (context option fft_wide, default 1).  Measured at
// 96^3 x 256: 0.571 ms per pass against 0.633 ms with 256-byte rows at four CTAs per SM (6.35 against
// 5.72 TB/s).  The same shape made the kinetic pass slower, and double-precision passes (32 states,
// one CTA of 256 threads per SM) much slower (1.66 against 1.15 ms), so those keep 256-byte rows.
inline bool wide_var(int var) { return var == FWD_STORE || var == INV_STORE || var == FWD_PERM || var == INV_PERM; }

template <typename R, typename CR, int N>
void launch_nc(Ctx &ctx, const Basis &b, const PassArgs<R> &a, Geom2 gg, int var, bool wide = false) {
  if constexpr (sizeof(R) == 4 && sizeof(CR) == 4) {
    // 512-byte rows (64 single-precision states) for the plain streaming passes
    if (wide) {
      switch (var) {
        case FWD_STORE: launch_kernel<R, CR, N, FWD_STORE, 1>(ctx, b, a, gg); return;
        case INV_STORE: launch_kernel<R, CR, N, INV_STORE, 1>(ctx, b, a, gg); return;
        case FWD_PERM: launch_kernel<R, CR, N, FWD_PERM, 1>(ctx, b, a, gg); return;
        case INV_PERM: launch_kernel<R, CR, N, INV_PERM, 1>(ctx, b, a, gg); return;
        default: break;
      }
    }
  }
  switch (var) {
    case FWD_STORE: launch_kernel<R, CR, N, FWD_STORE>(ctx, b, a, gg); break;
    case INV_STORE: launch_kernel<R, CR, N, INV_STORE>(ctx, b, a, gg); break;
    case MID_KIN: launch_kernel<R, CR, N, MID_KIN>(ctx, b, a, gg); break;
    case INV_FINAL: launch_kernel<R, CR, N, INV_FINAL>(ctx, b, a, gg); break;
    case FWD_VPSI: launch_kernel<R, CR, N, FWD_VPSI>(ctx, b, a, gg); break;
    case FWD_PERM:
    case INV_PERM:
    case INV_FINAL_PERM:
      // digit-reversed passes exist for equal storage and arithmetic types only
      if constexpr (sizeof(CR) == sizeof(R)) {
        if (var == FWD_PERM) launch_kernel<R, CR, N, FWD_PERM>(ctx, b, a, gg);
        else if (var == INV_PERM) launch_kernel<R, CR, N, INV_PERM>(ctx, b, a, gg);
        else launch_kernel<R, CR, N, INV_FINAL_PERM>(ctx, b, a, gg);
      } else {
        throw Error(INQB_ERR_UNSUPPORTED, "digit-reversed FFT passes need equal storage and arithmetic types");
      }
      break;
    default: launch_kernel<R, CR, N, FWD_LAPLADD>(ctx, b, a, gg); break;
  }
}

// Arithmetic of the passes over single-precision orbitals (context option mixed_compute):
//   0 single precision everywhere; 1 double precision everywhere;
//   2 double except the final (inverse, epilogue) pass of the real-space operator;
//   3 as 2 and the first forward pass (z) of every transform also single.
// whether a pass over single-precision orbitals runs single-precision arithmetic (context option mixed_compute)
template <typename R> bool single_arith(const Ctx &ctx, const PassArgs<R> &a, int var) {
  const int mode = ctx.mixed_compute;
  const int bv = base_var(var);
  return mode == 0 || (mode >= 2 && bv == INV_FINAL) || (mode == 3 && a.axis == 2 && (bv == FWD_STORE || var == FWD_VPSI));
}

template <typename R, int N>
void launch_n(Ctx &ctx, const Basis &b, const PassArgs<R> &a, Geom2 gg, int var) {
  if constexpr (sizeof(R) == 4) {
    const bool single = single_arith(ctx, a, var);
    if (single) {
      // 64-state tiles unless they would leave more of the last tile empty than 32-state tiles do
      // (85 states: 43 empty slots against 11)
      const int pad64 = (64 - a.S % 64) % 64, pad32 = (32 - a.S % 32) % 32;
      const bool wide = ctx.fft_wide && wide_var(var) && (gg.flat || (a.S >= 64 && pad64 <= pad32 + 8));
      launch_nc<R, float, N>(ctx, b, a, gg, var, wide);
      return;
    }
  }
  launch_nc<R, double, N>(ctx, b, a, gg, var);
}

// Returns false (and does nothing) when the pass is not covered by a specialised kernel.
template <typename R> bool launch(Ctx &ctx, const Basis &b, const PassArgs<R> &a, int prologue, int epilogue) {
  using T = C2<R>;
  if (ctx.fft_impl == 1) return false;
  const int n = b.n[a.axis];
  if (n != 24 && n != 32 && n != 40 && n != 48 && n != 64 && n != 72 && n != 96 && n != 120 && n != 128) return false;
  if (a.S < 256 / int(sizeof(T))) return false;  // fewer states than one 256-byte row: generic kernel
  int var;
  if (a.mid_kinetic) var = MID_KIN;
  else if (prologue == PRO_VPSI) var = FWD_VPSI;
  else if (epilogue == EPI_FINAL_REAL) var = INV_FINAL;
  else if (epilogue == EPI_LAPL_ADD) var = FWD_LAPLADD;
  else var = a.dir > 0 ? FWD_STORE : INV_STORE;
  if ((var == INV_FINAL && a.dir > 0) || ((var == FWD_VPSI || var == FWD_LAPLADD) && a.dir < 0)) return false;
  // y and x passes without per-line data over flattened columns (context option fft_flat), when the
  // rows of the flattened view are 16-byte multiples
  // (and the 32-bit words of a view row stay below 2^31, the range of a TMA coordinate).  When every tile
  // width divides the state count (a multiple of 512-byte rows) the two decompositions give the same
  // tiles, and the line tiles' per-tile index arithmetic is the cheaper (96^3 x 256 single: x pass 0.65
  // against 0.69 ms), so they are kept there.
  const long long view_words = (a.axis == 1 ? (long long)b.n[2] : (long long)b.n[1] * b.n[2]) * a.S * (sizeof(T) / 4);
  const bool flat = ctx.fft_flat && a.axis != 2 && (var == FWD_STORE || var == INV_STORE || var == MID_KIN) &&
                    (size_t(b.n[2]) * a.S * sizeof(T)) % 16 == 0 && view_words < (1LL << 31) &&
                    (size_t(a.S) * sizeof(T)) % 512 != 0;
  // rows that are not 16-byte multiples (an odd number of single-precision states): only the kernels with
  // a producer warp (single-precision arithmetic) move them, with 8-byte copies; otherwise the generic kernel
  if (!flat && (size_t(a.S) * sizeof(T)) % 16 != 0 && !(sizeof(R) == 4 && single_arith(ctx, a, var))) return false;
  if (a.perm) {
    INQB_REQUIRE(var == FWD_STORE || var == INV_STORE || var == INV_FINAL, INQB_ERR_UNSUPPORTED,
                 "digit-reversed frequency order is only kept by the plain forward and inverse passes");
    var = var == FWD_STORE ? FWD_PERM : (var == INV_STORE ? INV_PERM : INV_FINAL_PERM);
  }

  constexpr int W = 256 / int(sizeof(T));
  Geom2 gg;
  for (int i = 0; i < 3; i++) gg.g.n[i] = b.n[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) gg.g.rlat[i][j] = b.rlat[i][j];
  const long long ny = b.n[1], nz = b.n[2];
  if (a.axis == 2) { gg.g.nb = int(ny); gg.g.sa = ny * nz; gg.g.sb = nz; gg.g.sp = 1; }
  else if (a.axis == 1) { gg.g.nb = int(nz); gg.g.sa = ny * nz; gg.g.sb = 1; gg.g.sp = nz; }
  else { gg.g.nb = int(nz); gg.g.sa = nz; gg.g.sb = 1; gg.g.sp = ny * nz; }
  gg.axis = a.axis;
  gg.flat = flat ? 1 : 0;
  gg.ncols = a.axis == 1 ? nz * a.S : ny * nz * a.S;
  gg.nsb = (a.S + W - 1) / W;
  gg.ntiles = (b.npoints / n) * gg.nsb;
  gg.cwords = int(sizeof(T) / 4);
  gg.stages = 2;
  switch (n) {
    case 24: launch_n<R, 24>(ctx, b, a, gg, var); break;
    case 32: launch_n<R, 32>(ctx, b, a, gg, var); break;
    case 40: launch_n<R, 40>(ctx, b, a, gg, var); break;
    case 48: launch_n<R, 48>(ctx, b, a, gg, var); break;
    case 64: launch_n<R, 64>(ctx, b, a, gg, var); break;
    case 72: launch_n<R, 72>(ctx, b, a, gg, var); break;
    case 96: launch_n<R, 96>(ctx, b, a, gg, var); break;
    case 120: launch_n<R, 120>(ctx, b, a, gg, var); break;
    default: launch_n<R, 128>(ctx, b, a, gg, var); break;
  }
  return true;
}

}  // namespace v2
}  // namespace inqb
