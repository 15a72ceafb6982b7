// Device pieces shared by the FFT pass kernels (fft.cu, fft2.cuh): radix codelets,
// line geometry, the Laplacian factor and the per-point nonlocal term.
#pragma once

#include "inqb_internal.h"

namespace inqb {

// ------------------------------------------------------------------ radix codelets
// forward (sgn = +1) computes y_k = sum_j x_j exp(-2 pi i jk/r); backward (sgn = -1) the conjugate kernel.

template <typename T> __device__ __forceinline__ T mul_mi(T a, int sgn) {  // a * (-i*sgn)
  return sgn > 0 ? mk<T>(a.y, -a.x) : mk<T>(-a.y, a.x);
}

template <typename T> __device__ __forceinline__ void dft2(T *v) {
  T a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename T> __device__ __forceinline__ void dft4(T *v, int sgn) {
  T t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  T t2 = cadd(v[1], v[3]), t3 = mul_mi(csub(v[1], v[3]), sgn);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

template <typename T> __device__ __forceinline__ void dft8(T *v, int sgn) {
  using R = decltype(T::x);
  const R h = R(0.70710678118654752440084436210484903928);
  T e[4] = {v[0], v[2], v[4], v[6]};
  T o[4] = {v[1], v[3], v[5], v[7]};
  dft4(e, sgn);
  dft4(o, sgn);
  T w1 = sgn > 0 ? mk<T>((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h)
                 : mk<T>((o[1].x - o[1].y) * h, (o[1].y + o[1].x) * h);
  T w2 = mul_mi(o[2], sgn);
  T w3 = sgn > 0 ? mk<T>((o[3].y - o[3].x) * h, (-o[3].x - o[3].y) * h)
                 : mk<T>((-o[3].x - o[3].y) * h, (o[3].x - o[3].y) * h);
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], w1);
  v[5] = csub(e[1], w1);
  v[2] = cadd(e[2], w2);
  v[6] = csub(e[2], w2);
  v[3] = cadd(e[3], w3);
  v[7] = csub(e[3], w3);
}

// odd prime radix: y_k = x0 + sum_m [a_m cos(2pi mk/r) - i sgn b_m sin(2pi mk/r)],
// a_m = x_m + x_{r-m}, b_m = x_m - x_{r-m}
template <typename T, int RR> __device__ __forceinline__ void dft_odd(T *v, int sgn, const double *cs, const double *sn) {
  using R = decltype(T::x);
  constexpr int H = (RR - 1) / 2;
  T a[H], b[H];
#pragma unroll
  for (int m = 1; m <= H; m++) {
    a[m - 1] = cadd(v[m], v[RR - m]);
    b[m - 1] = csub(v[m], v[RR - m]);
  }
  T x0 = v[0];
  T s = x0;
#pragma unroll
  for (int m = 0; m < H; m++) s = cadd(s, a[m]);
  T y[RR];
  y[0] = s;
#pragma unroll
  for (int k = 1; k <= H; k++) {
    T re = x0, im = mk<T>(R(0), R(0));
#pragma unroll
    for (int m = 1; m <= H; m++) {
      int idx = (m * k) % RR;            // cos/sin of 2 pi idx / r, idx in [1, r-1]
      R c, sn_;
      if (idx <= H) {
        c = R(cs[idx - 1]);
        sn_ = R(sn[idx - 1]);
      } else {
        c = R(cs[RR - idx - 1]);
        sn_ = -R(sn[RR - idx - 1]);
      }
      re = cadd(re, cscale(a[m - 1], c));
      im = cadd(im, cscale(b[m - 1], sn_));
    }
    T t = mul_mi(im, sgn);               // -i sgn * sum b sin
    y[k] = cadd(re, t);
    y[RR - k] = csub(re, t);
  }
#pragma unroll
  for (int k = 0; k < RR; k++) v[k] = y[k];
}

// cos(2 pi m / r), sin(2 pi m / r) for m = 1..(r-1)/2 (values to 40 digits, rounded by the compiler)
static __device__ __constant__ double c3_cos[1] = {-0.5};
static __device__ __constant__ double c3_sin[1] = {0.86602540378443864676372317075293618347};
static __device__ __constant__ double c5_cos[2] = {0.30901699437494742410229341718281905886,
                                            -0.80901699437494742410229341718281905886};
static __device__ __constant__ double c5_sin[2] = {0.95105651629515357211643933337938214341,
                                            0.58778525229247312916870595463907276860};
static __device__ __constant__ double c7_cos[3] = {0.62348980185873353052500488400423981063,
                                            -0.22252093395631440428890256449679475947,
                                            -0.90096886790241912623610231950744505117};
static __device__ __constant__ double c7_sin[3] = {0.78183148246802980870844452667405775023,
                                            0.97492791218182360701813168299393121723,
                                            0.43388373911755812047576833284835875461};

// One Stockham radix-r pass over all lines of the tile: src/dst are [n][W] in shared memory.
template <typename T, int RR>
__device__ __forceinline__ void stockham_pass(const T *__restrict__ src, T *__restrict__ dst, int n, int W, int Ns,
                                              int sgn, const T *__restrict__ tw, int w, int jg, int njg) {
  const int nr = n / RR;
  const int tstep = n / (Ns * RR);
  for (int j = jg; j < nr; j += njg) {
    T v[RR];
#pragma unroll
    for (int q = 0; q < RR; q++) v[q] = src[(j + q * nr) * W + w];
    const int k = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int q = 1; q < RR; q++) {
        // single-precision tables interleave each twiddle's float part and remainder
        T t = __ldg(&tw[(sizeof(decltype(T::x)) == 4 ? 2 : 1) * (k * q * tstep)]);
        if (sgn < 0) t.y = -t.y;
        v[q] = cmul(v[q], t);
      }
    }
    if constexpr (RR == 2) dft2(v);
    else if constexpr (RR == 4) dft4(v, sgn);
    else if constexpr (RR == 8) dft8(v, sgn);
    else if constexpr (RR == 3) dft_odd<T, 3>(v, sgn, c3_cos, c3_sin);
    else if constexpr (RR == 5) dft_odd<T, 5>(v, sgn, c5_cos, c5_sin);
    else if constexpr (RR == 7) dft_odd<T, 7>(v, sgn, c7_cos, c7_sin);
    const int base = (j / Ns) * Ns * RR + k;
#pragma unroll
    for (int q = 0; q < RR; q++) dst[(base + q * Ns) * W + w] = v[q];
  }
}

struct Radices {
  int n;
  int count;
  int r[16];
};

// Runs all radix passes; returns the buffer holding the natural-order result.
template <typename T>
__device__ T *run_fft(T *a, T *b, const Radices &rad, int W, int sgn, const T *tw, int w, int jg, int njg) {
  int Ns = 1;
  for (int p = 0; p < rad.count; p++) {
    const int r = rad.r[p];
    switch (r) {
      case 2: stockham_pass<T, 2>(a, b, rad.n, W, Ns, sgn, tw, w, jg, njg); break;
      case 3: stockham_pass<T, 3>(a, b, rad.n, W, Ns, sgn, tw, w, jg, njg); break;
      case 4: stockham_pass<T, 4>(a, b, rad.n, W, Ns, sgn, tw, w, jg, njg); break;
      case 5: stockham_pass<T, 5>(a, b, rad.n, W, Ns, sgn, tw, w, jg, njg); break;
      case 7: stockham_pass<T, 7>(a, b, rad.n, W, Ns, sgn, tw, w, jg, njg); break;
      default: stockham_pass<T, 8>(a, b, rad.n, W, Ns, sgn, tw, w, jg, njg); break;
    }
    __syncthreads();
    T *t = a;
    a = b;
    b = t;
    Ns *= r;
  }
  return a;
}

struct Geom {
  int n[3];
  // line decomposition for this axis: line L -> (a, b), point offset = a*sa + b*sb + p*sp
  int nb;
  long long sa, sb, sp;
  double rlat[3][3];
};

__device__ __forceinline__ int sym_index(int i, int n) { return i >= (n + 1) / 2 ? i - n : i; }

__device__ __forceinline__ void line_coords(int axis, int a, int b, int p, int &ix, int &iy, int &iz) {
  if (axis == 2) { ix = a; iy = b; iz = p; }
  else if (axis == 1) { ix = a; iy = p; iz = b; }
  else { ix = p; iy = a; iz = b; }
}

// factor*(-|G|^2 + gc.G) with G = 2 pi * symmetric index (covariant), |G|^2 through the
// cell metric (fourier_space.hpp:77-125, cell.hpp:196-211).
__device__ __forceinline__ double lapl_value(const Geom &g, int ix, int iy, int iz, double factor, const double *gc) {
  const double tp = 6.283185307179586476925286766559;
  double G0 = tp * sym_index(ix, g.n[0]);
  double G1 = tp * sym_index(iy, g.n[1]);
  double G2 = tp * sym_index(iz, g.n[2]);
  double c0 = (g.rlat[0][0] * G0 + g.rlat[1][0] * G1) + g.rlat[2][0] * G2;
  double c1 = (g.rlat[0][1] * G0 + g.rlat[1][1] * G1) + g.rlat[2][1] * G2;
  double c2 = (g.rlat[0][2] * G0 + g.rlat[1][2] * G1) + g.rlat[2][2] * G2;
  double g2 = c0 * c0 + c1 * c1 + c2 * c2;
  return factor * (-g2 + (gc[0] * G0 + gc[1] * G1 + gc[2] * G2));
}

// nonlocal term at one grid point and state: sum over sphere hits h of sum_l hcoef[h][l] * projD[p][l][s]
template <typename R>
__device__ __forceinline__ C2<R> nl_term(const PassArgs<R> &a, long long pt, int s) {
  using T = C2<R>;
  T acc = mk<T>(R(0), R(0));
  const int h0 = __ldg(&a.nl_offs[pt]), h1 = __ldg(&a.nl_offs[pt + 1]);
  for (int h = h0; h < h1; h++) {
    const int p = __ldg(&a.nl_hitp[h]);
#pragma unroll
    for (int l = 0; l < 4; l++) {
      T c = a.nl_hcoef[h * 4 + l];
      T pj = a.projD[((long long)p * 4 + l) * a.S + s];
      acc = cadd(acc, cmul(c, pj));
    }
  }
  return acc;
}

}  // namespace inqb
