// Batched 1-D FFT passes over one axis of a state-fastest [nx][ny][nz][S] orbital array.
//
// A CTA owns one "tile": the n points of one grid line along the axis times W
// consecutive states.  Each of the tile's n rows is W*sizeof(complex) contiguous
// bytes (256 B for FP64 with W = 16, FP32 with W = 32), so global loads and stores
// are fully coalesced whatever the axis.  The line is transformed in shared memory
// with mixed-radix Stockham passes (radix 2,3,4,5,7,8; lanes run over states, so
// every radix-r butterfly reads and writes bank-conflict-free rows), with twiddles
// from a per-axis table exp(-2 pi i t/n) built on the host in long double.
//
// Fusions (these remove whole-array passes of the reference's operator sequence,
// ks_hamiltonian.hpp:137-180):
//   * mid_kinetic: forward transform, multiply by factor*(-|G|^2 + gc.G)
//     (laplacian.hpp:31-36), backward transform -- all in one tile visit;
//   * EPI_FINAL_REAL: out = scale*fft + (V + shift)*psi + nonlocal(psi) with the
//     nonlocal term taken from the per-grid-point hit lists (owner computes, no
//     atomics; projector_all.hpp:276-288) and the 1/N of to_real (transform.hpp:175-181);
//     optionally a Horner step of a Taylor exponential, out = base + c*out (exponential.hpp:21-34);
//   * PRO_VPSI: the tile is loaded as (V + shift)*psi + nonlocal (Fourier-form operator,
//     ks_hamiltonian.hpp:166-172);
//   * EPI_LAPL_ADD: out = fft + lapl(G)*psi_fourier (laplacian_add, laplacian.hpp:24-38).

#include "fft_common.cuh"

namespace inqb {

template <typename R, int PRO, int EPI>
__global__ void __launch_bounds__(256) fft_pass_kernel(PassArgs<R> a, Geom g, Radices rad, const C2<R> *__restrict__ tw,
                                                       int W) {
  using T = C2<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *bufA = reinterpret_cast<T *>(smem_raw);
  T *bufB = bufA + rad.n * W;

  const int nsb = (a.S + W - 1) / W;
  const long long tile = blockIdx.x;
  const long long L = tile / nsb;
  const int s0 = int(tile % nsb) * W;
  const int la = int(L / g.nb), lb = int(L % g.nb);
  const long long pbase = la * g.sa + lb * g.sb;  // point index of the line start
  const int w = threadIdx.x % W;
  const int jg = threadIdx.x / W;
  const int njg = blockDim.x / W;
  const int s = s0 + w;
  const bool active = s < a.S;
  const int n = rad.n;

  // ---- load (coalesced rows of W states)
  for (int p = jg; p < n; p += njg) {
    T v = mk<T>(R(0), R(0));
    if (active) {
      const long long pt = pbase + p * g.sp;
      const long long e = pt * a.S + s;
      v = a.in[e];
      if (PRO == PRO_VPSI) {
        R vv = a.V[pt * a.nspin + a.spin] + a.vshift;
        v = cscale(v, vv);
        if (a.nl_offs) v = cadd(v, nl_term<R>(a, pt, s));
      }
    }
    bufA[p * W + w] = v;
  }
  __syncthreads();

  T *res = run_fft<T>(bufA, bufB, rad, W, a.dir, tw, w, jg, njg);

  if (a.mid_kinetic) {
    for (int p = jg; p < n; p += njg) {
      int ix, iy, iz;
      line_coords(a.axis, la, lb, p, ix, iy, iz);
      R f = R(lapl_value(g, ix, iy, iz, a.lap_factor, a.gc));
      res[p * W + w] = cscale(res[p * W + w], f);
    }
    __syncthreads();
    T *other = (res == bufA) ? bufB : bufA;
    res = run_fft<T>(res, other, rad, W, -a.dir, tw, w, jg, njg);
  }

  // ---- store
  if (!active) return;
  for (int p = jg; p < n; p += njg) {
    const long long pt = pbase + p * g.sp;
    const long long e = pt * a.S + s;
    T v = res[p * W + w];
    if (a.scale != 1.0) v = cscale(v, R(a.scale));
    if (EPI == EPI_FINAL_REAL) {
      R vv = a.V[pt * a.nspin + a.spin] + a.vshift;
      v = cadd(v, cscale(a.psi[e], vv));
      if (a.nl_offs) v = cadd(v, nl_term<R>(a, pt, s));
    } else if (EPI == EPI_LAPL_ADD) {
      int ix, iy, iz;
      line_coords(a.axis, la, lb, p, ix, iy, iz);
      R f = R(lapl_value(g, ix, iy, iz, a.lap_factor, a.gc));
      v = cadd(v, cscale(a.psi[e], f));
    }
    if (a.hbase) v = cadd(a.hbase[e], cmul(a.hc, v));
    a.out[e] = v;
  }
}

template <typename R>
void launch_fft_pass(Ctx &ctx, const Basis &b, const PassArgs<R> &a, int prologue, int epilogue) {
  using T = C2<R>;
  if (launch_fft2<R>(ctx, b, a, prologue, epilogue)) return;
  INQB_REQUIRE(!a.perm && !a.perm_n2[1] && !a.perm_n2[2], INQB_ERR_UNSUPPORTED,
               "digit-reversed frequency order needs the specialised FFT kernel");
  const int axis = a.axis;
  Geom g;
  for (int i = 0; i < 3; i++) g.n[i] = b.n[i];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g.rlat[i][j] = b.rlat[i][j];
  const long long nx = b.n[0], ny = b.n[1], nz = b.n[2];
  if (axis == 2) { g.nb = int(ny); g.sa = ny * nz; g.sb = nz; g.sp = 1; }
  else if (axis == 1) { g.nb = int(nz); g.sa = ny * nz; g.sb = 1; g.sp = nz; }
  else { g.nb = int(nz); g.sa = nz; g.sb = 1; g.sp = ny * nz; }
  const int n = b.n[axis];
  const long long nlines = b.npoints / n;

  Radices rad;
  rad.n = n;
  rad.count = int(b.radices[axis].size());
  INQB_REQUIRE(rad.count <= 16, INQB_ERR_UNSUPPORTED, "FFT length has too many factors");
  for (int i = 0; i < rad.count; i++) rad.r[i] = b.radices[axis][i];

  // W states per tile: 256-byte rows, fewer for long lines or few states
  int W = sizeof(R) == 8 ? 16 : 32;
  while (W > 4 && size_t(2) * n * W * sizeof(T) > 160 * 1024) W /= 2;
  while (W > 4 && W / 2 >= a.S) W /= 2;
  const int njg = (n >= 8 * 8) ? 8 : 4;
  const int threads = W * njg;
  const size_t smem = size_t(2) * n * W * sizeof(T);
  INQB_REQUIRE(smem <= ctx.max_smem_optin, INQB_ERR_UNSUPPORTED, "FFT line too long for shared memory");
  const long long tiles = nlines * ((a.S + W - 1) / W);
  INQB_REQUIRE(tiles < (1LL << 31), INQB_ERR_UNSUPPORTED, "too many FFT tiles");

  const T *tw = reinterpret_cast<const T *>(sizeof(R) == 8 ? b.tw64[axis] : b.tw32[axis]);

  auto go = [&](auto kern) {
    ensure_smem_attr(reinterpret_cast<const void *>(kern), smem);
    kern<<<unsigned(tiles), threads, smem, ctx.stream>>>(a, g, rad, tw, W);
    INQB_CUDA(cudaGetLastError());
    ctx.launches++;
  };
  if (prologue == PRO_NONE && epilogue == EPI_STORE) go(fft_pass_kernel<R, PRO_NONE, EPI_STORE>);
  else if (prologue == PRO_NONE && epilogue == EPI_FINAL_REAL) go(fft_pass_kernel<R, PRO_NONE, EPI_FINAL_REAL>);
  else if (prologue == PRO_NONE && epilogue == EPI_LAPL_ADD) go(fft_pass_kernel<R, PRO_NONE, EPI_LAPL_ADD>);
  else if (prologue == PRO_VPSI && epilogue == EPI_STORE) go(fft_pass_kernel<R, PRO_VPSI, EPI_STORE>);
  else throw Error(INQB_ERR_UNSUPPORTED, "unsupported FFT pass fusion");
}

// N2 of the two-level split when the specialised TMA kernels (fft2.cuh) run every pass along `axis` for
// S states of elem_bytes each (the conditions of v2::launch), else 0.
int fft2_perm_n2(const Ctx &ctx, const Basis &b, int S, int elem_bytes, int axis) {
  if (ctx.fft_impl == 1) return 0;
  const int n = b.n[axis];
  if (n != 24 && n != 32 && n != 40 && n != 48 && n != 64 && n != 72 && n != 96 && n != 120 && n != 128) return 0;
  // rows that are not 16-byte multiples: single-precision orbitals only (the producer-warp kernels copy
  // them); the caller keeps natural order when the arithmetic is not single precision
  if ((size_t(S) * elem_bytes) % 16 != 0 && elem_bytes != 8) return 0;
  if (S < 256 / elem_bytes) return 0;
  return n / 8;
}

template void launch_fft_pass<double>(Ctx &, const Basis &, const PassArgs<double> &, int, int);
template void launch_fft_pass<float>(Ctx &, const Basis &, const PassArgs<float> &, int, int);

}  // namespace inqb
