// extern "C" entry points of libinqb200 (declared in include/inqb.h).
//
// Each entry point validates its arguments, runs the device work on the
// context's stream and converts exceptions into status codes.  The operator
// sequences follow the reference's ks_hamiltonian (ks_hamiltonian.hpp:137-180);
// the kernels they call fuse several of the reference's whole-array passes
// (fft.cu explains which).

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <numeric>

#include "inqb_internal.h"
#include "sphere.h"

using namespace inqb;

namespace {

thread_local std::string g_err_noctx;

template <typename F> int guarded(Ctx *ctx, F &&f) {
  try {
    f();
    return INQB_OK;
  } catch (const Error &e) {
    if (ctx) ctx->err = e.what();
    else g_err_noctx = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    if (ctx) ctx->err = "host allocation failed";
    return INQB_ERR_MEMORY;
  } catch (const std::exception &e) {
    if (ctx) ctx->err = e.what();
    else g_err_noctx = e.what();
    return INQB_ERR_STATE;
  }
}

void set_device(Ctx &ctx) { INQB_CUDA(cudaSetDevice(ctx.device)); }

size_t csize(int precision) { return precision == INQB_F64 ? 16 : 8; }

// cell_metric conversions for the small vectors of the operator (cell.hpp:176-211)
void cov_to_cart(const Basis &b, const double v[3], double out[3]) {
  for (int j = 0; j < 3; j++) out[j] = (b.rlat[0][j] * v[0] + b.rlat[1][j] * v[1]) + b.rlat[2][j] * v[2];
}
void cart_to_contra(const Basis &b, const double v[3], double out[3]) {
  for (int k = 0; k < 3; k++) out[k] = b.rlat[k][0] * v[0] + b.rlat[k][1] * v[1] + b.rlat[k][2] * v[2];
}
void cart_to_cov(const Basis &b, const double v[3], double out[3]) {
  for (int k = 0; k < 3; k++) out[k] = b.lat[k][0] * v[0] + b.lat[k][1] * v[1] + b.lat[k][2] * v[2];
}
void contra_to_cart(const Basis &b, const double v[3], double out[3]) {
  for (int j = 0; j < 3; j++) out[j] = (b.lat[0][j] * v[0] + b.lat[1][j] * v[1]) + b.lat[2][j] * v[2];
}
double norm_cov(const Basis &b, const double v[3]) {
  double c[3];
  cov_to_cart(b, v, c);
  return c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
}

void check_same_shape(const Orbitals &a, const Orbitals &b) {
  INQB_REQUIRE(a.basis == b.basis, INQB_ERR_ARG, "orbital sets live on different bases");
  INQB_REQUIRE(a.nst == b.nst, INQB_ERR_ARG, "orbital sets have different numbers of states");
  INQB_REQUIRE(a.precision == b.precision, INQB_ERR_ARG, "orbital sets have different precisions");
}

// ------------------------------------------------------------------ transforms

template <typename R>
void fft3d(Ctx &ctx, const Basis &b, const C2<R> *in, C2<R> *out, int S, int dir, double scale) {
  PassArgs<R> a;
  a.S = S;
  a.dir = dir;
  const int order_f[3] = {2, 1, 0};
  const int order_b[3] = {0, 1, 2};
  const int *order = dir > 0 ? order_f : order_b;
  for (int k = 0; k < 3; k++) {
    a.axis = order[k];
    a.in = (k == 0) ? in : out;
    a.out = out;
    a.scale = (k == 2) ? scale : 1.0;
    launch_fft_pass<R>(ctx, b, a, PRO_NONE, EPI_STORE);
  }
}

// ------------------------------------------------------------------ Hamiltonian pieces

template <typename R> C2<R> *proj_buf(Hamiltonian &h, int S, int which) {
  const size_t need = size_t(std::max(1, h.proj.nproj)) * 4 * S * sizeof(C2<double>);
  if (need > h.proj_bytes) {
    if (h.d_projraw) INQB_CUDA(cudaFreeAsync(h.d_projraw, h.ctx->stream));
    if (h.d_projD) INQB_CUDA(cudaFreeAsync(h.d_projD, h.ctx->stream));
    h.d_projraw = h.d_projD = nullptr;
    h.proj_bytes = 0;
    INQB_CUDA(counted_malloc_async(&h.d_projraw, need, h.ctx->stream));
    INQB_CUDA(counted_malloc_async(&h.d_projD, need, h.ctx->stream));
    h.proj_bytes = need;
  }
  return static_cast<C2<R> *>(which == 0 ? h.d_projraw : h.d_projD);
}

void ensure_tables(Hamiltonian &h, const double kA[3]) {
  if (h.proj.nproj == 0) return;
  if (h.proj.kA[0] == kA[0] && h.proj.kA[1] == kA[1] && h.proj.kA[2] == kA[2]) return;
  launch_nl_tables(*h.ctx, *h.basis, h, kA);
}

// A Horner step of a Taylor exponential fused into the operator: out = base + c (H in) instead of H in.
struct Horner {
  const void *base = nullptr;
  std::complex<double> c = 0.0;
};

template <typename R>
void apply_real(Hamiltonian &h, const Orbitals &in, Orbitals &out, const Horner &hz) {
  Ctx &ctx = *h.ctx;
  const Basis &b = *h.basis;
  const int S = in.nst;
  const C2<R> *psi = static_cast<const C2<R> *>(in.data);
  C2<R> *hpsi = static_cast<C2<R> *>(out.data);
  double kA[3] = {in.kpoint[0] + h.A[0], in.kpoint[1] + h.A[1], in.kpoint[2] + h.A[2]};

  C2<R> *projD = nullptr;
  if (h.proj.nproj > 0) {
    ensure_tables(h, kA);
    C2<R> *praw = proj_buf<R>(h, S, 0);
    projD = proj_buf<R>(h, S, 1);
    launch_nl_project<R>(ctx, b, h, psi, S, praw, projD);
  }
  double ktmp[3], kc[3];
  cov_to_cart(b, kA, ktmp);
  cart_to_contra(b, ktmp, kc);

  // The z frequencies stay in digit-reversed order between the forward z pass and the final inverse z
  // pass (the intermediate never leaves this function): the final pass, which also reads psi for the
  // V psi epilogue, then needs no transposition barrier and runs its epilogue in the last step
  // (96^3 x 256 single: 0.93 ms against 0.98 ms; 120^3: 3.6 ms against 5.1 ms).  The y passes keep
  // natural order, which measured as fast or faster.  Kept only when the specialised kernels run every
  // pass involved and every pass computes in the storage type (plain FP64, or single throughout).
  const int es = int(sizeof(C2<R>));
  const int py = 0;
  int pz = fft2_perm_n2(ctx, b, S, es, 2);
  if (!fft2_perm_n2(ctx, b, S, es, 0) || (sizeof(R) == 4 && ctx.mixed_compute != 0)) pz = 0;

  PassArgs<R> a;
  a.S = S;
  a.dir = +1;
  // forward z, y
  a.axis = 2;
  a.in = psi;
  a.out = hpsi;
  a.perm = pz ? 1 : 0;
  launch_fft_pass<R>(ctx, b, a, PRO_NONE, EPI_STORE);
  a.axis = 1;
  a.in = hpsi;
  a.perm = py ? 1 : 0;
  launch_fft_pass<R>(ctx, b, a, PRO_NONE, EPI_STORE);
  // x: forward, kinetic factor -0.5*(-|G|^2 + gc.G), gc = -2 (k+A)^contra, backward; the 1/N of the
  // inverse transform is folded into the per-point factor (formed in double, rounded once)
  a.axis = 0;
  a.perm = 0;
  a.perm_n2[1] = py;
  a.perm_n2[2] = pz;
  a.mid_kinetic = 1;
  a.lap_factor = -0.5 / double(b.npoints);
  for (int i = 0; i < 3; i++) a.gc[i] = -2.0 * kc[i];
  launch_fft_pass<R>(ctx, b, a, PRO_NONE, EPI_STORE);
  a.mid_kinetic = 0;
  a.perm_n2[1] = a.perm_n2[2] = 0;
  // backward y, then z with the real-space epilogue
  a.dir = -1;
  a.axis = 1;
  a.perm = py ? 1 : 0;
  launch_fft_pass<R>(ctx, b, a, PRO_NONE, EPI_STORE);
  a.axis = 2;
  a.perm = pz ? 1 : 0;
  a.psi = psi;
  if constexpr (sizeof(R) == 8) a.V = h.d_V;
  else a.V = h.d_V32;
  a.nspin = h.nspin;
  a.spin = in.spin_index;
  a.vshift = R(0.5 * norm_cov(b, kA));
  a.hbase = static_cast<const C2<R> *>(hz.base);
  a.hc = mk<C2<R>>(R(hz.c.real()), R(hz.c.imag()));
  launch_fft_pass<R>(ctx, b, a, PRO_NONE, EPI_FINAL_REAL);
  // nonlocal term (times the Horner coefficient in a Horner step) added at the sphere points by its own
  // kernel: as a fully occupied kernel of its own it hides the latency of the hit-table and projection
  // reads, which stall the FFT epilogue
  if (h.proj.nproj > 0) launch_nl_apply<R>(ctx, h, projD, S, hpsi, hz.base != nullptr, a.hc);
}

template <typename R> void apply_fourier(Hamiltonian &h, const Orbitals &in, Orbitals &out) {
  Ctx &ctx = *h.ctx;
  const Basis &b = *h.basis;
  const int S = in.nst;
  const C2<R> *fpsi = static_cast<const C2<R> *>(in.data);
  C2<R> *w = static_cast<C2<R> *>(out.data);
  double kA[3] = {in.kpoint[0] + h.A[0], in.kpoint[1] + h.A[1], in.kpoint[2] + h.A[2]};
  double ktmp[3], kc[3];
  cov_to_cart(b, kA, ktmp);
  cart_to_contra(b, ktmp, kc);

  // psi_rs = to_real(fpsi) in the output buffer
  fft3d<R>(ctx, b, fpsi, w, S, -1, 1.0 / double(b.npoints));
  C2<R> *projD = nullptr;
  if (h.proj.nproj > 0) {
    ensure_tables(h, kA);
    C2<R> *praw = proj_buf<R>(h, S, 0);
    projD = proj_buf<R>(h, S, 1);
    launch_nl_project<R>(ctx, b, h, w, S, praw, projD);
  }
  PassArgs<R> a;
  a.S = S;
  a.dir = +1;
  a.axis = 2;
  a.in = w;
  a.out = w;
  if constexpr (sizeof(R) == 8) a.V = h.d_V;
  else a.V = h.d_V32;
  a.nspin = h.nspin;
  a.spin = in.spin_index;
  a.vshift = R(0.5 * norm_cov(b, kA));
  if (h.proj.nproj > 0) {
    a.nl_offs = h.proj.d_offs;
    a.nl_hitp = h.proj.d_hitp;
    if constexpr (sizeof(R) == 8) a.nl_hcoef = h.proj.d_hcoef;
    else a.nl_hcoef = h.proj.d_hcoef32;
    a.projD = projD;
  }
  launch_fft_pass<R>(ctx, b, a, PRO_VPSI, EPI_STORE);
  PassArgs<R> c;
  c.S = S;
  c.dir = +1;
  c.axis = 1;
  c.in = w;
  c.out = w;
  launch_fft_pass<R>(ctx, b, c, PRO_NONE, EPI_STORE);
  c.axis = 0;
  c.psi = fpsi;
  c.lap_factor = -0.5;
  for (int i = 0; i < 3; i++) c.gc[i] = -2.0 * kc[i];
  launch_fft_pass<R>(ctx, b, c, PRO_NONE, EPI_LAPL_ADD);
}

// The options that choose kernels and their shapes, settable on a context and overridable per
// Hamiltonian (inqb_hamiltonian_set_option); nullptr for other keys.
int *kernel_option(Ctx &ctx, const std::string &k) {
  if (k == "fft_impl") return &ctx.fft_impl;
  if (k == "fft_stages") return &ctx.fft_stages;
  if (k == "fft_wide") return &ctx.fft_wide;
  if (k == "fft_flat") return &ctx.fft_flat;
  if (k == "nl_bulk") return &ctx.nl_bulk;
  if (k == "nl_apply_points") return &ctx.nl_apply_points;
  if (k == "nl_project_points") return &ctx.nl_project_points;
  if (k == "nl_project_ranges") return &ctx.nl_project_ranges;
  if (k == "grid_sms") return &ctx.num_sms;
  return nullptr;
}
void check_kernel_option(const Ctx &ctx, const std::string &k, long long value) {
  if (k == "grid_sms")
    INQB_REQUIRE(value >= 0 && value <= ctx.device_sms, INQB_ERR_ARG,
                 "grid_sms is 0 (every SM) or 1.." + std::to_string(ctx.device_sms));
  if (k == "fft_impl") INQB_REQUIRE(value == 0 || value == 1, INQB_ERR_ARG, "fft_impl is 0 (specialised) or 1 (generic)");
  if (k == "fft_stages") INQB_REQUIRE(value >= 0 && value <= 8, INQB_ERR_ARG, "fft_stages is 0 (automatic) or 1..8");
  if (k == "fft_wide") INQB_REQUIRE(value == 0 || value == 1, INQB_ERR_ARG, "fft_wide is 0 (256-byte rows) or 1 (512-byte rows)");
  if (k == "fft_flat")
    INQB_REQUIRE(value == 0 || value == 1, INQB_ERR_ARG, "fft_flat is 0 (line x state-block tiles) or 1 (flattened columns)");
  if (k == "nl_bulk")
    INQB_REQUIRE(value >= -1 && value <= 1, INQB_ERR_ARG, "nl_bulk is 0 (automatic), 1 (always) or -1 (never)");
  if (k == "nl_apply_points" || k == "nl_project_points")
    INQB_REQUIRE(value >= 0 && value <= 32, INQB_ERR_ARG, k + " is 0 (automatic) or 1..32");
  if (k == "nl_project_ranges")
    INQB_REQUIRE(value >= 0 && value <= 64, INQB_ERR_ARG, "nl_project_ranges is 0 (16) or 1..64");
}

// The Hamiltonian's kernel-option overrides (inqb_hamiltonian_set_option) in force on its context for
// the lifetime of the scope: every launch of an operator application reads them.
struct OptionScope {
  Ctx &ctx;
  std::vector<std::pair<int *, int>> saved;
  explicit OptionScope(Hamiltonian &h) : ctx(*h.ctx) {
    for (const auto &kv : h.opt_overrides) {
      int *f = kernel_option(ctx, kv.first);
      saved.emplace_back(f, *f);
      *f = kv.second;
    }
  }
  ~OptionScope() {
    for (auto it = saved.rbegin(); it != saved.rend(); ++it) *it->first = it->second;
  }
};

void apply_any(Hamiltonian &h, const Orbitals &in, Orbitals &out, const Horner &hz = Horner()) {
  OptionScope scope(h);
  check_same_shape(in, out);
  INQB_REQUIRE(in.basis == h.basis, INQB_ERR_ARG, "orbitals and Hamiltonian live on different bases");
  INQB_REQUIRE(in.data != out.data, INQB_ERR_ARG, "H|psi> needs distinct input and output sets");
  INQB_REQUIRE(in.spin_index >= 0 && in.spin_index < h.nspin, INQB_ERR_ARG, "spin index out of range");
  if (in.space == INQB_REAL_SPACE) {
    INQB_REQUIRE(hz.base == nullptr || hz.base != out.data, INQB_ERR_ARG,
                 "the base of a Horner step must be distinct from the operator's output");
    if (in.precision == INQB_F64) apply_real<double>(h, in, out, hz);
    else apply_real<float>(h, in, out, hz);
  } else {
    INQB_REQUIRE(hz.base == nullptr, INQB_ERR_UNSUPPORTED, "Taylor exponentials are implemented for real-space sets");
    if (in.precision == INQB_F64) apply_fourier<double>(h, in, out);
    else apply_fourier<float>(h, in, out);
  }
  out.space = in.space;
  for (int i = 0; i < 3; i++) out.kpoint[i] = in.kpoint[i];
  out.spin_index = in.spin_index;
}

// scratch orbital set with the shape of `like`
struct TempSet {
  Orbitals o;
  Ctx *ctx;
  explicit TempSet(const Orbitals &like) : o(like), ctx(like.ctx) { o.data = dev_alloc(*ctx, like.bytes()); }
  ~TempSet() {
    if (o.data) cudaFreeAsync(o.data, ctx->stream);
  }
  TempSet(const TempSet &) = delete;
  TempSet &operator=(const TempSet &) = delete;
};

void copy_set(const Orbitals &src, Orbitals &dst) {
  check_same_shape(src, dst);
  INQB_CUDA(cudaMemcpyAsync(dst.data, src.data, src.bytes(), cudaMemcpyDeviceToDevice, src.ctx->stream));
  dst.space = src.space;
}

// out = exp(f H) base to the given Taylor order (exponential.hpp:21-34), in Horner form: w_1 = base +
// (f / order) H base, w_k = base + (f / (order - k + 1)) H w_{k-1}, out = w_order -- the same polynomial
// in H as the reference's sum of f^n H^n base / n!, with each step fused into the epilogues of its H
// application (the final FFT pass reads the base as a third tile, the nonlocal apply scales its term).
// base must differ from out; one scratch set.
void exponential_from(Hamiltonian &h, std::complex<double> f, const Orbitals &base, Orbitals &out, int order) {
  INQB_REQUIRE(order >= 1, INQB_ERR_ARG, "order must be >= 1");
  INQB_REQUIRE(base.space == INQB_REAL_SPACE, INQB_ERR_UNSUPPORTED, "exponential is implemented for real-space sets");
  INQB_REQUIRE(base.data != out.data, INQB_ERR_ARG, "exponential_from needs distinct base and output sets");
  check_same_shape(base, out);
  std::unique_ptr<TempSet> t;
  if (order > 1) t.reset(new TempSet(base));
  const Orbitals *src = &base;
  for (int k = 1; k <= order; k++) {
    Orbitals *dst = ((order - k) % 2 == 0) ? &out : &t->o;  // the last step writes out
    Horner hz;
    hz.base = base.data;
    hz.c = f / double(order - k + 1);
    apply_any(h, *src, *dst, hz);
    src = dst;
  }
  out.space = base.space;
  for (int i = 0; i < 3; i++) out.kpoint[i] = base.kpoint[i];
  out.spin_index = base.spin_index;
}

// exponential_in_place (exponential.hpp:21-34): phi <- exp(f H) phi
void exponential_in_place(Hamiltonian &h, std::complex<double> f, Orbitals &phi, int order) {
  TempSet base(phi);
  copy_set(phi, base.o);
  exponential_from(h, f, base.o, phi, order);
}

// exponential_2_for_1 (exponential.hpp:50-69): exp1 <- exp(f1 H) phi, phi <- exp(f2 H) phi from one set of
// H^n phi.  The terms u_n = H^n phi are kept, and one element-wise pass forms both sums, adding the terms
// in the reference's order; with the sums in the H epilogues instead, every term would cost two more
// reads and writes of a set per accumulator.  Holds `order` scratch sets.
void exponential_2_for_1(Hamiltonian &h, std::complex<double> f1, std::complex<double> f2, Orbitals &phi,
                         Orbitals &exp1, int order) {
  INQB_REQUIRE(order >= 1 && order <= 8, INQB_ERR_ARG, "order must be 1..8");
  INQB_REQUIRE(phi.space == INQB_REAL_SPACE, INQB_ERR_UNSUPPORTED, "exponential is implemented for real-space sets");
  check_same_shape(phi, exp1);
  std::vector<std::unique_ptr<TempSet>> u;
  const Orbitals *src = &phi;
  double2 c1[8], c2[8];
  std::complex<double> k1 = 1.0, k2 = 1.0;
  for (int n = 1; n <= order; n++) {
    u.emplace_back(new TempSet(phi));
    apply_any(h, *src, u.back()->o);
    src = &u.back()->o;
    k1 *= f1 / double(n);
    k2 *= f2 / double(n);
    c1[n - 1] = make_double2(k1.real(), k1.imag());
    c2[n - 1] = make_double2(k2.real(), k2.imag());
  }
  Ctx &ctx = *phi.ctx;
  const long long n = phi.basis->npoints * phi.nst;
  if (phi.precision == INQB_F64) {
    const double2 *up[8];
    for (int k = 0; k < order; k++) up[k] = static_cast<const double2 *>(u[k]->o.data);
    launch_taylor_combine<double>(ctx, static_cast<const double2 *>(phi.data), up, order, c1, c2,
                                  static_cast<double2 *>(exp1.data), static_cast<double2 *>(phi.data), n);
  } else {
    const float2 *up[8];
    for (int k = 0; k < order; k++) up[k] = static_cast<const float2 *>(u[k]->o.data);
    launch_taylor_combine<float>(ctx, static_cast<const float2 *>(phi.data), up, order, c1, c2,
                                 static_cast<float2 *>(exp1.data), static_cast<float2 *>(phi.data), n);
  }
  exp1.space = phi.space;
  for (int i = 0; i < 3; i++) exp1.kpoint[i] = phi.kpoint[i];
  exp1.spin_index = phi.spin_index;
}

template <typename R> double *occ_to_device(Ctx &ctx, const double *occ, int S) {
  double *d = static_cast<double *>(dev_alloc(ctx, sizeof(double) * S));
  INQB_CUDA(cudaMemcpyAsync(d, occ, sizeof(double) * S, cudaMemcpyHostToDevice, ctx.stream));
  return d;
}

// self_consistency::update_hamiltonian (self_consistency.hpp:88-170), unpolarised, static ions, no
// external fields: V = V_ion + V_H[n] + V_xc[n] from a device density, left in the Hamiltonian's
// potential; energies (if given) = {external, Hartree, xc, int n v_xc}.
void update_hamiltonian_dev(Hamiltonian &h, const double *d_dens, double *energies) {
  Ctx &ctx = *h.ctx;
  const Basis &b = *h.basis;
  INQB_REQUIRE(h.d_vion, INQB_ERR_ARG, "the Hamiltonian has no interaction (inqb_hamiltonian_set_interaction)");
  INQB_REQUIRE(h.nspin == 1, INQB_ERR_UNSUPPORTED, "the interacting update is implemented for one spin channel");
  double2 *vh = nullptr;
  if (h.hartree) {
    // solvers::poisson::solve (poisson.hpp:98-104): forward transform, 4 pi / |G|^2, unnormalised backward
    vh = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * b.npoints));
    launch_real_to_complex(ctx, d_dens, vh, b.npoints);
    fft3d<double>(ctx, b, vh, vh, 1, +1, 1.0);
    launch_poisson_factor(ctx, b, vh);
    fft3d<double>(ctx, b, vh, vh, 1, -1, 1.0);
  }
  double *partial = static_cast<double *>(dev_alloc(ctx, sizeof(double) * KS_BLOCKS * 4));
  launch_ks_potential(ctx, d_dens, h.d_vion, vh, h.xc, b.npoints, h.d_V, h.d_V32, partial);
  if (energies) {
    std::vector<double> hp(size_t(KS_BLOCKS) * 4);
    INQB_CUDA(cudaMemcpyAsync(hp.data(), partial, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, ctx.stream));
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
    double e[4] = {0.0, 0.0, 0.0, 0.0};
    for (int blk = 0; blk < KS_BLOCKS; blk++)
      for (int k = 0; k < 4; k++) e[k] += hp[size_t(blk) * 4 + k];
    const double dv = b.volume / double(b.npoints);
    energies[0] = dv * e[0];
    energies[1] = h.hartree ? 0.5 * dv * e[1] : 0.0;
    energies[2] = h.xc ? dv * e[2] : 0.0;
    energies[3] = h.xc ? dv * e[3] : 0.0;
  }
  dev_free(ctx, partial);
  if (vh) dev_free(ctx, vh);
}

void density_dev(Ctx &ctx, inqb_orbitals *const *phis, int nsets, const double *const *occ, double *dens) {
  for (int k = 0; k < nsets; k++) {
    const Orbitals &o = *phis[k];
    double *docc = static_cast<double *>(dev_alloc(ctx, sizeof(double) * o.nst));
    INQB_CUDA(cudaMemcpyAsync(docc, occ[k], sizeof(double) * o.nst, cudaMemcpyHostToDevice, ctx.stream));
    if (o.precision == INQB_F64)
      launch_density<double>(ctx, static_cast<const double2 *>(o.data), o.nst, o.basis->npoints, docc, dens, k > 0);
    else
      launch_density<float>(ctx, static_cast<const float2 *>(o.data), o.nst, o.basis->npoints, docc, dens, k > 0);
    dev_free(ctx, docc);
  }
}

void dipole_host(const Basis &b, const double *dens, double out[3]) {
  double acc[3] = {0, 0, 0};
  const int nx = b.n[0], ny = b.n[1], nz = b.n[2];
  long long pt = 0;
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny; iy++)
      for (int iz = 0; iz < nz; iz++, pt++) {
        const int s[3] = {ix >= (nx + 1) / 2 ? ix - nx : ix, iy >= (ny + 1) / 2 ? iy - ny : iy,
                          iz >= (nz + 1) / 2 ? iz - nz : iz};
        const double c[3] = {s[0] * (1.0 / nx), s[1] * (1.0 / ny), s[2] * (1.0 / nz)};
        double r[3];
        contra_to_cart(b, c, r);
        for (int j = 0; j < 3; j++) acc[j] += r[j] * dens[pt];
      }
  const double dv = b.volume / double(b.npoints);
  for (int j = 0; j < 3; j++) out[j] = dv * acc[j];
}

// Cholesky S = U^H U (upper, matrix/cholesky.hpp:28-89) and U^{-1} (invert_triangular.hpp:20-60), host FP64.
void cholesky_inverse(int n, const std::complex<double> *S, std::complex<double> *X) {
  std::vector<std::complex<double>> U(size_t(n) * n, 0.0);
  for (int j = 0; j < n; j++) {
    double d = S[size_t(j) * n + j].real();
    for (int k = 0; k < j; k++) d -= std::norm(U[size_t(k) * n + j]);
    INQB_REQUIRE(d > 0.0, INQB_ERR_NUMERIC, "overlap matrix is not positive definite (orthogonalize)");
    const double ujj = std::sqrt(d);
    U[size_t(j) * n + j] = ujj;
    for (int i = j + 1; i < n; i++) {
      std::complex<double> v = S[size_t(j) * n + i];
      for (int k = 0; k < j; k++) v -= std::conj(U[size_t(k) * n + j]) * U[size_t(k) * n + i];
      U[size_t(j) * n + i] = v / ujj;
    }
  }
  std::fill(X, X + size_t(n) * n, std::complex<double>(0.0));
  for (int i = 0; i < n; i++) {
    X[size_t(i) * n + i] = 1.0 / U[size_t(i) * n + i];
    for (int j = i + 1; j < n; j++) {
      std::complex<double> s = 0.0;
      for (int k = i; k < j; k++) s += X[size_t(i) * n + k] * U[size_t(k) * n + j];
      X[size_t(i) * n + j] = -s / U[size_t(j) * n + j];
    }
  }
}

// Eigen-decomposition of a Hermitian matrix (matrix::diagonalize, diagonalize.hpp:100-190) by cyclic
// Jacobi rotations in FP64.  A is [n][n] row-major and read from its upper triangle (the reference
// passes "U" to zheev / Zheevd); on return w holds the eigenvalues in ascending order and column k of
// the row-major V the eigenvector of w[k].
void hermitian_eigen(int n, const std::complex<double> *Ain, double *w, std::complex<double> *V) {
  using cd = std::complex<double>;
  std::vector<cd> A(size_t(n) * n);
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) {
      A[size_t(i) * n + j] = Ain[size_t(i) * n + j];
      A[size_t(j) * n + i] = std::conj(Ain[size_t(i) * n + j]);
    }
  for (int i = 0; i < n; i++) A[size_t(i) * n + i] = A[size_t(i) * n + i].real();
  std::vector<cd> Vm(size_t(n) * n, 0.0);
  for (int i = 0; i < n; i++) Vm[size_t(i) * n + i] = 1.0;
  auto off = [&] {
    double s = 0.0;
    for (int i = 0; i < n; i++)
      for (int j = i + 1; j < n; j++) s += std::norm(A[size_t(i) * n + j]);
    return s;
  };
  double total = 0.0;
  for (auto &x : A) total += std::norm(x);
  for (int sweep = 0; sweep < 60 && off() > 1e-30 * total; sweep++) {
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const cd b = A[size_t(p) * n + q];
        const double r = std::abs(b);
        if (r < 1e-300) continue;
        const double a = A[size_t(p) * n + p].real(), d = A[size_t(q) * n + q].real();
        const cd ph = b / r;  // e^{i phi}
        // real rotation zeroing [[a, r], [r, d]]
        const double theta = 0.5 * std::atan2(2.0 * r, d - a);
        const double c = std::cos(theta), sn = std::sin(theta);
        // U = diag(1, conj(ph)) * [[c, s], [-s, c]]: columns p, q
        const cd upp = c, upq = sn, uqp = -sn * std::conj(ph), uqq = c * std::conj(ph);
        for (int k = 0; k < n; k++) {  // A <- A U
          const cd akp = A[size_t(k) * n + p], akq = A[size_t(k) * n + q];
          A[size_t(k) * n + p] = akp * upp + akq * uqp;
          A[size_t(k) * n + q] = akp * upq + akq * uqq;
        }
        for (int k = 0; k < n; k++) {  // A <- U^H A
          const cd apk = A[size_t(p) * n + k], aqk = A[size_t(q) * n + k];
          A[size_t(p) * n + k] = std::conj(upp) * apk + std::conj(uqp) * aqk;
          A[size_t(q) * n + k] = std::conj(upq) * apk + std::conj(uqq) * aqk;
        }
        A[size_t(p) * n + q] = 0.0;
        A[size_t(q) * n + p] = 0.0;
        A[size_t(p) * n + p] = A[size_t(p) * n + p].real();
        A[size_t(q) * n + q] = A[size_t(q) * n + q].real();
        for (int k = 0; k < n; k++) {  // V <- V U
          const cd vkp = Vm[size_t(k) * n + p], vkq = Vm[size_t(k) * n + q];
          Vm[size_t(k) * n + p] = vkp * upp + vkq * uqp;
          Vm[size_t(k) * n + q] = vkp * upq + vkq * uqq;
        }
      }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return A[size_t(x) * n + x].real() < A[size_t(y) * n + y].real(); });
  for (int k = 0; k < n; k++) {
    w[k] = A[size_t(order[k]) * n + order[k]].real();
    for (int i = 0; i < n; i++) V[size_t(i) * n + k] = Vm[size_t(i) * n + order[k]];
  }
}

void overlap_dev(const Orbitals &a, const Orbitals &b, double2 *out_dev) {
  Ctx &ctx = *a.ctx;
  INQB_REQUIRE(a.basis == b.basis && a.precision == b.precision, INQB_ERR_ARG, "overlap of incompatible sets");
  INQB_REQUIRE(a.space == b.space, INQB_ERR_ARG, "overlap of sets in different spaces");
  const double dv = set_volume_element(a);
  if (a.precision == INQB_F64)
    launch_overlap<double>(ctx, static_cast<const double2 *>(a.data), a.nst, static_cast<const double2 *>(b.data),
                           b.nst, a.basis->npoints, dv, out_dev);
  else if (ctx.overlap_tc)
    launch_overlap_tc(ctx, static_cast<const float2 *>(a.data), a.nst, static_cast<const float2 *>(b.data), b.nst,
                      a.basis->npoints, dv, out_dev);
  else
    launch_overlap<float>(ctx, static_cast<const float2 *>(a.data), a.nst, static_cast<const float2 *>(b.data), b.nst,
                          a.basis->npoints, dv, out_dev);
}

void ovdiag_dev(const Orbitals &a, const Orbitals &b, double2 *out_dev) {
  check_same_shape(a, b);
  Ctx &ctx = *a.ctx;
  const double dv = set_volume_element(a);
  if (a.precision == INQB_F64)
    launch_overlap_diag<double>(ctx, static_cast<const double2 *>(a.data), static_cast<const double2 *>(b.data), a.nst,
                                a.basis->npoints, dv, out_dev);
  else
    launch_overlap_diag<float>(ctx, static_cast<const float2 *>(a.data), static_cast<const float2 *>(b.data), a.nst,
                               a.basis->npoints, dv, out_dev);
}

void rotate_dev(Orbitals &phi, const double2 *Rdev) {
  if (phi.precision == INQB_F64)
    launch_rotate<double>(*phi.ctx, static_cast<double2 *>(phi.data), phi.nst, phi.basis->npoints, Rdev);
  else
    launch_rotate<float>(*phi.ctx, static_cast<float2 *>(phi.data), phi.nst, phi.basis->npoints, Rdev);
}

template <typename T> std::vector<T> download(Ctx &ctx, const void *dev, size_t n) {
  std::vector<T> h(n);
  INQB_CUDA(cudaMemcpyAsync(h.data(), dev, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx.stream));
  INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  return h;
}

}  // namespace

// all device memory of the library is stream-ordered (cudaMallocAsync / cudaFreeAsync on the owning
// context's stream): releasing an object never synchronises the device, so contexts driven by
// different host threads (the serving slots) do not stall one another
void inqb::free_projectors(Projectors &P, cudaStream_t st) {
  void *ptrs[] = {P.d_pt, P.d_pos, P.d_mat, P.d_coeff, P.d_coeff32, P.d_npts, P.d_offs, P.d_hit, P.d_hitpts, P.d_hitp,
                  P.d_hrec, P.d_gcoef, P.d_hcoef, P.d_gcoef32, P.d_hcoef32};
  for (void *p : ptrs)
    if (p) cudaFreeAsync(p, st);
  P = Projectors();
}

namespace {

// the caller synchronises the stream before the host vector goes away
template <typename T> T *upload_vec(const std::vector<T> &v, cudaStream_t st) {
  T *d = nullptr;
  const size_t bytes = std::max<size_t>(sizeof(T), v.size() * sizeof(T));
  INQB_CUDA(counted_malloc_async(&d, bytes, st));
  if (!v.empty()) INQB_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return d;
}

// projector_all packing (projector_all.hpp:40-109) + per-grid-point hit lists for the owner-computes scatter
void set_projectors(Hamiltonian &h, int nproj, int maxsph, int maxnlm, const int32_t *points, const float *pos,
                    const double *matrices, const double *coeff, const int32_t *npts, const int32_t *nlm) {
  const Basis &b = *h.basis;
  INQB_REQUIRE(nproj >= 0 && maxsph >= 0, INQB_ERR_ARG, "negative projector table size");
  INQB_REQUIRE(maxnlm >= 0 && maxnlm <= 4, INQB_ERR_UNSUPPORTED, "at most 4 (l <= 1) projector functions per atom");
  cudaStream_t st = h.ctx->stream;
  free_projectors(h.proj, st);
  Projectors &P = h.proj;
  P.nproj = nproj;
  P.maxsph = maxsph;
  P.maxnlm = maxnlm;
  if (nproj == 0) return;
  P.h_points.assign(points, points + size_t(nproj) * maxsph * 3);
  P.h_pos.assign(pos, pos + size_t(nproj) * maxsph * 3);
  P.h_mat.assign(matrices, matrices + size_t(nproj) * maxnlm * maxsph);
  P.h_coeff.assign(coeff, coeff + size_t(nproj) * maxnlm * maxnlm);
  P.h_npts.assign(npts, npts + nproj);
  P.h_nlm.assign(nlm, nlm + nproj);

  std::vector<int> flat(size_t(nproj) * maxsph, -1);
  std::vector<double> mat4(size_t(nproj) * 4 * maxsph, 0.0);
  std::vector<double> coeff4(size_t(nproj) * 16, 0.0);
  std::vector<float> coeff4f(size_t(nproj) * 16, 0.0f);
  std::vector<std::pair<long long, int>> hits;  // (grid point, p*maxsph + i)
  for (int p = 0; p < nproj; p++) {
    INQB_REQUIRE(npts[p] >= 0 && npts[p] <= maxsph, INQB_ERR_ARG, "sphere size out of range");
    INQB_REQUIRE(nlm[p] >= 0 && nlm[p] <= maxnlm, INQB_ERR_ARG, "nlm out of range");
    for (int i = 0; i < npts[p]; i++) {
      const int32_t *g = points + (size_t(p) * maxsph + i) * 3;
      INQB_REQUIRE(g[0] >= 0 && g[0] < b.n[0] && g[1] >= 0 && g[1] < b.n[1] && g[2] >= 0 && g[2] < b.n[2],
                   INQB_ERR_ARG, "projector point outside the grid");
      const long long pt = (static_cast<long long>(g[0]) * b.n[1] + g[1]) * b.n[2] + g[2];
      flat[size_t(p) * maxsph + i] = int(pt);
      hits.push_back({pt, p * maxsph + i});
    }
    for (int l = 0; l < nlm[p]; l++)
      for (int i = 0; i < npts[p]; i++)
        mat4[(size_t(p) * 4 + l) * maxsph + i] = matrices[(size_t(p) * maxnlm + l) * maxsph + i];
    for (int l = 0; l < nlm[p]; l++)
      for (int j = 0; j < nlm[p]; j++) {
        coeff4[p * 16 + l * 4 + j] = coeff[(size_t(p) * maxnlm + l) * maxnlm + j];
        coeff4f[p * 16 + l * 4 + j] = float(coeff4[p * 16 + l * 4 + j]);
      }
  }
  std::stable_sort(hits.begin(), hits.end(),
                   [](const std::pair<long long, int> &x, const std::pair<long long, int> &y) { return x.first < y.first; });
  P.total = (long long)hits.size();
  INQB_REQUIRE(P.total < (1LL << 31), INQB_ERR_UNSUPPORTED, "too many sphere points");
  std::vector<int> offs(size_t(b.npoints) + 1, 0);
  std::vector<int> hit(hits.size());
  for (size_t k = 0; k < hits.size(); k++) {
    offs[size_t(hits[k].first) + 1]++;
    hit[k] = hits[k].second;
  }
  for (long long i = 0; i < b.npoints; i++) offs[size_t(i) + 1] += offs[size_t(i)];
  std::vector<int> hitp(hits.size());
  for (size_t k = 0; k < hits.size(); k++) hitp[k] = hits[k].second / maxsph;
  std::vector<int> hitpts;
  for (size_t k = 0; k < hits.size(); k++)
    if (k == 0 || hits[k].first != hits[k - 1].first) hitpts.push_back(int(hits[k].first));
  P.nhitpts = (long long)hitpts.size();
  // one record per hit point: (point, first hit, hit count, projector of the first hit)
  std::vector<int4> hrec(hitpts.size());
  for (size_t r = 0; r < hitpts.size(); r++) {
    const int pt = hitpts[r], h0 = offs[size_t(pt)];
    hrec[r] = make_int4(pt, h0, offs[size_t(pt) + 1] - h0, hitp[size_t(h0)]);
  }

  P.d_pt = upload_vec(flat, st);
  P.d_pos = upload_vec(P.h_pos, st);
  P.d_mat = upload_vec(mat4, st);
  P.d_coeff = upload_vec(coeff4, st);
  P.d_coeff32 = upload_vec(coeff4f, st);
  P.d_npts = upload_vec(P.h_npts, st);
  P.d_offs = upload_vec(offs, st);
  P.d_hit = upload_vec(hit, st);
  P.d_hitpts = upload_vec(hitpts, st);
  P.d_hitp = upload_vec(hitp, st);
  P.d_hrec = upload_vec(hrec, st);
  INQB_CUDA(counted_malloc_async(&P.d_gcoef, sizeof(double2) * std::max<size_t>(1, size_t(nproj) * maxsph * 4), st));
  INQB_CUDA(counted_malloc_async(&P.d_gcoef32, sizeof(float2) * std::max<size_t>(1, size_t(nproj) * maxsph * 4), st));
  INQB_CUDA(counted_malloc_async(&P.d_hcoef, sizeof(double2) * std::max<size_t>(1, size_t(P.total) * 4), st));
  INQB_CUDA(counted_malloc_async(&P.d_hcoef32, sizeof(float2) * std::max<size_t>(1, size_t(P.total) * 4), st));
  INQB_CUDA(cudaStreamSynchronize(st));  // the host tables above go out of scope
  P.kA[0] = P.kA[1] = P.kA[2] = 1e300;  // tables are built on first use for a given k + A
}

}  // namespace

// ------------------------------------------------------------------ restart files (operations/io.hpp)

// utils::num_to_str (utils/num_str.hpp:16-20): ten digits, zero padded
std::string num10(long n) {
  char b[16];
  std::snprintf(b, sizeof(b), "%010ld", n);
  return std::string(b);
}

void write_file(const std::string &name, const void *data, size_t bytes) {
  std::ofstream f(name, std::ios::binary | std::ios::trunc);
  INQB_REQUIRE(f.good(), INQB_ERR_ARG, "cannot create restart file '" + name + "'");
  f.write(static_cast<const char *>(data), std::streamsize(bytes));
  INQB_REQUIRE(f.good(), INQB_ERR_ARG, "cannot write restart file '" + name + "'");
}

void read_file(const std::string &name, void *data, size_t bytes) {
  std::ifstream f(name, std::ios::binary);
  INQB_REQUIRE(f.good(), INQB_ERR_ARG, "cannot open restart file '" + name + "'");
  f.read(static_cast<char *>(data), std::streamsize(bytes));
  INQB_REQUIRE(size_t(f.gcount()) == bytes, INQB_ERR_ARG, "restart file '" + name + "' is too short");
}

// states of a set through contiguous complex128 rows, a block of states at a time (about 256 MB)
template <typename R> void save_states(const Orbitals &phi, const std::string &dir) {
  Ctx &ctx = *phi.ctx;
  const long long np = phi.basis->npoints;
  const int S = phi.nst;
  const int blk = int(std::max<long long>(1, std::min<long long>(S, (256LL << 20) / (np * 16))));
  double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * size_t(np) * blk));
  std::vector<double2> h(size_t(np) * blk);
  for (int s0 = 0; s0 < S; s0 += blk) {
    const int ns = std::min(blk, S - s0);
    launch_extract_states<R>(ctx, static_cast<const C2<R> *>(phi.data), S, np, s0, ns, d);
    INQB_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double2) * size_t(np) * ns, cudaMemcpyDeviceToHost, ctx.stream));
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
    for (int k = 0; k < ns; k++)
      write_file(dir + "/" + num10(s0 + k) + "_" + num10(0), h.data() + size_t(k) * np, sizeof(double2) * size_t(np));
  }
  dev_free(ctx, d);
}

template <typename R> void load_states(Orbitals &phi, const std::string &dir) {
  Ctx &ctx = *phi.ctx;
  const long long np = phi.basis->npoints;
  const int S = phi.nst;
  const int blk = int(std::max<long long>(1, std::min<long long>(S, (256LL << 20) / (np * 16))));
  double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * size_t(np) * blk));
  std::vector<double2> h(size_t(np) * blk);
  for (int s0 = 0; s0 < S; s0 += blk) {
    const int ns = std::min(blk, S - s0);
    for (int k = 0; k < ns; k++)
      read_file(dir + "/" + num10(s0 + k) + "_" + num10(0), h.data() + size_t(k) * np, sizeof(double2) * size_t(np));
    INQB_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(double2) * size_t(np) * ns, cudaMemcpyHostToDevice, ctx.stream));
    launch_insert_states<R>(ctx, d, S, np, s0, ns, static_cast<C2<R> *>(phi.data));
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));  // the host block is refilled next
  }
  dev_free(ctx, d);
}

// ============================================================================ C ABI

// operations::orthogonalize (orthogonalize.hpp:25-31)
void orthogonalize_dev(Orbitals &phi) {
  Ctx &ctx = *phi.ctx;
  const int S = phi.nst;
  double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * S * S));
  overlap_dev(phi, phi, d);
  auto Sh = download<std::complex<double>>(ctx, d, size_t(S) * S);
  std::vector<std::complex<double>> X(size_t(S) * S);
  cholesky_inverse(S, Sh.data(), X.data());
  INQB_CUDA(cudaMemcpyAsync(d, X.data(), sizeof(double2) * S * S, cudaMemcpyHostToDevice, ctx.stream));
  rotate_dev(phi, d);
  dev_free(ctx, d);
  INQB_CUDA(cudaStreamSynchronize(ctx.stream));
}

// eigensolvers::steepest_descent (steepest_descent.hpp:23-86) with the Teter-Payne-Allan preconditioner
// (preconditioner.hpp:24-46) on a Fourier-space set: five line-minimisation steps per state along the
// preconditioned residual, then orthogonalize.  The per-state overlaps are FP64 reductions; the step
// lengths are formed on the host.
template <typename R> void steepest_descent_t(Hamiltonian &h, Orbitals &phi) {
  Ctx &ctx = *h.ctx;
  const Basis &b = *h.basis;
  const int S = phi.nst;
  const long long np = b.npoints;
  using T = C2<R>;
  constexpr int num_steps = 5;
  TempSet hphi(phi), res(phi), hres(phi), lap(phi);
  auto D = [](Orbitals &o) { return static_cast<T *>(o.data); };
  auto CD = [](const Orbitals &o) { return static_cast<const T *>(o.data); };
  double2 *dov = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * S));
  double2 *dcoef = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * S));
  double *dkin = static_cast<double *>(dev_alloc(ctx, sizeof(double) * S));
  auto ovd = [&](const Orbitals &x, const Orbitals &y) {
    ovdiag_dev(x, y, dov);
    return download<std::complex<double>>(ctx, dov, size_t(S));
  };
  apply_any(h, phi, hphi.o);
  std::vector<double2> coef(S);
  std::vector<double> kin(S);
  const double zero[3] = {0.0, 0.0, 0.0};
  for (int istep = 0; istep < num_steps; istep++) {
    copy_set(hphi.o, res.o);
    const auto ev = ovd(res.o, phi);
    const auto nrm = ovd(phi, phi);
    for (int s = 0; s < S; s++) {
      const std::complex<double> e = ev[s] / nrm[s].real();
      coef[s] = make_double2(e.real(), e.imag());
    }
    INQB_CUDA(cudaMemcpyAsync(dcoef, coef.data(), sizeof(double2) * S, cudaMemcpyHostToDevice, ctx.stream));
    launch_shift_cvec<R>(ctx, D(res.o), CD(phi), S, np, dcoef, -1.0);
    // preconditioner: kinetic energy per state, then K(0.5 |G|^2 / T_s)
    launch_laplacian<R>(ctx, b, CD(res.o), D(lap.o), S, -0.5, zero);
    const auto tv = ovd(lap.o, res.o);
    const auto tn = ovd(res.o, res.o);
    for (int s = 0; s < S; s++) kin[s] = (tv[s] / tn[s]).real();
    INQB_CUDA(cudaMemcpyAsync(dkin, kin.data(), sizeof(double) * S, cudaMemcpyHostToDevice, ctx.stream));
    launch_tpa_precondition<R>(ctx, b, D(res.o), S, dkin);
    apply_any(h, res.o, hres.o);
    const auto m0 = ovd(res.o, res.o), m1 = ovd(phi, res.o), m2 = ovd(res.o, hres.o), m3 = ovd(phi, hres.o);
    for (int s = 0; s < S; s++) {
      const double ca = (m0[s] * m3[s] - m2[s] * m1[s]).real();
      const double cb = (nrm[s] * m2[s] - ev[s] * m0[s]).real();
      const double cc = (ev[s] * m1[s] - m3[s] * nrm[s]).real();
      const double den = cb + std::sqrt(cb * cb - 4.0 * ca * cc);
      coef[s] = make_double2(std::fabs(den) < 1e-15 ? 0.0 : 2.0 * cc / den, 0.0);
    }
    INQB_CUDA(cudaMemcpyAsync(dcoef, coef.data(), sizeof(double2) * S, cudaMemcpyHostToDevice, ctx.stream));
    launch_shift_cvec<R>(ctx, D(phi), CD(res.o), S, np, dcoef, 1.0);
    if (istep != num_steps - 1) launch_shift_cvec<R>(ctx, D(hphi.o), CD(hres.o), S, np, dcoef, 1.0);
  }
  INQB_CUDA(cudaStreamSynchronize(ctx.stream));  // the host factors above go out of scope
  dev_free(ctx, dov);
  dev_free(ctx, dcoef);
  dev_free(ctx, dkin);
}

extern "C" {

int inqb_ctx_create(int device, inqb_ctx **out) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(out != nullptr, INQB_ERR_ARG, "null output handle");
    int ndev = 0;
    INQB_CUDA(cudaGetDeviceCount(&ndev));
    INQB_REQUIRE(device >= 0 && device < ndev, INQB_ERR_ARG, "no such CUDA device");
    INQB_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    INQB_CUDA(cudaGetDeviceProperties(&prop, device));
    INQB_REQUIRE(prop.major >= 10, INQB_ERR_UNSUPPORTED,
                 "libinqb200 is built for sm_100a (B200); this device is sm_" + std::to_string(prop.major) +
                     std::to_string(prop.minor));
    auto *c = new inqb_ctx();
    c->device = device;
    c->num_sms = c->device_sms = prop.multiProcessorCount;
    c->max_smem_optin = prop.sharedMemPerBlockOptin;
    try {
      INQB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      note_device_alloc();
      INQB_CUDA(cudaMalloc(&c->d_err, sizeof(int)));
      INQB_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
      noalloc_prepare(*c);
    } catch (...) {
      if (c->d_err) cudaFree(c->d_err);
      if (c->stream) cudaStreamDestroy(c->stream);
      delete c;
      throw;
    }
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = c;
  });
}

int inqb_ctx_destroy(inqb_ctx *ctx) {
  if (!ctx) return INQB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (cudaStream_t st : ctx->aux) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (cudaEvent_t ev : ctx->aux_events) cudaEventDestroy(ev);
  cudaStreamDestroy(ctx->stream);
  if (ctx->d_err) cudaFree(ctx->d_err);
  delete ctx;
  return INQB_OK;
}

const char *inqb_last_error(const inqb_ctx *ctx) { return ctx ? ctx->err.c_str() : g_err_noctx.c_str(); }

int inqb_ctx_synchronize(inqb_ctx *ctx) {
  return guarded(ctx, [&] {
    set_device(*ctx);
    INQB_CUDA(cudaStreamSynchronize(ctx->stream));
    int flag = 0;
    INQB_CUDA(cudaMemcpy(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      INQB_CUDA(cudaMemset(ctx->d_err, 0, sizeof(int)));
      throw Error(INQB_ERR_TIMEOUT, "a device-side wait exceeded its time limit; the results of the calls since the "
                                    "last synchronize are invalid");
    }
  });
}

int inqb_ctx_check_wait_timeout(inqb_ctx *ctx, long long limit_ns) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(limit_ns >= 1000000 && limit_ns <= 1000000000, INQB_ERR_ARG, "limit_ns is 1e6 .. 1e9");
    set_device(*ctx);
    launch_wait_timeout(*ctx, limit_ns);
    INQB_CUDA(cudaGetLastError());
  });
}

int inqb_ctx_set_option(inqb_ctx *ctx, const char *key, long long value) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && key, INQB_ERR_ARG, "null argument");
    const std::string k(key);
    if (int *field = kernel_option(*ctx, k)) {
      check_kernel_option(*ctx, k, value);
      // grid_sms 0: every SM of the device
      *field = (k == "grid_sms" && value == 0) ? ctx->device_sms : int(value);
    } else if (k == "mixed_compute") {
      INQB_REQUIRE(value >= 0 && value <= 3, INQB_ERR_ARG, "mixed_compute is 0, 1, 2 or 3");
      ctx->mixed_compute = int(value);
    } else if (k == "fp64_mma") {
      INQB_REQUIRE(value == 0 || value == 1, INQB_ERR_ARG, "fp64_mma is 0 (SIMT) or 1 (FP64 tensor cores)");
      ctx->fp64_mma = int(value);
    } else if (k == "overlap_tc") {
      INQB_REQUIRE(value == 0 || value == 1, INQB_ERR_ARG, "overlap_tc is 0 (FP64 SIMT) or 1 (tensor cores)");
      ctx->overlap_tc = int(value);
    } else if (k == "stream_priority") {
      INQB_REQUIRE(value == 0 || value == 1, INQB_ERR_ARG, "stream_priority is 0 (low) or 1 (high)");
      if (int(value) != ctx->stream_priority) {
        set_device(*ctx);
        int least = 0, greatest = 0;
        INQB_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        cudaStream_t st = nullptr;
        INQB_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, value ? greatest : least));
        // work queued on the old stream finishes before anything queued on the new one
        cudaEvent_t ev = nullptr;
        INQB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        INQB_CUDA(cudaEventRecord(ev, ctx->stream));
        INQB_CUDA(cudaStreamWaitEvent(st, ev, 0));
        INQB_CUDA(cudaEventDestroy(ev));
        INQB_CUDA(cudaStreamSynchronize(ctx->stream));
        INQB_CUDA(cudaStreamDestroy(ctx->stream));
        ctx->stream = st;
        ctx->stream_priority = int(value);
      }
    } else {
      throw Error(INQB_ERR_ARG, "unknown option " + k);
    }
  });
}

int inqb_hamiltonian_set_option(inqb_hamiltonian *h, const char *key, long long value) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && key, INQB_ERR_ARG, "null argument");
    const std::string k(key);
    INQB_REQUIRE(kernel_option(*h->ctx, k) != nullptr, INQB_ERR_ARG,
                 "a Hamiltonian overrides fft_impl, fft_stages, fft_wide, fft_flat, nl_bulk, nl_apply_points, "
                 "nl_project_points, nl_project_ranges and grid_sms only (got " + k + ")");
    if (value < 0 && k != "nl_bulk") {
      // a negative value removes the override (the context's value applies again)
      for (size_t i = 0; i < h->opt_overrides.size(); i++)
        if (h->opt_overrides[i].first == k) h->opt_overrides.erase(h->opt_overrides.begin() + long(i));
      return;
    }
    check_kernel_option(*h->ctx, k, value);
    const int v = (k == "grid_sms" && value == 0) ? h->ctx->device_sms : int(value);
    for (auto &kv : h->opt_overrides)
      if (kv.first == k) {
        kv.second = v;
        return;
      }
    h->opt_overrides.emplace_back(k, v);
  });
}

int inqb_ctx_stream(inqb_ctx *ctx, void **stream) {
  return guarded(ctx, [&] { *stream = reinterpret_cast<void *>(ctx->stream); });
}

int inqb_ctx_launch_count(inqb_ctx *ctx, long long *count) {
  return guarded(ctx, [&] { *count = ctx->launches; });
}

int inqb_device_alloc_count(long long *count) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(count, INQB_ERR_ARG, "null argument");
    *count = device_alloc_count();
  });
}

int inqb_ctx_mem_info(inqb_ctx *ctx, size_t *free_bytes, size_t *total_bytes) {
  return guarded(ctx, [&] {
    set_device(*ctx);
    INQB_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
  });
}

int inqb_basis_create(inqb_ctx *ctx, const double lattice[9], int nx, int ny, int nz, inqb_basis **out) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && lattice && out, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nx > 0 && ny > 0 && nz > 0, INQB_ERR_ARG, "grid sizes must be positive");
    set_device(*ctx);
    auto *b = new inqb_basis();
    try {
      b->ctx = ctx;
      basis_metric(lattice, b->lat, b->rec, b->rlat, b->volume);
      b->n[0] = nx;
      b->n[1] = ny;
      b->n[2] = nz;
      b->npoints = (long long)nx * ny * nz;
      for (int ax = 0; ax < 3; ax++) {
        const int n = b->n[ax];
        b->radices[ax] = fft_radices(n);
        std::vector<double2> t64(n);
        std::vector<float2> t32(2 * n);  // per twiddle: float part, then remainder (cos - float(cos), ...)
        const long double two_pi = 6.283185307179586476925286766559005768L;
        for (int t = 0; t < n; t++) {
          const long double ang = two_pi * (long double)t / (long double)n;
          t64[t] = make_double2(double(cosl(ang)), double(-sinl(ang)));
          const long double c = cosl(ang), sn = -sinl(ang);
          t32[2 * t] = make_float2(float(c), float(sn));
          t32[2 * t + 1] = make_float2(float(c - (long double)t32[2 * t].x), float(sn - (long double)t32[2 * t].y));
        }
        INQB_CUDA(counted_malloc_async(&b->tw64[ax], sizeof(double2) * n, ctx->stream));
        INQB_CUDA(counted_malloc_async(&b->tw32[ax], sizeof(float2) * 2 * n, ctx->stream));
        INQB_CUDA(cudaMemcpyAsync(b->tw64[ax], t64.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, ctx->stream));
        INQB_CUDA(cudaMemcpyAsync(b->tw32[ax], t32.data(), sizeof(float2) * 2 * n, cudaMemcpyHostToDevice, ctx->stream));
        INQB_CUDA(cudaStreamSynchronize(ctx->stream));
      }
    } catch (...) {
      for (int ax = 0; ax < 3; ax++) {
        if (b->tw64[ax]) cudaFreeAsync(b->tw64[ax], ctx->stream);
        if (b->tw32[ax]) cudaFreeAsync(b->tw32[ax], ctx->stream);
      }
      delete b;
      throw;
    }
    *out = b;
  });
}

int inqb_basis_destroy(inqb_basis *b) {
  if (!b) return INQB_OK;
  cudaSetDevice(b->ctx->device);
  for (int ax = 0; ax < 3; ax++) {
    if (b->tw64[ax]) cudaFreeAsync(b->tw64[ax], b->ctx->stream);
    if (b->tw32[ax]) cudaFreeAsync(b->tw32[ax], b->ctx->stream);
  }
  delete b;
  return INQB_OK;
}

int inqb_basis_volume_element(const inqb_basis *b, double *dv) {
  return guarded(b ? b->ctx : nullptr, [&] {
    INQB_REQUIRE(b && dv, INQB_ERR_ARG, "null argument");
    *dv = b->volume / double(b->npoints);
  });
}

int inqb_orbitals_create(inqb_ctx *ctx, const inqb_basis *basis, int nst, int spinor_dim, const double kpoint_cov[3],
                         int spin_index, int space, int precision, inqb_orbitals **out) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && basis && out, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nst > 0, INQB_ERR_ARG, "number of states must be positive");
    INQB_REQUIRE(spinor_dim == 1, INQB_ERR_UNSUPPORTED, "spinor orbital sets are not implemented");
    INQB_REQUIRE(space == INQB_REAL_SPACE || space == INQB_FOURIER_SPACE, INQB_ERR_ARG, "bad space tag");
    INQB_REQUIRE(precision == INQB_F64 || precision == INQB_F32, INQB_ERR_ARG, "bad precision tag");
    INQB_REQUIRE(spin_index >= 0, INQB_ERR_ARG, "bad spin index");
    set_device(*ctx);
    auto *o = new inqb_orbitals();
    o->ctx = ctx;
    o->basis = basis;
    o->nst = nst;
    for (int i = 0; i < 3; i++) o->kpoint[i] = kpoint_cov ? kpoint_cov[i] : 0.0;
    o->spin_index = spin_index;
    o->space = space;
    o->precision = precision;
    cudaError_t e = counted_malloc_async(&o->data, o->bytes(), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // usable from any stream on return
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      delete o;
      throw Error(INQB_ERR_MEMORY, "device allocation of an orbital set failed: " + std::string(cudaGetErrorString(e)));
    }
    *out = o;
  });
}

int inqb_orbitals_wrap(inqb_ctx *ctx, const inqb_basis *basis, void *data, int nst, int spinor_dim,
                       const double kpoint_cov[3], int spin_index, int space, int precision, inqb_orbitals **out) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && basis && data && out, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(basis->ctx == ctx, INQB_ERR_ARG, "the basis belongs to another context");
    INQB_REQUIRE(nst > 0, INQB_ERR_ARG, "number of states must be positive");
    INQB_REQUIRE(spinor_dim == 1, INQB_ERR_UNSUPPORTED, "spinor orbital sets are not implemented");
    INQB_REQUIRE(space == INQB_REAL_SPACE || space == INQB_FOURIER_SPACE, INQB_ERR_ARG, "bad space tag");
    INQB_REQUIRE(precision == INQB_F64 || precision == INQB_F32, INQB_ERR_ARG, "bad precision tag");
    INQB_REQUIRE(spin_index >= 0, INQB_ERR_ARG, "bad spin index");
    INQB_REQUIRE(reinterpret_cast<uintptr_t>(data) % 16 == 0, INQB_ERR_ARG,
                 "wrapped orbital storage must be aligned to 16 bytes");
    set_device(*ctx);
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, data);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      throw Error(INQB_ERR_ARG, std::string("wrapped storage is not a CUDA pointer: ") + cudaGetErrorString(e));
    }
    INQB_REQUIRE(attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged, INQB_ERR_ARG,
                 "wrapped storage must be device or managed memory (got host or unregistered memory)");
    if (attr.type == cudaMemoryTypeDevice)
      INQB_REQUIRE(attr.device == ctx->device, INQB_ERR_ARG,
                   "wrapped storage is memory of device " + std::to_string(attr.device) + ", the context's is " +
                       std::to_string(ctx->device));
    auto *o = new inqb_orbitals();
    o->ctx = ctx;
    o->basis = basis;
    o->nst = nst;
    for (int i = 0; i < 3; i++) o->kpoint[i] = kpoint_cov ? kpoint_cov[i] : 0.0;
    o->spin_index = spin_index;
    o->space = space;
    o->precision = precision;
    o->data = data;
    o->owned = false;
    if (attr.type == cudaMemoryTypeManaged) {
      // the reference's allocator prefetches its managed arrays to the device (gpu/array.hpp:84-88); the
      // same here, ordered before every kernel the context queues on the set
      const cudaError_t pe = cudaMemPrefetchAsync(data, o->bytes(), ctx->device, ctx->stream);
      if (pe != cudaSuccess) {
        (void)cudaGetLastError();
        delete o;
        throw Error(INQB_ERR_CUDA, std::string("prefetch of managed orbital storage failed: ") + cudaGetErrorString(pe));
      }
    }
    *out = o;
  });
}

int inqb_orbitals_destroy(inqb_orbitals *o) {
  if (!o) return INQB_OK;
  cudaSetDevice(o->ctx->device);
  if (o->data && o->owned) cudaFreeAsync(o->data, o->ctx->stream);
  delete o;
  return INQB_OK;
}

int inqb_orbitals_upload(inqb_orbitals *o, const void *host) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o && host, INQB_ERR_ARG, "null argument");
    set_device(*o->ctx);
    INQB_CUDA(cudaMemcpyAsync(o->data, host, o->bytes(), cudaMemcpyHostToDevice, o->ctx->stream));
    INQB_CUDA(cudaStreamSynchronize(o->ctx->stream));
  });
}

int inqb_orbitals_download(const inqb_orbitals *o, void *host) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o && host, INQB_ERR_ARG, "null argument");
    set_device(*o->ctx);
    INQB_CUDA(cudaMemcpyAsync(host, o->data, o->bytes(), cudaMemcpyDeviceToHost, o->ctx->stream));
    INQB_CUDA(cudaStreamSynchronize(o->ctx->stream));
  });
}

int inqb_orbitals_device_ptr(const inqb_orbitals *o, void **ptr) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o && ptr, INQB_ERR_ARG, "null argument");
    *ptr = o->data;
  });
}

int inqb_orbitals_copy(const inqb_orbitals *src, inqb_orbitals *dst) {
  return guarded(src ? src->ctx : nullptr, [&] {
    INQB_REQUIRE(src && dst, INQB_ERR_ARG, "null argument");
    set_device(*src->ctx);
    copy_set(*src, *dst);
    for (int i = 0; i < 3; i++) dst->kpoint[i] = src->kpoint[i];
    dst->spin_index = src->spin_index;
  });
}

int inqb_orbitals_fill(inqb_orbitals *o, double re, double im) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o, INQB_ERR_ARG, "null argument");
    set_device(*o->ctx);
    const long long n = o->basis->npoints * o->nst;
    if (o->precision == INQB_F64) launch_fill<double>(*o->ctx, static_cast<double2 *>(o->data), n, re, im);
    else launch_fill<float>(*o->ctx, static_cast<float2 *>(o->data), n, re, im);
  });
}

int inqb_orbitals_set_space(inqb_orbitals *o, int space) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o && (space == INQB_REAL_SPACE || space == INQB_FOURIER_SPACE), INQB_ERR_ARG, "bad argument");
    o->space = space;
  });
}

int inqb_orbitals_info(const inqb_orbitals *o, int *nst, int *space, int *precision, long long *npoint) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o, INQB_ERR_ARG, "null argument");
    if (nst) *nst = o->nst;
    if (space) *space = o->space;
    if (precision) *precision = o->precision;
    if (npoint) *npoint = o->basis->npoints;
  });
}

int inqb_orbitals_randomize_gsphere(inqb_orbitals *o, uint64_t seed, double ecut) {
  return guarded(o ? o->ctx : nullptr, [&] {
    INQB_REQUIRE(o, INQB_ERR_ARG, "null argument");
    set_device(*o->ctx);
    if (o->precision == INQB_F64)
      launch_randomize_gsphere<double>(*o->ctx, *o->basis, static_cast<double2 *>(o->data), o->nst, seed, ecut);
    else
      launch_randomize_gsphere<float>(*o->ctx, *o->basis, static_cast<float2 *>(o->data), o->nst, seed, ecut);
    o->space = INQB_FOURIER_SPACE;
  });
}

int inqb_orbitals_convert(const inqb_orbitals *src, inqb_orbitals *dst) {
  return guarded(src ? src->ctx : nullptr, [&] {
    INQB_REQUIRE(src && dst, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(src->basis == dst->basis && src->nst == dst->nst, INQB_ERR_ARG, "conversion between different shapes");
    set_device(*src->ctx);
    launch_convert(*src->ctx, src->data, src->precision, dst->data, dst->precision, src->basis->npoints * src->nst);
    dst->space = src->space;
    for (int i = 0; i < 3; i++) dst->kpoint[i] = src->kpoint[i];
    dst->spin_index = src->spin_index;
  });
}

int inqb_to_fourier(const inqb_orbitals *in, inqb_orbitals *out) {
  return guarded(in ? in->ctx : nullptr, [&] {
    INQB_REQUIRE(in && out, INQB_ERR_ARG, "null argument");
    check_same_shape(*in, *out);
    INQB_REQUIRE(in->space == INQB_REAL_SPACE, INQB_ERR_ARG, "to_fourier needs a real-space set");
    set_device(*in->ctx);
    if (in->precision == INQB_F64)
      fft3d<double>(*in->ctx, *in->basis, static_cast<const double2 *>(in->data), static_cast<double2 *>(out->data),
                    in->nst, +1, 1.0);
    else
      fft3d<float>(*in->ctx, *in->basis, static_cast<const float2 *>(in->data), static_cast<float2 *>(out->data),
                   in->nst, +1, 1.0f);
    out->space = INQB_FOURIER_SPACE;
    for (int i = 0; i < 3; i++) out->kpoint[i] = in->kpoint[i];
    out->spin_index = in->spin_index;
  });
}

int inqb_to_real(const inqb_orbitals *in, inqb_orbitals *out, int normalize) {
  return guarded(in ? in->ctx : nullptr, [&] {
    INQB_REQUIRE(in && out, INQB_ERR_ARG, "null argument");
    check_same_shape(*in, *out);
    INQB_REQUIRE(in->space == INQB_FOURIER_SPACE, INQB_ERR_ARG, "to_real needs a Fourier-space set");
    set_device(*in->ctx);
    const double sc = normalize ? 1.0 / double(in->basis->npoints) : 1.0;
    if (in->precision == INQB_F64)
      fft3d<double>(*in->ctx, *in->basis, static_cast<const double2 *>(in->data), static_cast<double2 *>(out->data),
                    in->nst, -1, sc);
    else
      fft3d<float>(*in->ctx, *in->basis, static_cast<const float2 *>(in->data), static_cast<float2 *>(out->data),
                   in->nst, -1, sc);
    out->space = INQB_REAL_SPACE;
    for (int i = 0; i < 3; i++) out->kpoint[i] = in->kpoint[i];
    out->spin_index = in->spin_index;
  });
}

int inqb_laplacian(const inqb_orbitals *in, inqb_orbitals *out, double factor, const double gradcoeff_contra[3]) {
  return guarded(in ? in->ctx : nullptr, [&] {
    INQB_REQUIRE(in && out, INQB_ERR_ARG, "null argument");
    check_same_shape(*in, *out);
    INQB_REQUIRE(in->space == INQB_FOURIER_SPACE, INQB_ERR_ARG, "laplacian is implemented for Fourier-space sets");
    set_device(*in->ctx);
    double gc[3] = {0, 0, 0};
    if (gradcoeff_contra)
      for (int i = 0; i < 3; i++) gc[i] = gradcoeff_contra[i];
    if (in->precision == INQB_F64)
      launch_laplacian<double>(*in->ctx, *in->basis, static_cast<const double2 *>(in->data),
                               static_cast<double2 *>(out->data), in->nst, factor, gc);
    else
      launch_laplacian<float>(*in->ctx, *in->basis, static_cast<const float2 *>(in->data),
                              static_cast<float2 *>(out->data), in->nst, factor, gc);
    out->space = INQB_FOURIER_SPACE;
  });
}

int inqb_hamiltonian_create(inqb_ctx *ctx, const inqb_basis *basis, int nspin, inqb_hamiltonian **out) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && basis && out, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nspin >= 1 && nspin <= 2, INQB_ERR_UNSUPPORTED, "nspin must be 1 or 2");
    set_device(*ctx);
    auto *h = new inqb_hamiltonian();
    h->ctx = ctx;
    h->basis = basis;
    h->nspin = nspin;
    const size_t nv = size_t(basis->npoints) * nspin;
    INQB_CUDA(counted_malloc_async(&h->d_V, sizeof(double) * nv, ctx->stream));
    INQB_CUDA(counted_malloc_async(&h->d_V32, sizeof(float) * nv, ctx->stream));
    INQB_CUDA(cudaMemsetAsync(h->d_V, 0, sizeof(double) * nv, ctx->stream));
    INQB_CUDA(cudaMemsetAsync(h->d_V32, 0, sizeof(float) * nv, ctx->stream));
    INQB_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = h;
  });
}

int inqb_hamiltonian_destroy(inqb_hamiltonian *h) {
  if (!h) return INQB_OK;
  cudaSetDevice(h->ctx->device);
  cudaStream_t st = h->ctx->stream;
  free_projectors(h->proj, st);
  if (h->d_V) cudaFreeAsync(h->d_V, st);
  if (h->d_V32) cudaFreeAsync(h->d_V32, st);
  if (h->d_projraw) cudaFreeAsync(h->d_projraw, st);
  if (h->d_projD) cudaFreeAsync(h->d_projD, st);
  if (h->d_vion) cudaFreeAsync(h->d_vion, st);
  delete h;
  return INQB_OK;
}

int inqb_potential_set(inqb_hamiltonian *h, const double *V) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && V, INQB_ERR_ARG, "null argument");
    set_device(*h->ctx);
    const size_t nv = size_t(h->basis->npoints) * h->nspin;
    std::vector<float> v32(V, V + nv);
    INQB_CUDA(cudaMemcpyAsync(h->d_V, V, sizeof(double) * nv, cudaMemcpyHostToDevice, h->ctx->stream));
    INQB_CUDA(cudaMemcpyAsync(h->d_V32, v32.data(), sizeof(float) * nv, cudaMemcpyHostToDevice, h->ctx->stream));
    INQB_CUDA(cudaStreamSynchronize(h->ctx->stream));
  });
}

int inqb_hamiltonian_set_interaction(inqb_hamiltonian *h, const double *vion, int hartree, int xc) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h, INQB_ERR_ARG, "null argument");
    set_device(*h->ctx);
    if (!vion) {  // back to a fixed potential
      if (h->d_vion) dev_free(*h->ctx, h->d_vion);
      h->d_vion = nullptr;
      h->hartree = h->xc = 0;
      return;
    }
    INQB_REQUIRE(xc == 0 || xc == 1, INQB_ERR_ARG, "xc is 0 (none) or 1 (LDA: Slater exchange, PZ81 correlation)");
    INQB_REQUIRE(h->nspin == 1, INQB_ERR_UNSUPPORTED, "the interacting update is implemented for one spin channel");
    set_device(*h->ctx);
    const size_t n = size_t(h->basis->npoints);
    if (!h->d_vion) h->d_vion = static_cast<double *>(dev_alloc(*h->ctx, sizeof(double) * n));
    INQB_CUDA(cudaMemcpyAsync(h->d_vion, vion, sizeof(double) * n, cudaMemcpyHostToDevice, h->ctx->stream));
    INQB_CUDA(cudaStreamSynchronize(h->ctx->stream));
    h->hartree = hartree ? 1 : 0;
    h->xc = xc;
  });
}

int inqb_update_hamiltonian(inqb_hamiltonian *h, const double *density, double energies[4]) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && density, INQB_ERR_ARG, "null argument");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    const size_t n = size_t(h->basis->npoints);
    double *d = static_cast<double *>(dev_alloc(ctx, sizeof(double) * n));
    INQB_CUDA(cudaMemcpyAsync(d, density, sizeof(double) * n, cudaMemcpyHostToDevice, ctx.stream));
    double e[4];
    update_hamiltonian_dev(*h, d, e);
    if (energies)
      for (int k = 0; k < 4; k++) energies[k] = e[k];
    dev_free(ctx, d);
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  });
}

int inqb_vector_potential_set(inqb_hamiltonian *h, const double A_cov[3]) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && A_cov, INQB_ERR_ARG, "null argument");
    for (int i = 0; i < 3; i++) h->A[i] = A_cov[i];
  });
}

int inqb_projectors_set(inqb_hamiltonian *h, int nproj, int maxsph, int maxnlm, const int32_t *points, const float *pos,
                        const double *matrices, const double *coeff, const int32_t *npts, const int32_t *nlm) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nproj == 0 || (points && pos && matrices && coeff && npts && nlm), INQB_ERR_ARG, "null table");
    set_device(*h->ctx);
    set_projectors(*h, nproj, maxsph, maxnlm, points, pos, matrices, coeff, npts, nlm);
    h->dev_natoms = 0;  // explicit tables: nothing to move
  });
}

// what the last Gaussian build was made of, for inqb_projectors_move
static DeviceProjectorSpec gaussian_spec(int natoms, double radius, double rc, const double *kb) {
  DeviceProjectorSpec sp;
  sp.gaussian = 1;
  sp.radius = radius;
  sp.rc = rc;
  sp.kb.assign(kb, kb + size_t(natoms) * 16);
  return sp;
}

int inqb_projectors_build_gaussian_device(inqb_hamiltonian *h, int natoms, const double *positions, double radius,
                                          double rc, const double *kb) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && (natoms == 0 || (positions && kb)), INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(natoms >= 0, INQB_ERR_ARG, "negative atom count");
    INQB_REQUIRE(radius > 0.0 && rc > 0.0, INQB_ERR_ARG, "radius and rc must be positive");
    set_device(*h->ctx);
    DeviceProjectorSpec sp = gaussian_spec(natoms, radius, rc, natoms ? kb : nullptr);
    build_projectors_device(*h, natoms, positions, sp);
    h->dev_natoms = natoms;
    h->dev_spec = std::move(sp);
  });
}

int inqb_projectors_build_radial(inqb_hamiltonian *h, int natoms, const double *positions, const int32_t *species,
                                 int nspecies, const double *radius, int nr, double dr, int ntables,
                                 const double *tables, const int32_t *ngroups, const int32_t *functions,
                                 const double *kb) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && natoms >= 0 && nspecies >= 0 && ntables >= 0, INQB_ERR_ARG, "bad argument");
    INQB_REQUIRE(natoms == 0 || (positions && species && radius && ngroups), INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nr > 0 && dr > 0.0, INQB_ERR_ARG, "radial tables need nr > 0 points and dr > 0");
    DeviceProjectorSpec sp;
    sp.gaussian = 0;
    sp.species.assign(species, species + natoms);
    sp.sradius.assign(radius, radius + nspecies);
    sp.ngroups.assign(ngroups, ngroups + nspecies);
    int groups = 0;
    for (int s = 0; s < nspecies; s++) {
      INQB_REQUIRE(ngroups[s] >= 0 && radius[s] >= 0.0, INQB_ERR_ARG, "bad species description");
      groups += ngroups[s];
    }
    INQB_REQUIRE(groups == 0 || (functions && kb && (ntables == 0 || tables)), INQB_ERR_ARG, "null table");
    sp.fn.assign(functions, functions + size_t(groups) * 12);
    sp.gkb.assign(kb, kb + size_t(groups) * 16);
    sp.tables.assign(tables, tables + size_t(ntables) * nr);
    sp.nr = nr;
    sp.dr = dr;
    set_device(*h->ctx);
    build_projectors_device(*h, natoms, positions, sp);
    h->dev_natoms = natoms;
    h->dev_spec = std::move(sp);
  });
}

int inqb_projectors_move(inqb_hamiltonian *h, const double *positions) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && positions, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(h->dev_natoms > 0, INQB_ERR_ARG, "no Gaussian or radial projectors were built on this Hamiltonian");
    set_device(*h->ctx);
    const DeviceProjectorSpec sp = h->dev_spec;
    build_projectors_device(*h, h->dev_natoms, positions, sp);
  });
}

int inqb_projectors_build_gaussian(inqb_hamiltonian *h, int natoms, const double *positions, double radius, double rc,
                                   const double *kb) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && (natoms == 0 || (positions && kb)), INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(radius > 0.0 && rc > 0.0, INQB_ERR_ARG, "radius and rc must be positive");
    set_device(*h->ctx);
    if (natoms > 0) {
      h->dev_natoms = natoms;
      h->dev_spec = gaussian_spec(natoms, radius, rc, kb);
    }
    std::vector<SphereList> sph(natoms);
    int maxsph = 0;
    for (int a = 0; a < natoms; a++) {
      spherical_grid_build(*h->basis, positions + 3 * a, radius, sph[a]);
      maxsph = std::max<int>(maxsph, int(sph[a].points.size()));
    }
    std::vector<int32_t> points(size_t(natoms) * maxsph * 3, -1), npts(natoms), nlm(natoms, 4);
    std::vector<float> pos(size_t(natoms) * maxsph * 3, 0.0f);
    std::vector<double> mats(size_t(natoms) * 4 * maxsph, 0.0);
    for (int a = 0; a < natoms; a++) {
      const size_t n = sph[a].points.size();
      npts[a] = int(n);
      std::vector<double> m;
      gaussian_projector_values(*h->basis, sph[a], rc, m);
      for (size_t i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) {
          points[(size_t(a) * maxsph + i) * 3 + d] = sph[a].points[i][d];
          pos[(size_t(a) * maxsph + i) * 3 + d] = sph[a].relpos[i][d];
        }
        for (int l = 0; l < 4; l++) mats[(size_t(a) * 4 + l) * maxsph + i] = m[l * n + i];
      }
    }
    set_projectors(*h, natoms, maxsph, 4, points.data(), pos.data(), mats.data(), kb, npts.data(), nlm.data());
  });
}

int inqb_spherical_grid(const double lattice[9], int nx, int ny, int nz, const double center[3], double radius,
                        long long capacity, int32_t *points, float *distance, float *relpos, long long *npoints) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(lattice && center && npoints, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nx > 0 && ny > 0 && nz > 0 && radius >= 0.0, INQB_ERR_ARG, "bad grid or radius");
    Basis b;
    basis_metric(lattice, b.lat, b.rec, b.rlat, b.volume);
    b.n[0] = nx;
    b.n[1] = ny;
    b.n[2] = nz;
    b.npoints = (long long)nx * ny * nz;
    SphereList sph;
    spherical_grid_build(b, center, radius, sph);
    const long long n = (long long)sph.points.size();
    *npoints = n;
    INQB_REQUIRE(n <= capacity, INQB_ERR_ARG, "capacity too small for the sphere");
    for (long long i = 0; i < n; i++) {
      for (int d = 0; d < 3; d++) {
        if (points) points[i * 3 + d] = sph.points[size_t(i)][d];
        if (relpos) relpos[i * 3 + d] = sph.relpos[size_t(i)][d];
      }
      if (distance) distance[i] = sph.distance[size_t(i)];
    }
  });
}

int inqb_projectors_info(const inqb_hamiltonian *h, int *nproj, int *maxsph, long long *total_points) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h, INQB_ERR_ARG, "null argument");
    if (nproj) *nproj = h->proj.nproj;
    if (maxsph) *maxsph = h->proj.maxsph;
    if (total_points) *total_points = h->proj.total;
  });
}

int inqb_projectors_get(const inqb_hamiltonian *h, int32_t *points, float *pos, double *matrices, int32_t *npts) {
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h, INQB_ERR_ARG, "null argument");
    const Projectors &P = h->proj;
    if (P.device_built && P.nproj > 0) {
      // tables built on the device: read them back in the packed host layout
      set_device(*h->ctx);
      Ctx &ctx = *h->ctx;
      const size_t slots = size_t(P.nproj) * P.maxsph;
      if (points) {
        std::vector<int> flat = download<int>(ctx, P.d_pt, slots);
        const int ny = h->basis->n[1], nz = h->basis->n[2];
        for (size_t e = 0; e < slots; e++) {
          const int f = flat[e];
          points[3 * e] = f < 0 ? -1 : f / (ny * nz);
          points[3 * e + 1] = f < 0 ? -1 : (f / nz) % ny;
          points[3 * e + 2] = f < 0 ? -1 : f % nz;
        }
      }
      if (pos) {
        std::vector<float> v = download<float>(ctx, P.d_pos, 3 * slots);
        std::copy(v.begin(), v.end(), pos);
      }
      if (matrices) {
        std::vector<double> v = download<double>(ctx, P.d_mat, 4 * slots);
        std::copy(v.begin(), v.end(), matrices);
      }
    } else {
      if (points) std::copy(P.h_points.begin(), P.h_points.end(), points);
      if (pos) std::copy(P.h_pos.begin(), P.h_pos.end(), pos);
      if (matrices) std::copy(P.h_mat.begin(), P.h_mat.end(), matrices);
    }
    if (npts) std::copy(P.h_npts.begin(), P.h_npts.end(), npts);
  });
}

int inqb_apply(const inqb_hamiltonian *hc, const inqb_orbitals *in, inqb_orbitals *out) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && in && out, INQB_ERR_ARG, "null argument");
    set_device(*h->ctx);
    apply_any(*h, *in, *out);
  });
}

// Streams, events and device blocks of one inqb_apply_host call; released after every copy and
// kernel of the call has finished (also when the call fails half-way).
struct HostApplyRes {
  Ctx *ctx = nullptr;
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t ev_in[2] = {}, ev_comp[2] = {}, ev_out[2] = {}, ev_join = nullptr;
  void *bin[2] = {}, *bout[2] = {};
  ~HostApplyRes() {
    if (up) cudaStreamSynchronize(up);
    if (down) cudaStreamSynchronize(down);
    if (ctx) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < 2; i++) {
      // stream-ordered frees back to the pool: the next call reuses the blocks without cudaMalloc
      if (bin[i]) cudaFreeAsync(bin[i], ctx->stream);
      if (bout[i]) cudaFreeAsync(bout[i], ctx->stream);
      for (cudaEvent_t e : {ev_in[i], ev_comp[i], ev_out[i]})
        if (e) cudaEventDestroy(e);
    }
    if (ev_join) cudaEventDestroy(ev_join);
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
  }
};

// H over nsets host sets of one shape, streamed through one pipeline of state blocks: the blocks of the
// sets follow one another, so the upload of a set's first block overlaps the download of the previous
// set's last one.
void apply_host_sets(inqb_hamiltonian *h, int nsets, int nst, const double kpoint_cov[3], int spin_index,
                     int precision, const void *const *host_in, void *const *host_out, int block_states) {
  INQB_REQUIRE(h && host_in && host_out && nsets >= 1, INQB_ERR_ARG, "null argument");
  INQB_REQUIRE(nst > 0 && block_states >= 0, INQB_ERR_ARG, "bad state count");
  INQB_REQUIRE(precision == INQB_F64 || precision == INQB_F32, INQB_ERR_ARG, "bad precision tag");
  INQB_REQUIRE(spin_index >= 0 && spin_index < h->nspin, INQB_ERR_ARG, "spin index out of range");
  for (int k = 0; k < nsets; k++) {
    INQB_REQUIRE(host_in[k] && host_out[k], INQB_ERR_ARG, "null argument");
    for (int j = 0; j < nsets; j++)
      INQB_REQUIRE(host_in[k] != host_out[j], INQB_ERR_ARG, "H|psi> needs distinct input and output buffers");
  }
  set_device(*h->ctx);
  Ctx &ctx = *h->ctx;
  const size_t cs = precision == INQB_F64 ? 16 : 8;
  const size_t npts = size_t(h->basis->npoints);
  int B = block_states > 0 ? block_states : int(512 / cs);  // 512-byte rows of a block by default
  if (B > nst) B = nst;
  // block boundaries: blocks of B states, the last one shorter.  Measured at 96^3 x 256 single (box to box
  // 45-51 ms per call): neither a half-size first and last block nor quarter-size last blocks did better
  // than equal 64-state blocks; rows of 128 bytes download at 22-35 GB/s against 48 GB/s for 512 bytes
  std::vector<int> starts;
  for (int s0 = 0; s0 < nst; s0 += B) starts.push_back(s0);
  starts.push_back(nst);
  const int nblocks = int(starts.size()) - 1;
  const int total = nblocks * nsets;
  HostApplyRes r;
  r.ctx = &ctx;
  INQB_CUDA(cudaStreamCreateWithFlags(&r.up, cudaStreamNonBlocking));
  INQB_CUDA(cudaStreamCreateWithFlags(&r.down, cudaStreamNonBlocking));
  for (int i = 0; i < 2; i++) {
    INQB_CUDA(cudaEventCreateWithFlags(&r.ev_in[i], cudaEventDisableTiming));
    INQB_CUDA(cudaEventCreateWithFlags(&r.ev_comp[i], cudaEventDisableTiming));
    INQB_CUDA(cudaEventCreateWithFlags(&r.ev_out[i], cudaEventDisableTiming));
    for (void **p : {&r.bin[i], &r.bout[i]}) {
      if (i == 1 && total == 1) continue;
      cudaError_t e = counted_malloc_async(p, npts * B * cs, ctx.stream);
      if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(INQB_ERR_MEMORY, "device allocation of a state block failed: " + std::string(cudaGetErrorString(e)));
      }
    }
  }
  INQB_CUDA(cudaEventCreateWithFlags(&r.ev_join, cudaEventDisableTiming));
  // the copies start after the work already queued on the context's stream
  INQB_CUDA(cudaEventRecord(r.ev_join, ctx.stream));
  INQB_CUDA(cudaStreamWaitEvent(r.up, r.ev_join, 0));
  for (int i = 0; i < total; i++) {
    const int set = i / nblocks, blk = i % nblocks;
    const char *hin = static_cast<const char *>(host_in[set]);
    char *hout = static_cast<char *>(host_out[set]);
    const int slot = i & 1, s0 = starts[blk], nb = starts[blk + 1] - starts[blk];
    // block i reuses the buffers of block i - 2: its upload waits for that block's operator, its
    // operator for that block's download
    if (i >= 2) INQB_CUDA(cudaStreamWaitEvent(r.up, r.ev_comp[slot], 0));
    INQB_CUDA(cudaMemcpy2DAsync(r.bin[slot], nb * cs, hin + s0 * cs, nst * cs, nb * cs, npts, cudaMemcpyHostToDevice,
                                r.up));
    INQB_CUDA(cudaEventRecord(r.ev_in[slot], r.up));
    INQB_CUDA(cudaStreamWaitEvent(ctx.stream, r.ev_in[slot], 0));
    if (i >= 2) INQB_CUDA(cudaStreamWaitEvent(ctx.stream, r.ev_out[slot], 0));
    Orbitals in, out;
    in.ctx = out.ctx = &ctx;
    in.basis = out.basis = h->basis;
    in.nst = out.nst = nb;
    for (int k = 0; k < 3; k++) in.kpoint[k] = out.kpoint[k] = kpoint_cov ? kpoint_cov[k] : 0.0;
    in.spin_index = out.spin_index = spin_index;
    in.space = out.space = INQB_REAL_SPACE;
    in.precision = out.precision = precision;
    in.data = r.bin[slot];
    out.data = r.bout[slot];
    apply_any(*h, in, out);
    INQB_CUDA(cudaEventRecord(r.ev_comp[slot], ctx.stream));
    INQB_CUDA(cudaStreamWaitEvent(r.down, r.ev_comp[slot], 0));
    INQB_CUDA(cudaMemcpy2DAsync(hout + s0 * cs, nst * cs, r.bout[slot], nb * cs, nb * cs, npts,
                                cudaMemcpyDeviceToHost, r.down));
    INQB_CUDA(cudaEventRecord(r.ev_out[slot], r.down));
  }
  INQB_CUDA(cudaEventRecord(r.ev_join, r.down));
  INQB_CUDA(cudaStreamWaitEvent(ctx.stream, r.ev_join, 0));
  INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  int flag = 0;
  INQB_CUDA(cudaMemcpy(&flag, ctx.d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    INQB_CUDA(cudaMemset(ctx.d_err, 0, sizeof(int)));
    throw Error(INQB_ERR_TIMEOUT, "a device-side wait exceeded its time limit; host_out is invalid");
  }
}

int inqb_apply_host(const inqb_hamiltonian *hc, int nst, const double kpoint_cov[3], int spin_index, int precision,
                    const void *host_in, void *host_out, int block_states) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && host_in && host_out, INQB_ERR_ARG, "null argument");
    const void *ins[1] = {host_in};
    void *outs[1] = {host_out};
    apply_host_sets(h, 1, nst, kpoint_cov, spin_index, precision, ins, outs, block_states);
  });
}

int inqb_apply_host_many(const inqb_hamiltonian *hc, int nsets, int nst, const double kpoint_cov[3], int spin_index,
                         int precision, const void *const *host_in, void *const *host_out, int block_states) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && nsets >= 1, INQB_ERR_ARG, "null argument or no sets");
    apply_host_sets(h, nsets, nst, kpoint_cov, spin_index, precision, host_in, host_out, block_states);
  });
}

int inqb_non_local(const inqb_hamiltonian *hc, const inqb_orbitals *in, inqb_orbitals *out) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && in && out, INQB_ERR_ARG, "null argument");
    check_same_shape(*in, *out);
    INQB_REQUIRE(in->space == INQB_REAL_SPACE, INQB_ERR_ARG, "non_local needs a real-space set");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    const long long n = h->basis->npoints * in->nst;
    if (h->proj.nproj == 0) {
      if (in->precision == INQB_F64) launch_fill<double>(ctx, static_cast<double2 *>(out->data), n, 0, 0);
      else launch_fill<float>(ctx, static_cast<float2 *>(out->data), n, 0, 0);
      return;
    }
    double kA[3] = {in->kpoint[0] + h->A[0], in->kpoint[1] + h->A[1], in->kpoint[2] + h->A[2]};
    ensure_tables(*h, kA);
    if (in->precision == INQB_F64) {
      auto *praw = proj_buf<double>(*h, in->nst, 0);
      auto *pd = proj_buf<double>(*h, in->nst, 1);
      launch_nl_project<double>(ctx, *h->basis, *h, static_cast<const double2 *>(in->data), in->nst, praw, pd);
      launch_nl_scatter<double>(ctx, *h->basis, *h, pd, in->nst, static_cast<double2 *>(out->data));
    } else {
      auto *praw = proj_buf<float>(*h, in->nst, 0);
      auto *pd = proj_buf<float>(*h, in->nst, 1);
      launch_nl_project<float>(ctx, *h->basis, *h, static_cast<const float2 *>(in->data), in->nst, praw, pd);
      launch_nl_scatter<float>(ctx, *h->basis, *h, pd, in->nst, static_cast<float2 *>(out->data));
    }
    out->space = INQB_REAL_SPACE;
  });
}

int inqb_non_local_energy(const inqb_hamiltonian *hc, const inqb_orbitals *phi, const double *occ, double *energy) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phi && occ && energy, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(phi->space == INQB_REAL_SPACE, INQB_ERR_ARG, "non_local_energy needs a real-space set");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    *energy = 0.0;
    if (h->proj.nproj == 0) return;
    const int S = phi->nst;
    double kA[3] = {phi->kpoint[0] + h->A[0], phi->kpoint[1] + h->A[1], phi->kpoint[2] + h->A[2]};
    ensure_tables(*h, kA);
    const size_t n = size_t(h->proj.nproj) * 4 * S;
    std::vector<double> pr, pd;
    if (phi->precision == INQB_F64) {
      auto *praw = proj_buf<double>(*h, S, 0);
      auto *pD = proj_buf<double>(*h, S, 1);
      launch_nl_project<double>(ctx, *h->basis, *h, static_cast<const double2 *>(phi->data), S, praw, pD);
      pr = download<double>(ctx, praw, 2 * n);
      pd = download<double>(ctx, pD, 2 * n);
    } else {
      auto *praw = proj_buf<float>(*h, S, 0);
      auto *pD = proj_buf<float>(*h, S, 1);
      launch_nl_project<float>(ctx, *h->basis, *h, static_cast<const float2 *>(phi->data), S, praw, pD);
      auto a = download<float>(ctx, praw, 2 * n), b = download<float>(ctx, pD, 2 * n);
      pr.assign(a.begin(), a.end());
      pd.assign(b.begin(), b.end());
    }
    // projector_all::energy (projector_all.hpp:306-327): sum f_s Re(conj(p) D p)
    double en = 0.0;
    for (size_t k = 0; k < n; k++) {
      const int s = int(k % S);
      en += occ[s] * (pr[2 * k] * pd[2 * k] + pr[2 * k + 1] * pd[2 * k + 1]);
    }
    *energy = en;
  });
}

int inqb_kinetic_expectation_value(const inqb_hamiltonian *hc, const inqb_orbitals *phi, double *out) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phi && out, INQB_ERR_ARG, "null argument");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    const Basis &b = *h->basis;
    const int S = phi->nst;
    double kA[3] = {phi->kpoint[0] + h->A[0], phi->kpoint[1] + h->A[1], phi->kpoint[2] + h->A[2]};
    double kt[3], kc[3];
    cov_to_cart(b, kA, kt);
    cart_to_contra(b, kt, kc);
    double gc[3] = {-2.0 * kc[0], -2.0 * kc[1], -2.0 * kc[2]};
    double gcart[3];
    contra_to_cart(b, gc, gcart);
    const double k2 = -0.25 * (gcart[0] * gcart[0] + gcart[1] * gcart[1] + gcart[2] * gcart[2]);
    const double fac = -0.5 * (b.volume / (double(b.npoints) * double(b.npoints)));
    double *d_out = static_cast<double *>(dev_alloc(ctx, sizeof(double) * S));
    if (phi->space == INQB_REAL_SPACE) {
      TempSet f(*phi);
      if (phi->precision == INQB_F64) {
        fft3d<double>(ctx, b, static_cast<const double2 *>(phi->data), static_cast<double2 *>(f.o.data), S, +1, 1.0);
        launch_kinetic_ev<double>(ctx, b, static_cast<const double2 *>(f.o.data), S, fac, gc, k2, d_out);
      } else {
        fft3d<float>(ctx, b, static_cast<const float2 *>(phi->data), static_cast<float2 *>(f.o.data), S, +1, 1.0f);
        launch_kinetic_ev<float>(ctx, b, static_cast<const float2 *>(f.o.data), S, fac, gc, k2, d_out);
      }
    } else {
      if (phi->precision == INQB_F64)
        launch_kinetic_ev<double>(ctx, b, static_cast<const double2 *>(phi->data), S, fac, gc, k2, d_out);
      else
        launch_kinetic_ev<float>(ctx, b, static_cast<const float2 *>(phi->data), S, fac, gc, k2, d_out);
    }
    auto v = download<double>(ctx, d_out, S);
    std::copy(v.begin(), v.end(), out);
    dev_free(ctx, d_out);
  });
}

int inqb_overlap(const inqb_orbitals *a, const inqb_orbitals *b, double *out) {
  return guarded(a ? a->ctx : nullptr, [&] {
    INQB_REQUIRE(a && b && out, INQB_ERR_ARG, "null argument");
    set_device(*a->ctx);
    Ctx &ctx = *a->ctx;
    double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * a->nst * b->nst));
    overlap_dev(*a, *b, d);
    auto v = download<double>(ctx, d, size_t(2) * a->nst * b->nst);
    std::copy(v.begin(), v.end(), out);
    dev_free(ctx, d);
  });
}

int inqb_overlap_diagonal(const inqb_orbitals *a, const inqb_orbitals *b, double *out) {
  return guarded(a ? a->ctx : nullptr, [&] {
    INQB_REQUIRE(a && b && out, INQB_ERR_ARG, "null argument");
    set_device(*a->ctx);
    Ctx &ctx = *a->ctx;
    double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * a->nst));
    ovdiag_dev(*a, *b, d);
    auto v = download<double>(ctx, d, size_t(2) * a->nst);
    std::copy(v.begin(), v.end(), out);
    dev_free(ctx, d);
  });
}

int inqb_orthogonalize(inqb_orbitals *phi) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(phi, INQB_ERR_ARG, "null argument");
    set_device(*phi->ctx);
    orthogonalize_dev(*phi);
  });
}

int inqb_steepest_descent(const inqb_hamiltonian *hc, inqb_orbitals *fphi) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && fphi, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(fphi->space == INQB_FOURIER_SPACE, INQB_ERR_ARG, "steepest_descent needs a Fourier-space set");
    INQB_REQUIRE(fphi->basis == h->basis, INQB_ERR_ARG, "orbitals and Hamiltonian live on different bases");
    set_device(*h->ctx);
    if (fphi->precision == INQB_F64) steepest_descent_t<double>(*h, *fphi);
    else steepest_descent_t<float>(*h, *fphi);
    orthogonalize_dev(*fphi);
  });
}

int inqb_shift(double re, double im, const inqb_orbitals *chi, inqb_orbitals *phi) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(chi && phi, INQB_ERR_ARG, "null argument");
    check_same_shape(*chi, *phi);
    set_device(*phi->ctx);
    const long long n = phi->basis->npoints * phi->nst;
    if (phi->precision == INQB_F64)
      launch_axpy<double>(*phi->ctx, static_cast<double2 *>(phi->data), static_cast<const double2 *>(chi->data), n, re,
                          im);
    else
      launch_axpy<float>(*phi->ctx, static_cast<float2 *>(phi->data), static_cast<const float2 *>(chi->data), n, re, im);
  });
}

int inqb_rotate(inqb_orbitals *phi, const double *R) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(phi && R, INQB_ERR_ARG, "null argument");
    set_device(*phi->ctx);
    Ctx &ctx = *phi->ctx;
    const int S = phi->nst;
    double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * S * S));
    INQB_CUDA(cudaMemcpyAsync(d, R, sizeof(double2) * S * S, cudaMemcpyHostToDevice, ctx.stream));
    rotate_dev(*phi, d);
    dev_free(ctx, d);
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  });
}

int inqb_rotate_to(const inqb_orbitals *phi, inqb_orbitals *rotphi, const double *R, const double alpha[2],
                   const double beta[2]) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(phi && rotphi && R && alpha && beta, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(phi != rotphi, INQB_ERR_ARG, "rotate_to needs distinct sets (inqb_rotate rotates in place)");
    INQB_REQUIRE(phi->ctx == rotphi->ctx && phi->basis == rotphi->basis, INQB_ERR_ARG, "sets on different contexts or bases");
    INQB_REQUIRE(phi->precision == rotphi->precision && phi->space == rotphi->space, INQB_ERR_ARG,
                 "sets of different precisions or spaces");
    set_device(*phi->ctx);
    Ctx &ctx = *phi->ctx;
    const int Si = phi->nst, So = rotphi->nst;
    double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * Si * So));
    INQB_CUDA(cudaMemcpyAsync(d, R, sizeof(double2) * Si * So, cudaMemcpyHostToDevice, ctx.stream));
    const double2 a = make_double2(alpha[0], alpha[1]), be = make_double2(beta[0], beta[1]);
    const long long np = phi->basis->npoints;
    if (phi->precision == INQB_F64)
      launch_rotate_to<double>(ctx, static_cast<const double2 *>(phi->data), Si, static_cast<double2 *>(rotphi->data), So,
                               np, d, a, be);
    else
      launch_rotate_to<float>(ctx, static_cast<const float2 *>(phi->data), Si, static_cast<float2 *>(rotphi->data), So,
                              np, d, a, be);
    dev_free(ctx, d);
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  });
}

int inqb_hermitian_eigen(int n, const double *A, double *w, double *V) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(n > 0 && A && w && V, INQB_ERR_ARG, "bad argument");
    hermitian_eigen(n, reinterpret_cast<const std::complex<double> *>(A), w, reinterpret_cast<std::complex<double> *>(V));
  });
}

int inqb_cholesky_inverse(int n, const double *S, double *X) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(n > 0 && S && X, INQB_ERR_ARG, "bad argument");
    cholesky_inverse(n, reinterpret_cast<const std::complex<double> *>(S), reinterpret_cast<std::complex<double> *>(X));
  });
}

int inqb_eigenvalues(const inqb_hamiltonian *hc, const inqb_orbitals *phi, double *eig, double *normres) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phi && eig, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(phi->space == INQB_REAL_SPACE, INQB_ERR_ARG, "eigenvalues need a real-space set");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    const int S = phi->nst;
    TempSet hp(*phi);
    apply_any(*h, *phi, hp.o);
    // eigenvalues Re<phi|H phi>/<phi|phi> and, on request, |H phi - eig phi|^2 (energy.hpp:80-89): one pass over
    // phi and H phi for both sums of the eigenvalues, one more for the residual norms (r is never formed)
    double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * 2 * S));
    const double dv = set_volume_element(*phi);
    double2 *res = normres ? d + S : nullptr;
    if (phi->precision == INQB_F64)
      launch_eigen_sums<double>(ctx, static_cast<const double2 *>(phi->data), static_cast<const double2 *>(hp.o.data), S,
                                phi->basis->npoints, dv, d, res);
    else
      launch_eigen_sums<float>(ctx, static_cast<const float2 *>(phi->data), static_cast<const float2 *>(hp.o.data), S,
                               phi->basis->npoints, dv, d, res);
    auto v = download<double2>(ctx, d, size_t(2) * S);
    for (int s = 0; s < S; s++) eig[s] = v[s].y / v[s].x;  // overlap_diagonal_normalized, real part
    if (normres)
      for (int s = 0; s < S; s++) normres[s] = v[S + s].x;
    dev_free(ctx, d);
  });
}

int inqb_subspace_diagonalization(const inqb_hamiltonian *hc, inqb_orbitals *phi, double *eigenvalues) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phi && eigenvalues, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(phi->space == INQB_REAL_SPACE, INQB_ERR_ARG, "subspace diagonalization needs a real-space set");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    const int S = phi->nst;
    // subspace Hamiltonian <phi_i|H|phi_j> (overlap(phi, ham(phi)), subspace_diagonalization.hpp:25)
    double2 *d = static_cast<double2 *>(dev_alloc(ctx, sizeof(double2) * S * S));
    {
      TempSet hp(*phi);
      apply_any(*h, *phi, hp.o);
      overlap_dev(*phi, hp.o, d);
    }
    auto Hs = download<std::complex<double>>(ctx, d, size_t(S) * S);
    std::vector<std::complex<double>> V(size_t(S) * S);
    hermitian_eigen(S, Hs.data(), eigenvalues, V.data());
    // phi_k <- sum_j V[j][k] phi_j (operations::rotate with the eigenvectors, rotate.hpp:27-62)
    INQB_CUDA(cudaMemcpyAsync(d, V.data(), sizeof(double2) * S * S, cudaMemcpyHostToDevice, ctx.stream));
    rotate_dev(*phi, d);
    dev_free(ctx, d);
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  });
}

int inqb_exponential_in_place(const inqb_hamiltonian *hc, double re, double im, inqb_orbitals *phi, int order) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phi, INQB_ERR_ARG, "null argument");
    set_device(*h->ctx);
    exponential_in_place(*h, std::complex<double>(re, im), *phi, order);
  });
}

int inqb_exponential_2_for_1(const inqb_hamiltonian *hc, double f1_re, double f1_im, double f2_re, double f2_im,
                             inqb_orbitals *phi, inqb_orbitals *exp1, int order) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phi && exp1, INQB_ERR_ARG, "null argument");
    check_same_shape(*phi, *exp1);
    set_device(*h->ctx);
    exponential_2_for_1(*h, std::complex<double>(f1_re, f1_im), std::complex<double>(f2_re, f2_im), *phi, *exp1,
                        order);
  });
}

int inqb_density(inqb_orbitals *const *phis, int nsets, const double *const *occ, double *density_host) {
  Ctx *ctx = (phis && nsets > 0 && phis[0]) ? phis[0]->ctx : nullptr;
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && occ && density_host, INQB_ERR_ARG, "null argument");
    set_device(*ctx);
    const Basis &b = *phis[0]->basis;
    double *d = static_cast<double *>(dev_alloc(*ctx, sizeof(double) * b.npoints));
    density_dev(*ctx, phis, nsets, occ, d);
    // host or device output (cudaMemcpyDefault: the direction from the pointer)
    INQB_CUDA(cudaMemcpyAsync(density_host, d, sizeof(double) * b.npoints, cudaMemcpyDefault, ctx->stream));
    dev_free(*ctx, d);
    INQB_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int inqb_kick(inqb_orbitals *phi, const double efield_cart[3]) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(phi && efield_cart, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(phi->space == INQB_REAL_SPACE, INQB_ERR_ARG, "kick needs a real-space set");
    set_device(*phi->ctx);
    double ecov[3];
    cart_to_cov(*phi->basis, efield_cart, ecov);
    if (phi->precision == INQB_F64)
      launch_kick<double>(*phi->ctx, *phi->basis, static_cast<double2 *>(phi->data), phi->nst, ecov);
    else
      launch_kick<float>(*phi->ctx, *phi->basis, static_cast<float2 *>(phi->data), phi->nst, ecov);
  });
}

int inqb_dipole(const inqb_basis *b, const double *density_host, double dipole[3]) {
  return guarded(b ? b->ctx : nullptr, [&] {
    INQB_REQUIRE(b && density_host && dipole, INQB_ERR_ARG, "null argument");
    dipole_host(*b, density_host, dipole);
  });
}

int inqb_batch_apply(inqb_ctx *ctx, int n, inqb_hamiltonian *const *hams, const inqb_orbitals *const *ins,
                     inqb_orbitals *const *outs, int nstreams) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && n >= 0 && (n == 0 || (hams && ins && outs)), INQB_ERR_ARG, "null argument");
    set_device(*ctx);
    if (n == 0) return;
    const int K = std::max(1, std::min({nstreams, n, 32}));
    while (int(ctx->aux.size()) < K) {
      cudaStream_t st;
      INQB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      ctx->aux.push_back(st);
    }
    while (int(ctx->aux_events.size()) < K + 1) {
      cudaEvent_t ev;
      INQB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      ctx->aux_events.push_back(ev);
    }
    for (int i = 0; i < n; i++)
      INQB_REQUIRE(hams[i] && ins[i] && outs[i] && hams[i]->ctx == ctx && ins[i]->ctx == ctx && outs[i]->ctx == ctx,
                   INQB_ERR_ARG, "every system of a batch must use the batch's context");
    cudaStream_t main = ctx->stream;
    // fork: every auxiliary stream starts after the work already queued on the context's stream
    INQB_CUDA(cudaEventRecord(ctx->aux_events[0], main));
    for (int k = 0; k < K; k++) INQB_CUDA(cudaStreamWaitEvent(ctx->aux[k], ctx->aux_events[0], 0));
    try {
      // systems that share a Hamiltonian share its projection buffers: keep them on one stream
      std::vector<const inqb_hamiltonian *> seen;
      for (int i = 0; i < n; i++) {
        int slot = -1;
        for (size_t j = 0; j < seen.size(); j++)
          if (seen[j] == hams[i]) slot = int(j);
        if (slot < 0) {
          slot = int(seen.size());
          seen.push_back(hams[i]);
        }
        ctx->stream = ctx->aux[slot % K];
        apply_any(*hams[i], *ins[i], *outs[i]);
      }
    } catch (...) {
      ctx->stream = main;
      throw;
    }
    ctx->stream = main;
    // join
    for (int k = 0; k < K; k++) {
      INQB_CUDA(cudaEventRecord(ctx->aux_events[k + 1], ctx->aux[k]));
      INQB_CUDA(cudaStreamWaitEvent(main, ctx->aux_events[k + 1], 0));
    }
  });
}

int inqb_graph_capture_begin(inqb_ctx *ctx) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx, INQB_ERR_ARG, "null argument");
    set_device(*ctx);
    INQB_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  });
}

int inqb_graph_capture_end(inqb_ctx *ctx, void **graph_exec) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && graph_exec, INQB_ERR_ARG, "null argument");
    set_device(*ctx);
    cudaGraph_t g = nullptr;
    INQB_CUDA(cudaStreamEndCapture(ctx->stream, &g));
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    INQB_CUDA(e);
    *graph_exec = reinterpret_cast<void *>(ge);
  });
}

int inqb_graph_launch(inqb_ctx *ctx, void *graph_exec) {
  return guarded(ctx, [&] {
    INQB_REQUIRE(ctx && graph_exec, INQB_ERR_ARG, "null argument");
    set_device(*ctx);
    INQB_CUDA(cudaGraphLaunch(reinterpret_cast<cudaGraphExec_t>(graph_exec), ctx->stream));
  });
}

int inqb_graph_destroy(void *graph_exec) {
  if (graph_exec) cudaGraphExecDestroy(reinterpret_cast<cudaGraphExec_t>(graph_exec));
  return INQB_OK;
}

int inqb_etrs_step(const inqb_hamiltonian *hc, inqb_orbitals *const *phis, int nsets, const double *const *occ,
                   double dt, int nscf_max, double scf_threshold, double *density_host, double dipole[3],
                   int *iterations) {
  auto *h = const_cast<inqb_hamiltonian *>(hc);
  return guarded(h ? h->ctx : nullptr, [&] {
    INQB_REQUIRE(h && phis && nsets > 0 && occ, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(nscf_max >= 1, INQB_ERR_ARG, "nscf_max must be >= 1");
    set_device(*h->ctx);
    Ctx &ctx = *h->ctx;
    const Basis &b = *h->basis;
    // etrs.hpp:33-40: half step saved, full step predicted, both from one set of H^n phi
    std::vector<std::unique_ptr<TempSet>> save;
    for (int k = 0; k < nsets; k++) {
      save.emplace_back(new TempSet(*phis[k]));
      exponential_2_for_1(*h, std::complex<double>(0.0, -dt / 2.0), std::complex<double>(0.0, -dt), *phis[k],
                          save[k]->o, 4);
    }
    double *dens = static_cast<double *>(dev_alloc(ctx, sizeof(double) * b.npoints));
    double *old = static_cast<double *>(dev_alloc(ctx, sizeof(double) * b.npoints));
    double *delta_dev = static_cast<double *>(dev_alloc(ctx, sizeof(double) * 3));  // also the dipole's output
    double *delta_dev3 = delta_dev;
    density_dev(ctx, phis, nsets, occ, dens);
    // etrs.hpp:51: H(t + dt) from the predicted density (nothing to update for a fixed Hamiltonian)
    const bool interacting = h->d_vion != nullptr;
    if (interacting) update_hamiltonian_dev(*h, dens, nullptr);
    int it = 0;
    for (int iscf = 0; iscf < nscf_max; iscf++) {
      for (int k = 0; k < nsets; k++) {
        // phi = exp(-i H dt / 2) save (etrs.hpp:54-64), straight from the saved half step: no restore copy
        exponential_from(*h, std::complex<double>(0.0, -dt / 2.0), save[k]->o, *phis[k], 4);
      }
      std::swap(old, dens);
      density_dev(ctx, phis, nsets, occ, dens);
      launch_absdiff_sum(ctx, old, dens, b.npoints, delta_dev);
      double delta = 0.0;
      INQB_CUDA(cudaMemcpyAsync(&delta, delta_dev, sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
      INQB_CUDA(cudaStreamSynchronize(ctx.stream));
      delta *= b.volume / double(b.npoints);
      it = iscf + 1;
      if (interacting) update_hamiltonian_dev(*h, dens, nullptr);  // etrs.hpp:75
      if (delta < scf_threshold || iscf == nscf_max - 1) break;
    }
    if (iterations) *iterations = it;
    // the density goes to a host or a device buffer (cudaMemcpyDefault: the direction from the pointer)
    if (density_host)
      INQB_CUDA(cudaMemcpyAsync(density_host, dens, sizeof(double) * b.npoints, cudaMemcpyDefault, ctx.stream));
    if (dipole) {
      // on the device: only the three components cross to the host
      launch_dipole(ctx, b, dens, delta_dev3);
      INQB_CUDA(cudaMemcpyAsync(dipole, delta_dev3, sizeof(double) * 3, cudaMemcpyDeviceToHost, ctx.stream));
    }
    dev_free(ctx, dens);
    dev_free(ctx, old);
    dev_free(ctx, delta_dev);
    save.clear();
    INQB_CUDA(cudaStreamSynchronize(ctx.stream));
  });
}

int inqb_orbitals_save(const inqb_orbitals *phi, const char *dirname) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(phi && dirname, INQB_ERR_ARG, "null argument");
    set_device(*phi->ctx);
    std::error_code ec;
    std::filesystem::create_directories(dirname, ec);
    INQB_REQUIRE(!ec, INQB_ERR_ARG, std::string("cannot create directory '") + dirname + "'");
    if (phi->precision == INQB_F64) save_states<double>(*phi, dirname);
    else save_states<float>(*phi, dirname);
  });
}

int inqb_orbitals_load(inqb_orbitals *phi, const char *dirname) {
  return guarded(phi ? phi->ctx : nullptr, [&] {
    INQB_REQUIRE(phi && dirname, INQB_ERR_ARG, "null argument");
    INQB_REQUIRE(std::filesystem::is_directory(dirname), INQB_ERR_ARG,
                 std::string("no restart directory '") + dirname + "'");
    set_device(*phi->ctx);
    if (phi->precision == INQB_F64) load_states<double>(*phi, dirname);
    else load_states<float>(*phi, dirname);
  });
}

int inqb_field_save(const char *dirname, const double *data, long long npoint, int ncomp) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(dirname && data && npoint > 0 && ncomp > 0, INQB_ERR_ARG, "bad argument");
    std::error_code ec;
    std::filesystem::create_directories(dirname, ec);
    INQB_REQUIRE(!ec, INQB_ERR_ARG, std::string("cannot create directory '") + dirname + "'");
    std::vector<double> col(static_cast<size_t>(npoint));
    for (int c = 0; c < ncomp; c++) {
      for (long long p = 0; p < npoint; p++) col[size_t(p)] = data[size_t(p) * ncomp + c];
      write_file(std::string(dirname) + "/" + num10(c), col.data(), sizeof(double) * size_t(npoint));
    }
  });
}

int inqb_field_load(const char *dirname, double *data, long long npoint, int ncomp) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(dirname && data && npoint > 0 && ncomp > 0, INQB_ERR_ARG, "bad argument");
    std::vector<double> col(static_cast<size_t>(npoint));
    for (int c = 0; c < ncomp; c++) {
      read_file(std::string(dirname) + "/" + num10(c), col.data(), sizeof(double) * size_t(npoint));
      for (long long p = 0; p < npoint; p++) data[size_t(p) * ncomp + c] = col[size_t(p)];
    }
  });
}

int inqb_array_save(const char *dirname, const double *data, long long n) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(dirname && data && n >= 0, INQB_ERR_ARG, "bad argument");
    std::error_code ec;
    std::filesystem::create_directories(dirname, ec);
    INQB_REQUIRE(!ec, INQB_ERR_ARG, std::string("cannot create directory '") + dirname + "'");
    write_file(std::string(dirname) + "/array", data, sizeof(double) * size_t(n));
  });
}

int inqb_array_load(const char *dirname, double *data, long long n) {
  return guarded(nullptr, [&] {
    INQB_REQUIRE(dirname && data && n >= 0, INQB_ERR_ARG, "bad argument");
    read_file(std::string(dirname) + "/array", data, sizeof(double) * size_t(n));
  });
}

}  // extern "C"
