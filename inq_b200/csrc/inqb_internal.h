// Internal declarations of libinqb200: handle structs, device helpers, launchers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/inqb.h"

namespace inqb {

// ------------------------------------------------------------------ errors

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define INQB_CUDA(call)                                                                         \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw ::inqb::Error(INQB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define INQB_REQUIRE(cond, code, msg)                     \
  do {                                                    \
    if (!(cond)) throw ::inqb::Error((code), (msg));      \
  } while (0)

// ------------------------------------------------------------------ complex

template <typename R> struct c2_of;
template <> struct c2_of<double> { using type = double2; };
template <> struct c2_of<float> { using type = float2; };
template <typename R> using C2 = typename c2_of<R>::type;

template <typename T> __host__ __device__ __forceinline__ T mk(decltype(T::x) a, decltype(T::x) b) {
  T r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename T> __host__ __device__ __forceinline__ T cadd(T a, T b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __host__ __device__ __forceinline__ T csub(T a, T b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __host__ __device__ __forceinline__ T cmul(T a, T b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __host__ __device__ __forceinline__ T cconjmul(T a, T b) {  // conj(a) * b
  return mk<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename T> __host__ __device__ __forceinline__ T cscale(T a, decltype(T::x) s) {
  return mk<T>(a.x * s, a.y * s);
}

// ------------------------------------------------------------------ handles

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;
  int num_sms = 0;           // SMs the persistent kernels size their grids for (option "grid_sms")
  int device_sms = 0;        // SMs of the device
  size_t max_smem_optin = 0;
  int *d_err = nullptr;      // device flag raised by a kernel whose bounded wait expired
  std::vector<cudaStream_t> aux;        // fork streams of batched calls
  std::vector<cudaEvent_t> aux_events;  // [0] fork point, [1..] joins
  int fft_impl = 0;          // 0: specialised TMA kernels where available, 1: generic kernel only
  int fft_stages = 0;        // shared-memory ring depth of the TMA FFT kernels (0: from the memory budget)
  int mixed_compute = 0;     // butterfly arithmetic of single-precision orbitals (see inqb_ctx_set_option)
  int overlap_tc = 1;        // overlaps of single-precision sets on the tensor cores (split BF16)
  int nl_bulk = 0;           // nonlocal kernels: 0 automatic, 1 bulk-copy forms wherever they apply, -1 never
  int fft_wide = 1;          // single-precision FFT passes without a second input: 512-byte rows (64 states)
  int fft_flat = 1;          // y and x FFT passes over flattened (point, state) columns (option fft_flat)
  int nl_project_ranges = 0; // ranges of each sphere's points in the projection (0: 16)
  int fp64_mma = 1;          // FP64 overlaps on the FP64 tensor-core path (mma.sync m8n8k4) or SIMT (0)
  int nl_apply_points = 0;   // hit points per batch of the bulk-copy nonlocal apply (0: 8)
  int nl_project_points = 0; // sphere points per stage of the bulk-copy projection (0: about 16 KB of rows)
  int stream_priority = 0;   // 0: the device's lowest stream priority, 1: its highest
  void *noalloc_partial = nullptr;  // device address of noalloc.cu's fixed partial-sum array on this device
};

struct Basis {
  Ctx *ctx = nullptr;
  double lat[3][3];      // lattice vectors a_i (rows, cartesian)
  double rlat[3][3];     // reciprocal / 2pi (cell_metric::rlat_)
  double rec[3][3];      // reciprocal vectors (cell::reciprocal)
  double volume = 0.0;
  int n[3] = {0, 0, 0};
  long long npoints = 0;
  // per-axis twiddle tables exp(-2 pi i t / n), t < n
  void *tw64[3] = {nullptr, nullptr, nullptr};
  void *tw32[3] = {nullptr, nullptr, nullptr};
  std::vector<int> radices[3];
};

struct Orbitals {
  Ctx *ctx = nullptr;
  const Basis *basis = nullptr;
  int nst = 0;
  double kpoint[3] = {0, 0, 0};
  int spin_index = 0;
  int space = INQB_REAL_SPACE;
  int precision = INQB_F64;
  void *data = nullptr;
  bool owned = true;     // false: caller memory borrowed by inqb_orbitals_wrap, never freed here
  size_t bytes() const { return size_t(basis->npoints) * nst * (precision == INQB_F64 ? 16 : 8); }
};

// Nonlocal projector tables on the device, for one (k + A).
struct Projectors {
  int nproj = 0, maxsph = 0, maxnlm = 0;
  long long total = 0;                   // sum of sphere sizes
  // host copies (packed, as given)
  std::vector<int32_t> h_points;         // [nproj][maxsph][3]
  std::vector<float> h_pos;              // [nproj][maxsph][3]
  std::vector<double> h_mat;             // [nproj][maxnlm][maxsph]
  std::vector<double> h_coeff;           // [nproj][maxnlm][maxnlm]
  std::vector<int32_t> h_npts, h_nlm;
  // device
  int *d_pt = nullptr;                   // [nproj][maxsph] flat grid index, -1 pad
  float *d_pos = nullptr;                // [nproj][maxsph][3]
  double *d_mat = nullptr;               // [nproj][4][maxsph] (nlm padded to 4)
  double *d_coeff = nullptr;             // [nproj][4][4]
  float *d_coeff32 = nullptr;
  int *d_npts = nullptr;
  int *d_offs = nullptr;                 // [npoints + 1] CSR of sphere hits per grid point
  int *d_hit = nullptr;                  // [total] (p * maxsph + i) for each hit, sorted by point then p
  int *d_hitpts = nullptr;               // [nhitpts] grid points with at least one hit, ascending
  int *d_hitp = nullptr;                 // [total] projector index of each hit
  int4 *d_hrec = nullptr;                // [nhitpts] (point, first hit, hit count, first hit's projector)
  long long nhitpts = 0;
  bool device_built = false;             // tables built on the device (no host copies of points / values)
  // (k+A)-dependent coefficient tables
  double kA[3] = {1e300, 1e300, 1e300};
  double2 *d_gcoef = nullptr;            // [nproj][maxsph][4]  dV e^{+ik.r} M
  double2 *d_hcoef = nullptr;            // [total][4]          e^{-ik.r} M
  float2 *d_gcoef32 = nullptr;
  float2 *d_hcoef32 = nullptr;
};

// What device-built projectors are made of.  Gaussian: one projector per atom, radial exp(-d^2/rc^2)
// times Y_00 and Y_1m, KB blocks kb[atom][4][4].  Radial: per species a sphere radius and ngroups
// projectors, each with up to four functions (table, l, m index) of uniform radial tables r_k = k dr.
struct DeviceProjectorSpec {
  int gaussian = 1;
  double radius = 0.0, rc = 0.0;
  std::vector<double> kb;          // Gaussian: [natoms][16]
  std::vector<int> species;        // radial: [natoms]
  std::vector<double> sradius;     // [nspecies]
  std::vector<int> ngroups;        // [nspecies]
  std::vector<int> fn;             // [groups][4][3]
  std::vector<double> gkb;         // [groups][16]
  std::vector<double> tables;      // [ntables][nr]
  int nr = 0;
  double dr = 0.0;
};

struct Hamiltonian {
  Ctx *ctx = nullptr;
  const Basis *basis = nullptr;
  int nspin = 1;
  double *d_V = nullptr;                 // [npoints][nspin]
  float *d_V32 = nullptr;
  double A[3] = {0, 0, 0};
  Projectors proj;
  // device scratch for the projections of the current apply
  void *d_projraw = nullptr, *d_projD = nullptr;
  size_t proj_bytes = 0;
  // interaction (self_consistency::update_hamiltonian): ionic potential, Hartree and LDA terms
  double *d_vion = nullptr;              // [npoints]
  int hartree = 0, xc = 0;
  // what the last device-side projector build was made of (for moving the atoms); natoms 0: none
  int dev_natoms = 0;
  DeviceProjectorSpec dev_spec;
  // kernel-option overrides (key, value) applied to the context while this Hamiltonian is applied
  std::vector<std::pair<std::string, int>> opt_overrides;
};

void free_projectors(Projectors &P, cudaStream_t st);
// spheres, projector values and per-point hit lists built on the device (setup.cu)
void build_projectors_device(Hamiltonian &h, int natoms, const double *positions, const DeviceProjectorSpec &spec);

// ------------------------------------------------------------------ launchers (kernels.cu)

// One batched 1-D FFT pass over axis `axis` of a [nx][ny][nz][S] array.
enum Prologue { PRO_NONE = 0, PRO_VPSI = 1 };
enum Epilogue { EPI_STORE = 0, EPI_FINAL_REAL = 1, EPI_LAPL_ADD = 2 };

template <typename R> struct PassArgs {
  const C2<R> *in = nullptr;
  C2<R> *out = nullptr;
  int S = 0;
  int axis = 0;
  int dir = +1;                 // +1 forward (e^{-i}), -1 backward
  int mid_kinetic = 0;          // forward, multiply by lapl factor, backward (same axis)
  int perm = 0;                 // forward: output, inverse: input in digit-reversed frequency order along the axis
  int perm_n2[3] = {0, 0, 0};   // kinetic pass: axes held in digit-reversed order (their N2), 0 = natural
  double scale = 1.0;           // applied at the store
  // lapl factor data: factor*(-|G|^2 + gc.G)
  double lap_factor = 0.0, gc[3] = {0, 0, 0};
  // final-real / prologue data
  const C2<R> *psi = nullptr;   // orbital input for V psi (real form) or lapl-add source (Fourier form)
  const R *V = nullptr;
  int nspin = 1, spin = 0;
  R vshift = R(0);
  const int *nl_offs = nullptr;
  const int *nl_hitp = nullptr;     // projector index of each hit
  const C2<R> *nl_hcoef = nullptr;
  const C2<R> *projD = nullptr;
  // Horner step of a Taylor exponential (real-space final pass): out = hbase + hc * (H v), where v is
  // the pass's orbital input; hbase may not alias `out` (the operator's intermediates live there)
  const C2<R> *hbase = nullptr;
  C2<R> hc;
};

template <typename R>
void launch_fft_pass(Ctx &ctx, const Basis &b, const PassArgs<R> &a, int prologue, int epilogue);
// specialised persistent TMA kernels (fft2.cuh); false when the pass is not covered
template <typename R> bool launch_fft2(Ctx &ctx, const Basis &b, const PassArgs<R> &a, int prologue, int epilogue);
int fft2_perm_n2(const Ctx &ctx, const Basis &b, int S, int elem_bytes, int axis);
template <> bool launch_fft2<float>(Ctx &ctx, const Basis &b, const PassArgs<float> &a, int prologue, int epilogue);
template <> bool launch_fft2<double>(Ctx &ctx, const Basis &b, const PassArgs<double> &a, int prologue, int epilogue);

template <typename R>
void launch_nl_project(Ctx &ctx, const Basis &b, const Hamiltonian &h, const C2<R> *psi, int S, C2<R> *projraw,
                       C2<R> *projD);
void launch_nl_tables(Ctx &ctx, const Basis &b, Hamiltonian &h, const double kA[3]);
template <typename R>
void launch_nl_scatter(Ctx &ctx, const Basis &b, const Hamiltonian &h, const C2<R> *projD, int S, C2<R> *out);
// out += term (scaled: out += scale * term) at the sphere points
template <typename R>
void launch_nl_apply(Ctx &ctx, const Hamiltonian &h, const C2<R> *projD, int S, C2<R> *out, bool scaled, C2<R> scale);
// Taylor terms combined: e1 = x + sum_n c1[n] u[n], e2 = x + sum_n c2[n] u[n] (n < nterms <= 8, summed in
// order n = 0, 1, ...); e1 may be null, e2 may equal x
template <typename R>
void launch_taylor_combine(Ctx &ctx, const C2<R> *x, const C2<R> *const *u, int nterms, const double2 *c1,
                           const double2 *c2, C2<R> *e1, C2<R> *e2, long long n);

template <typename R> void launch_fill(Ctx &ctx, C2<R> *p, long long n, double re, double im);
template <typename R>
void launch_axpy(Ctx &ctx, C2<R> *y, const C2<R> *x, long long n, double re, double im);
template <typename R>
void launch_laplacian(Ctx &ctx, const Basis &b, const C2<R> *in, C2<R> *out, int S, double factor,
                      const double gc[3]);
template <typename R>
void launch_overlap(Ctx &ctx, const C2<R> *a, int Sa, const C2<R> *b, int Sb, long long npoints, double dv,
                    double2 *out_dev /*[Sa][Sb]*/);
template <typename R>
void launch_overlap_diag(Ctx &ctx, const C2<R> *a, const C2<R> *b, int S, long long npoints, double dv,
                         double2 *out_dev /*[S]*/);
// ne[s] = dv (<a|a>, Re<a|b>); res (optional) [s].x = dv sum_p |b - e_s a|^2, e_s = ne[s].y / ne[s].x
template <typename R>
void launch_eigen_sums(Ctx &ctx, const C2<R> *a, const C2<R> *b, int S, long long npoints, double dv,
                       double2 *ne_dev /*[S]*/, double2 *res_dev /*[S] or null*/);
template <typename R>
void launch_rotate(Ctx &ctx, C2<R> *phi, int S, long long npoints, const double2 *Rdev);
void launch_wait_timeout(Ctx &ctx, long long limit_ns);
// dipole.hpp:24-60 of a device density [npoints]: out3_dev = dV sum_r n(r) r
void launch_dipole(Ctx &ctx, const Basis &b, const double *dens, double *out3_dev);
template <typename R>
void launch_rotate_to(Ctx &ctx, const C2<R> *in, int Sin, C2<R> *out, int Sout, long long npoints, const double2 *Rdev,
                      double2 alpha, double2 beta);
template <typename R>
void launch_density(Ctx &ctx, const C2<R> *phi, int S, long long npoints, const double *occ_dev, double *dens,
                    int accumulate);
template <typename R> void launch_kick(Ctx &ctx, const Basis &b, C2<R> *phi, int S, const double ecov[3]);
template <typename R>
void launch_shift_cvec(Ctx &ctx, C2<R> *y, const C2<R> *x, int S, long long npoints, const double2 *coef_dev,
                       double scale);
template <typename R> void launch_tpa_precondition(Ctx &ctx, const Basis &b, C2<R> *x, int S, const double *kin_dev);
// states [s0, s0 + ns) of a [np][S] set to / from contiguous complex128 rows [ns][np]
template <typename R>
void launch_extract_states(Ctx &ctx, const C2<R> *in, int S, long long np, int s0, int ns, double2 *out);
template <typename R>
void launch_insert_states(Ctx &ctx, const double2 *in, int S, long long np, int s0, int ns, C2<R> *out);
template <typename R>
void launch_shift_vec(Ctx &ctx, C2<R> *y, const C2<R> *x, int S, long long npoints, const double *coef_dev,
                      double scale);
template <typename R>
void launch_kinetic_ev(Ctx &ctx, const Basis &b, const C2<R> *fphi, int S, double factor, const double gc[3],
                       double k2, double *out_dev /*[S]*/);
void launch_absdiff_sum(Ctx &ctx, const double *a, const double *b, long long n, double *out_dev);
template <typename R>
void launch_randomize_gsphere(Ctx &ctx, const Basis &b, C2<R> *phi, int S, unsigned long long seed, double ecut);
void launch_convert(Ctx &ctx, const void *in, int in_prec, void *out, int out_prec, long long n);

// ------------------------------------------------------------------ host helpers (host.cpp)

std::vector<int> fft_radices(int n);
void basis_metric(const double lattice[9], double lat[3][3], double rec[3][3], double rlat[3][3], double &volume);

void ensure_smem_attr(const void *kernel, size_t bytes);
// volume element of a set's basis: Omega / N (real space) or Omega / N^2 (Fourier space)
double set_volume_element(const Orbitals &o);
// interacting potential (kernels.cu): real -> complex copy, Poisson factor on the Fourier grid,
// V = V_ion + V_H + V_xc with per-block energy sums (KS_BLOCKS x 4 doubles)
constexpr int KS_BLOCKS = 148;
void launch_real_to_complex(Ctx &ctx, const double *in, double2 *out, long long n);
void launch_poisson_factor(Ctx &ctx, const Basis &b, double2 *f);
void launch_ks_potential(Ctx &ctx, const double *n, const double *vion, const double2 *vh, int xc, long long np,
                         double *V, float *V32, double *partial_dev);
// S = dv a^H b of single-precision sets on the tensor cores (overlap_tc.cu); out [Sa][Sb] on the device
void launch_overlap_tc(Ctx &ctx, const float2 *a, int Sa, const float2 *b, int Sb, long long npoints, double dv,
                       double2 *out);

// Looks up the device address of the fixed array of the allocation-free entry point (noalloc.cu) and
// loads its kernels, with the context's device current; called when a context is created, so the
// array and the kernels' code are resident before the entry point's first call.
void noalloc_prepare(Ctx &ctx);

// scratch allocation on the context stream (stream-ordered pool)
void *dev_alloc(Ctx &ctx, size_t bytes);
void dev_free(Ctx &ctx, void *p);

// Every device allocation of the library goes through counted_malloc_async (or dev_alloc, which calls
// it), so inqb_device_alloc_count can report how many the process has made.
void note_device_alloc();
long long device_alloc_count();
template <typename T> cudaError_t counted_malloc_async(T **p, size_t bytes, cudaStream_t st) {
  note_device_alloc();
  return cudaMallocAsync(reinterpret_cast<void **>(p), bytes, st);
}

}  // namespace inqb

struct inqb_ctx : inqb::Ctx {};
struct inqb_basis : inqb::Basis {};
struct inqb_orbitals : inqb::Orbitals {};
struct inqb_hamiltonian : inqb::Hamiltonian {};
