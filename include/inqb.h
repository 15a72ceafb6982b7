/*
 * inqb.h -- C ABI of libinqb200.so, the B200 (sm_100a) implementation of the
 * Kohn-Sham Hamiltonian application H|psi> and the real-time ETRS step.
 *
 * Every entry point returns an int status (INQB_OK = 0); the message of the
 * last failure on a context is returned by inqb_last_error().  No C++
 * exception crosses this boundary.  Handles own their device memory.  A
 * context owns one CUDA stream; calls on one context are not thread-safe,
 * calls on distinct contexts are.
 *
 * Data layouts are the reference's:
 *   orbitals  [npoint][nst] complex (state index fastest; npoint = nx*ny*nz
 *             with z fastest), i.e. field_set::matrix() of
 *             src/basis/field_set.hpp:41,62, hypercubic [nx][ny][nz][nst];
 *   potential [npoint][nspin] float64 (scalar_potential(), field_set of
 *             src/hamiltonian/ks_hamiltonian.hpp:45);
 *   vectors   covariant components for k-points and the vector potential,
 *             lattice vectors as rows in cartesian bohr.
 * Complex numbers are interleaved (re, im) pairs of the orbital precision:
 * float64 pairs for INQB_F64, float32 pairs for INQB_F32.
 */
#ifndef INQB_H
#define INQB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { INQB_OK = 0, INQB_ERR_ARG = 1, INQB_ERR_CUDA = 2, INQB_ERR_STATE = 3, INQB_ERR_MEMORY = 4,
       INQB_ERR_UNSUPPORTED = 5, INQB_ERR_NUMERIC = 6, INQB_ERR_TIMEOUT = 7 };

enum { INQB_REAL_SPACE = 0, INQB_FOURIER_SPACE = 1 };   /* orbital_set<real_space|fourier_space> */
enum { INQB_F64 = 0, INQB_F32 = 1 };                    /* plain FP64 form, mixed (FP32) form */

typedef struct inqb_ctx inqb_ctx;
typedef struct inqb_basis inqb_basis;
typedef struct inqb_orbitals inqb_orbitals;
typedef struct inqb_hamiltonian inqb_hamiltonian;

/* ---- context ------------------------------------------------------------- */
/* Replaces the process-wide runtime of the reference (input/environment.hpp:27-92,
 * and the reference's GPU runtime header gpu/host.hpp:40-145): one device, one stream, explicit
 * device memory. */
int inqb_ctx_create(int device, inqb_ctx **out);
int inqb_ctx_destroy(inqb_ctx *ctx);
const char *inqb_last_error(const inqb_ctx *ctx);
/* Waits for the context's stream; returns INQB_ERR_TIMEOUT if a kernel's bounded device-side
 * wait expired since the last call (the flag is then cleared). */
int inqb_ctx_synchronize(inqb_ctx *ctx);
/* The context's CUDA stream (cudaStream_t), for callers that order their own work. */
int inqb_ctx_stream(inqb_ctx *ctx, void **stream);
/* Number of kernels this library launched on the context so far. */
int inqb_ctx_launch_count(inqb_ctx *ctx, long long *count);
/* Tuning options: "fft_impl" = 0 (specialised persistent TMA kernels where a line length
 * has one, the default) or 1 (generic kernel for every length); "mixed_compute" selects
 * the butterfly arithmetic of single-precision orbitals: 0 (default) single everywhere, with
 * the products by constants and twiddles compensated (fma with the float remainder) so that
 * they carry no rounding bias, and single-precision projector sums; 1 double everywhere; 2
 * double except the last inverse pass of H; 3 as 2 and single for the first forward pass of
 * every transform too (1-3 sum the projections in double); "fft_stages" = 0 (ring depth of the TMA
 * kernels from their shared-memory budget, the default) or 2..8 stages; "overlap_tc" = 1
 * (default: overlaps of single-precision sets -- inqb_overlap, and the ones inside
 * inqb_orthogonalize and inqb_subspace_diagonalization -- on the tensor cores as split-BF16
 * products with FP32 accumulation and an FP64 sum of the per-SM partials; 16 significant bits
 * per value, so |error of S_ij| stays near 2^-16 |a_i| |b_j| / sqrt(npoint)) or 0 (FP64 SIMT
 * products, as for double-precision sets); "grid_sms" = 0 (default: the persistent kernels size
 * their grids for every SM) or 1..#SMs (grids sized for that many SMs, leaving room on the device
 * for the kernels of other contexts, e.g. small requests next to a large one in a serving loop);
 * "stream_priority" = 0 (default, the device's lowest stream priority) or 1 (its highest: the
 * block scheduler starts this context's pending blocks first); "nl_bulk" = 0 (default: the
 * nonlocal apply, and the projection when it has at least two CTAs per SM, move whole rows of
 * states through shared memory with bulk asynchronous copies), 1 (those forms wherever a row is a
 * multiple of 16 bytes) or -1 (never: register-held gathers); "fft_wide" = 1 (default: the plain streaming
 * FFT passes of single-precision sets of at least 64 states move 512-byte rows, 64 states, in three
 * stages at one CTA per SM, unless 64-state tiles would leave more than 8 more empty states in a line's
 * last tile than 32-state tiles) or 0 (256-byte rows, 32 states, as the other passes);
 * "fft_flat" = 1 (default: the y and x passes tile the flattened [nx][ny][nz*S] and [nx][ny*nz*S] views
 * of a set, so every row holds a full tile width of (point, state) columns whatever the state count,
 * odd counts included, when nz*S elements are a multiple of 16 bytes and the state rows are not already
 * whole 512-byte rows) or 0 (tiles of one grid line times a block of states, as the z passes);
 * "fp64_mma" = 1 (default: the FP64 products of overlaps of double-precision sets and of every rotation
 * run on the FP64 tensor cores, mma.sync m8n8k4) or 0 (FP64 SIMT fused multiply-adds);
 * "nl_apply_points" = 0 (default: 8) or 1..32 hit points per batch of the bulk-copy nonlocal apply;
 * "nl_project_points" = 0 (default: about 16 KB of rows) or 1..32 sphere points per stage of the
 * bulk-copy projection; "nl_project_ranges" = 0 (default: 16) or 1..64 ranges of each sphere's points,
 * one CTA each, in the projection (the projection's summation order follows it).  Changing the priority replaces
 * the context's stream (after the work queued on it), so callers query inqb_ctx_stream again. */
int inqb_ctx_set_option(inqb_ctx *ctx, const char *key, long long value);
/* Self-test of the bounded device-side waits: queues one kernel whose wait on an mbarrier phase that
 * nothing completes runs out after limit_ns (1e6 .. 1e9) and raises the context's error flag, as an
 * expired wait of the FFT, overlap or nonlocal kernels does.  The next inqb_ctx_synchronize returns
 * INQB_ERR_TIMEOUT and clears the flag; the context stays usable.  No fault or hang is involved. */
int inqb_ctx_check_wait_timeout(inqb_ctx *ctx, long long limit_ns);
/* Number of device allocations (cudaMalloc / cudaMallocAsync) the library has made in this
 * process so far, over all contexts; a diagnostic for callers that budget device memory. */
int inqb_device_alloc_count(long long *count);
/* Free and total device memory in bytes (admission control for serving). */
int inqb_ctx_mem_info(inqb_ctx *ctx, size_t *free_bytes, size_t *total_bytes);

/* ---- basis ---------------------------------------------------------------- */
/* basis::real_space(cell, sizes) (src/basis/real_space.hpp:40-49) with its
 * reciprocal basis::fourier_space (src/basis/fourier_space.hpp:33-38, serial order). */
int inqb_basis_create(inqb_ctx *ctx, const double lattice[9], int nx, int ny, int nz, inqb_basis **out);
int inqb_basis_destroy(inqb_basis *basis);
/* real_space::volume_element (real_space.hpp:216-218). */
int inqb_basis_volume_element(const inqb_basis *basis, double *dv);

/* ---- orbital sets --------------------------------------------------------- */
/* states::orbital_set(basis, nst, spinor_dim, kpoint, spin_index, comm)
 * (src/states/orbital_set.hpp:40-48); spinor_dim must be 1. */
int inqb_orbitals_create(inqb_ctx *ctx, const inqb_basis *basis, int nst, int spinor_dim,
                         const double kpoint_cov[3], int spin_index, int space, int precision,
                         inqb_orbitals **out);
/* The same set over caller-owned storage, with no copy: the zero-copy form of the boundary, for
 * orbitals that are already on the device, e.g. field_set::matrix().data_elements() of a
 * reference orbital_set, whose gpu::array lives in CUDA managed memory prefetched to the device
 * (external_libs/gpurun/include/gpu/array.hpp:66-110).  data holds npoint*nst complex numbers of
 * `precision` in the layout [npoint][nst], 16-byte aligned, in device memory of the context's
 * device or in managed memory (prefetched to the device on the context's stream here); anything
 * else is refused with INQB_ERR_ARG.  The set borrows the storage: inqb_orbitals_destroy does not
 * free it, and the caller keeps it alive, and leaves it alone while work queued on the context
 * reads or writes it, until then. */
int inqb_orbitals_wrap(inqb_ctx *ctx, const inqb_basis *basis, void *data, int nst, int spinor_dim,
                       const double kpoint_cov[3], int spin_index, int space, int precision,
                       inqb_orbitals **out);
int inqb_orbitals_destroy(inqb_orbitals *orb);
/* Host <-> device copies of the whole set, layout [npoint][nst] in the set's precision. */
int inqb_orbitals_upload(inqb_orbitals *orb, const void *host);
int inqb_orbitals_download(const inqb_orbitals *orb, void *host);
/* Device pointer of the set's storage (npoint*nst complex of the set's precision). */
int inqb_orbitals_device_ptr(const inqb_orbitals *orb, void **ptr);
/* Device-to-device copy src -> dst (same shape and precision); field_set copy-assign. */
int inqb_orbitals_copy(const inqb_orbitals *src, inqb_orbitals *dst);
/* Fill every coefficient with (re, im) (field_set::fill, src/basis/field_set.hpp). */
int inqb_orbitals_fill(inqb_orbitals *orb, double re, double im);
/* Re-tag the basis space of a set without touching its data. */
int inqb_orbitals_set_space(inqb_orbitals *orb, int space);
int inqb_orbitals_info(const inqb_orbitals *orb, int *nst, int *space, int *precision, long long *npoint);
/* Seeded synthetic orbitals (the generator of the benchmark configurations; the
 * reference's operations::randomize, src/operations/randomize.hpp:66, uses PCG32
 * instead): Fourier coefficients N(0,1) + i N(0,1) for |G|^2/2 < ecut, zero outside,
 * from SplitMix64 counters (seed, state*npoint + point) and Box-Muller. The set is
 * tagged Fourier-space. */
int inqb_orbitals_randomize_gsphere(inqb_orbitals *orb, uint64_t seed, double ecut);
/* Element-wise precision conversion src -> dst (F64 <-> F32, same shape otherwise). */
int inqb_orbitals_convert(const inqb_orbitals *src, inqb_orbitals *dst);

/* ---- transforms ----------------------------------------------------------- */
/* operations::transform::to_fourier (src/operations/transform.hpp:186-216): unnormalised forward DFT. */
int inqb_to_fourier(const inqb_orbitals *in, inqb_orbitals *out);
/* operations::transform::to_real (src/operations/transform.hpp:220-249): backward DFT, times 1/N if normalize. */
int inqb_to_real(const inqb_orbitals *in, inqb_orbitals *out, int normalize);
/* operations::laplacian (src/operations/laplacian.hpp:59-81) on a Fourier-space set:
 * out = factor*(-|G|^2 + gradcoeff.G) * in, gradcoeff contravariant. in may equal out. */
int inqb_laplacian(const inqb_orbitals *in, inqb_orbitals *out, double factor, const double gradcoeff_contra[3]);

/* ---- Hamiltonian ---------------------------------------------------------- */
/* hamiltonian::ks_hamiltonian<PotentialType>(basis, ...) (ks_hamiltonian.hpp:92-102):
 * scalar potential zero, no projectors, exchange disabled. */
int inqb_hamiltonian_create(inqb_ctx *ctx, const inqb_basis *basis, int nspin, inqb_hamiltonian **out);
int inqb_hamiltonian_destroy(inqb_hamiltonian *ham);
/* Kernel-choice options of this Hamiltonian's applications: fft_impl, fft_stages, fft_wide, fft_flat, nl_bulk,
 * nl_apply_points, nl_project_points, nl_project_ranges and grid_sms (meanings as in inqb_ctx_set_option) take `value`
 * while an operator application through this Hamiltonian is queued, whatever the context's setting; a
 * negative value (other than nl_bulk's -1) removes the override.  Lets one batch (inqb_batch_apply) run
 * every system with the options tuned for its shape, and with grid_sms give small systems fewer SMs so
 * that the systems on the batch's streams run side by side.  No counterpart in the reference. */
int inqb_hamiltonian_set_option(inqb_hamiltonian *ham, const char *key, long long value);
/* ks_hamiltonian::scalar_potential() assignment; V is host [npoint][nspin] float64. */
int inqb_potential_set(inqb_hamiltonian *ham, const double *V);
/* ks_hamiltonian::uniform_vector_potential() assignment (covariant, ks_hamiltonian.hpp:259-264). */
int inqb_vector_potential_set(inqb_hamiltonian *ham, const double A_cov[3]);
/* The interacting part of self_consistency::update_hamiltonian (self_consistency.hpp:88-170),
 * unpolarised, static ions, no external fields.  set_interaction stores the ionic potential
 * vion [npoint] (float64) and which terms follow the density: hartree != 0 adds the Hartree
 * potential of solvers::poisson (poisson.hpp:98-104, periodic cell: 4 pi n(G)/|G|^2, G = 0
 * dropped), xc = 1 the LDA of options::theory::lda (theory.hpp:48-54: Slater exchange and
 * Perdew-Zunger 1981 correlation; xc_term.hpp:186-236), xc = 0 none.  From then on
 * inqb_etrs_step rebuilds the potential V = vion + V_H[n] + V_xc[n] from every density it forms
 * (etrs.hpp:51 and :75), so its self-consistency loop is a real one.  inqb_update_hamiltonian
 * does the same for a given density [npoint] (host, float64) and returns energies[4] = {external
 * int n vion, Hartree 1/2 int n V_H, xc int n eps_xc, int n v_xc} (NULL: not wanted).
 * set_interaction with vion = NULL removes the interaction (the potential in place stays). */
int inqb_hamiltonian_set_interaction(inqb_hamiltonian *ham, const double *vion, int hartree, int xc);
int inqb_update_hamiltonian(inqb_hamiltonian *ham, const double *density, double energies[4]);
/* projector_all packing (projector_all.hpp:40-109): padded host tables
 *   points   [nproj][maxsph][3] int32 grid indices (-1 for padding)
 *   pos      [nproj][maxsph][3] float32 contravariant offsets from the atom
 *   matrices [nproj][maxnlm][maxsph] float64 projector values
 *   coeff    [nproj][maxnlm][maxnlm] float64 KB coefficients
 *   npts     [nproj], nlm [nproj] (nlm <= 4). */
int inqb_projectors_set(inqb_hamiltonian *ham, int nproj, int maxsph, int maxnlm, const int32_t *points,
                        const float *pos, const double *matrices, const double *coeff, const int32_t *npts,
                        const int32_t *nlm);
/* ks_hamiltonian::update_projectors for the synthetic Gaussian projectors
 * (projector.hpp:38-113 + spherical_grid.hpp:59-160): one projector per atom,
 * l = 0 and l = 1 (nlm = 4), radial exp(-r^2/rc^2) on the sphere |r-R| <= radius,
 * KB coefficients kb [natoms][4][4]. positions are cartesian [natoms][3]. */
int inqb_projectors_build_gaussian(inqb_hamiltonian *ham, int natoms, const double *positions, double radius,
                                   double rc, const double *kb);
/* The same tables built on the device (spherical_grid.hpp:59-160, projector.hpp:38-66 and the
 * per-grid-point hit lists): the host only lists each atom's periodic images and their containing
 * cubes; sphere membership (with the host construction's arithmetic, so the same points), the
 * compaction in cube order, the projector values and the hit lists run as kernels.  Points, offsets,
 * sphere sizes and hit lists equal the host build's; projector values agree to the last bits of exp. */
int inqb_projectors_build_gaussian_device(inqb_hamiltonian *ham, int natoms, const double *positions, double radius,
                                          double rc, const double *kb);
/* Projectors of pseudopotentials built on the device (projector.hpp:38-101 with tabulated radial
 * functions): atom a has species species[a]; species s has a sphere of radius radius[s] and
 * ngroups[s] projectors of up to four functions each.  The groups of species 0, then 1, ... are
 *   functions [group][4][3] = (table index, l <= 3, m index 0..2l), table index -1 = unused slot
 *   kb        [group][4][4] KB block of the group
 * and a function's value at distance d and cartesian offset x is table(d) * Y_lm(x): cubic
 * convolution on the uniform grid r_k = k dr of tables [ntables][nr], real harmonics (l = 1 as
 * (y, z, x) sqrt(3/4pi)/r, l = 2, 3 tesseral).  Projector p of the result is group g of atom a,
 * atom-major. */
int inqb_projectors_build_radial(inqb_hamiltonian *ham, int natoms, const double *positions, const int32_t *species,
                                 int nspecies, const double *radius, int nr, double dr, int ntables,
                                 const double *tables, const int32_t *ngroups, const int32_t *functions,
                                 const double *kb);
/* ks_hamiltonian::update_projectors for atoms that moved (etrs.hpp:45-48): rebuilds the tables on
 * the device for new cartesian positions [natoms][3], with everything else (atom count, species,
 * radii, radial functions or Gaussian parameters, KB coefficients) of the last Gaussian or radial
 * build on this Hamiltonian. */
int inqb_projectors_move(inqb_hamiltonian *ham, const double *positions);
int inqb_projectors_info(const inqb_hamiltonian *ham, int *nproj, int *maxsph, long long *total_points);
/* Host-only (no device, no context): basis::spherical_grid(basis, center, radius)
 * (src/basis/spherical_grid.hpp:59-160).  Writes up to `capacity` points: grid indices
 * [n][3] int32, float32 distances [n] and float32 contravariant offsets [n][3] (any
 * output may be NULL); *npoints receives the full count.  Returns INQB_ERR_ARG with the
 * count set when capacity is too small. */
int inqb_spherical_grid(const double lattice[9], int nx, int ny, int nz, const double center[3], double radius,
                        long long capacity, int32_t *points, float *distance, float *relpos, long long *npoints);
/* Host copy of the packed projector tables (any pointer may be NULL). */
int inqb_projectors_get(const inqb_hamiltonian *ham, int32_t *points, float *pos, double *matrices,
                        int32_t *npts);

/* ks_hamiltonian::operator() (ks_hamiltonian.hpp:137-180): out = H in.  Real- or
 * Fourier-space form from in's space tag; out must be a distinct set of the same shape. */
int inqb_apply(const inqb_hamiltonian *ham, const inqb_orbitals *in, inqb_orbitals *out);
/* ks_hamiltonian::operator() (ks_hamiltonian.hpp:137-156) for a real-space set held in host memory:
 * host_out = H host_in, both [npoint][nst] complex of `precision` (complex128 for INQB_F64, complex64
 * for INQB_F32), with k-point kpoint_cov (NULL: Gamma) and spin spin_index.  The states go through
 * the device in blocks of block_states (0: 512-byte rows, 32 double or 64 single states): the upload
 * of the next block and the download of the previous one overlap the operator on the current block
 * (two copy streams beside the context's stream).  Page-locked host buffers give that overlap;
 * pageable ones are copied correctly but without it.  Returns when host_out is complete.  Holds two
 * input and two output blocks of device memory during the call.  The reference returns a new
 * device-resident set instead (operator() allocates its result); this is the host-buffer form of
 * the same operator. */
int inqb_apply_host(const inqb_hamiltonian *ham, int nst, const double kpoint_cov[3], int spin_index, int precision,
                    const void *host_in, void *host_out, int block_states);
/* inqb_apply_host over nsets sets of one shape (host_in[k] -> host_out[k], every output buffer distinct
 * from every input): the blocks of all sets go through one pipeline, so the upload of a set's first
 * block overlaps the download of the previous set's last block, and the copy engines stay busy from
 * the first upload to the last download.  For callers that apply one operator to many host-resident
 * sets (successive requests, or states split into several arrays).  Returns when every host_out is
 * complete.  No counterpart in the reference. */
int inqb_apply_host_many(const inqb_hamiltonian *ham, int nsets, int nst, const double kpoint_cov[3], int spin_index,
                         int precision, const void *const *host_in, void *const *host_out, int block_states);
/* ks_hamiltonian::non_local (ks_hamiltonian.hpp:106-120). */
int inqb_non_local(const inqb_hamiltonian *ham, const inqb_orbitals *in, inqb_orbitals *out);
/* ks_hamiltonian::non_local_energy (ks_hamiltonian.hpp:124-133, projector_all.hpp:306-327);
 * occupations host [nst]. */
int inqb_non_local_energy(const inqb_hamiltonian *ham, const inqb_orbitals *phi, const double *occupations,
                          double *energy);
/* ks_hamiltonian::kinetic_expectation_value (ks_hamiltonian.hpp:184-197): host out [nst]. */
int inqb_kinetic_expectation_value(const inqb_hamiltonian *ham, const inqb_orbitals *phi, double *out);

/* ---- orbital-set linear algebra ------------------------------------------- */
/* operations::overlap (overlap.hpp:26-95): S[i][j] = dV sum_r conj(a[r][i]) b[r][j]; host out
 * [nst_a][nst_b] complex128.  Single-precision sets use the tensor cores unless the context
 * option "overlap_tc" is 0. */
int inqb_overlap(const inqb_orbitals *a, const inqb_orbitals *b, double *out);
/* operations::overlap_diagonal (overlap_diagonal.hpp:25-55): host out [nst] complex128. */
int inqb_overlap_diagonal(const inqb_orbitals *a, const inqb_orbitals *b, double *out);
/* No counterpart in the reference: inqb_overlap_diagonal for callers that cannot let the
 * library allocate device memory (a serving loop whose admission control has handed all
 * device memory to resident orbital sets; latency-sensitive code that must not risk the
 * implicit synchronisation of cudaMalloc/cudaFree).  Allocates nothing: out_dev is a
 * caller-owned buffer of nst complex128 (2*nst doubles, 8-byte aligned) in device memory of
 * the sets' device or in managed memory; host memory and other devices' memory are refused
 * with INQB_ERR_ARG.  The reduction's partial sums use a fixed 2.3 MiB array inside the
 * library, placed on a device by the first inqb_ctx_create there and held until the process
 * exits.  At most 512 states; larger sets get INQB_ERR_ARG.  Asynchronous on the context's
 * stream.  All calls share the array: calls that overlap on the GPU (different streams or
 * contexts) race.  A context, and so this entry point, does not survive cudaDeviceReset. */
int inqb_overlap_diagonal_noalloc(const inqb_orbitals *a, const inqb_orbitals *b, double *out_dev);
/* operations::orthogonalize (orthogonalize.hpp:25-31): FP64 overlap, FP64 Cholesky
 * (matrix/cholesky.hpp:28-99), phi <- phi U^-1 (rotate.hpp:147-156). */
int inqb_orthogonalize(inqb_orbitals *phi);
/* eigensolvers::steepest_descent (steepest_descent.hpp:23-86) with operations::preconditioner
 * (preconditioner.hpp:24-46, Teter-Payne-Allan) on a Fourier-space set, as the ground-state loop
 * calls it (ground_state/calculator.hpp:161-174): five preconditioned line-minimisation steps per
 * state, then orthogonalize.  fphi is updated in place. */
int inqb_steepest_descent(const inqb_hamiltonian *ham, inqb_orbitals *fphi);
/* operations::shift (shift.hpp:33-43): phi += (re + i im) * chi. */
int inqb_shift(double re, double im, const inqb_orbitals *chi, inqb_orbitals *phi);
/* operations::rotate (rotate.hpp:27-62): phi <- phi R, R host [nst][nst] complex128 row-major. */
int inqb_rotate(inqb_orbitals *phi, const double *R);
/* operations::rotate with alpha and beta (rotate.hpp:83-142): rotphi <- alpha phi R + beta rotphi, R host
 * [phi.nst][rotphi.nst] complex128 row-major, alpha and beta complex (re, im).  phi and rotphi are distinct
 * sets on one basis, of one precision and space.  The state-parallel rotation multiplies the local block
 * of states by its rows of R for each destination block (rotate.hpp:38-58). */
int inqb_rotate_to(const inqb_orbitals *phi, inqb_orbitals *rotphi, const double *R, const double alpha[2],
                   const double beta[2]);
/* matrix::cholesky (matrix/cholesky.hpp:28-99) then matrix::invert_triangular (invert_triangular.hpp:20-60)
 * on the host in FP64: S [n][n] complex128 Hermitian positive definite = U^H U, X = U^-1 (upper).  The
 * matrix inqb_orthogonalize applies; a state-partitioned orthogonalize forms it from the all-reduced
 * overlap on every rank.  INQB_ERR_NUMERIC if S is not positive definite (message via
 * inqb_last_error(NULL)). */
int inqb_cholesky_inverse(int n, const double *S, double *X);
/* matrix::diagonalize (diagonalize.hpp:100-190) on the host in FP64 by cyclic Jacobi rotations: A [n][n]
 * complex128 Hermitian, read from its upper triangle; w the eigenvalues ascending, column k of the
 * row-major V [n][n] the eigenvector of w[k].  The decomposition inqb_subspace_diagonalization uses. */
int inqb_hermitian_eigen(int n, const double *A, double *w, double *V);
/* energy::calculate eigenvalue part (energy.hpp:83-89): eig[s] = Re<phi|H phi>/<phi|phi>,
 * normres[s] = <r|r> with r = H phi - eig phi.  Host outputs [nst]. */
int inqb_eigenvalues(const inqb_hamiltonian *ham, const inqb_orbitals *phi, double *eig, double *normres);

/* ---- batches of systems and CUDA graphs ------------------------------------ */
/* H|psi> for n independent systems sharing one context: system i runs
 * ks_hamiltonian::operator() of hams[i] on ins[i] -> outs[i].  The systems' operator
 * chains are forked onto up to `nstreams` auxiliary streams and joined back into the
 * context's stream, so small systems run concurrently; inside a stream capture the
 * call records one graph with parallel branches.  Batched execution has no counterpart
 * in the reference (INQ applies one ks_hamiltonian per call, ks_hamiltonian.hpp:137). */
int inqb_batch_apply(inqb_ctx *ctx, int n, inqb_hamiltonian *const *hams, const inqb_orbitals *const *ins,
                     inqb_orbitals *const *outs, int nstreams);
/* Stream capture of the context's stream into a CUDA graph: begin, then any calls on
 * the context, then end (returns an instantiated cudaGraphExec_t); launch replays it
 * on the context's stream.  Calls made during capture must not allocate: run them once
 * eagerly first (tables, projection buffers and kernel attributes are then set up). */
int inqb_graph_capture_begin(inqb_ctx *ctx);
int inqb_graph_capture_end(inqb_ctx *ctx, void **graph_exec);
int inqb_graph_launch(inqb_ctx *ctx, void *graph_exec);
int inqb_graph_destroy(void *graph_exec);

/* ground_state::subspace_diagonalization (subspace_diagonalization.hpp:21-29): H_sub =
 * <phi|H|phi> (FP64 overlap), Hermitian eigen-decomposition in FP64 (matrix::diagonalize,
 * diagonalize.hpp:100-190; here cyclic Jacobi on the host), phi rotated onto the
 * eigenvectors; eigenvalues host [nst], ascending. */
int inqb_subspace_diagonalization(const inqb_hamiltonian *ham, inqb_orbitals *phi, double *eigenvalues);

/* ---- restart files (operations/io.hpp, systems/electrons.hpp:323-380) ----------- */
/* operations::io::save(dirname, orbital_set) (io.hpp:172-189): dirname is created and gets one
 * file per state, "<state %010d>_<spinor %010d>", each holding the state's npoint complex128
 * values in grid order (x slowest), native byte order -- the layout the reference reads back.
 * Single-precision sets are widened to complex128. */
int inqb_orbitals_save(const inqb_orbitals *phi, const char *dirname);
/* operations::io::load(dirname, orbital_set) (io.hpp:192-215): reads those files into phi
 * (narrowed for single precision); INQB_ERR_ARG when the directory or a file is missing or short. */
int inqb_orbitals_load(inqb_orbitals *phi, const char *dirname);
/* io::save / io::load of a field_set<real_space, double> (io.hpp:129-169): one file per
 * component, "<component %010d>", npoint float64; data is [npoint][ncomp] on the host (the
 * spin density of electrons::save). */
int inqb_field_save(const char *dirname, const double *data, long long npoint, int ncomp);
int inqb_field_load(const char *dirname, double *data, long long npoint, int ncomp);
/* io::save / io::load of a plain array (io.hpp:112-127): dirname/array, n float64 (the
 * occupations of electrons::save). */
int inqb_array_save(const char *dirname, const double *data, long long n);
int inqb_array_load(const char *dirname, double *data, long long n);

/* ---- real time ------------------------------------------------------------ */
/* operations::exponential_in_place (exponential.hpp:21-34): phi <- sum_n (f H)^n/n! phi, f = re + i im. */
int inqb_exponential_in_place(const inqb_hamiltonian *ham, double re, double im, inqb_orbitals *phi, int order);
/* operations::exponential_2_for_1 (exponential.hpp:50-69): exp1 <- exp(f1 H) phi, phi <- exp(f2 H) phi. */
int inqb_exponential_2_for_1(const inqb_hamiltonian *ham, double f1_re, double f1_im, double f2_re,
                             double f2_im, inqb_orbitals *phi, inqb_orbitals *exp1, int order);
/* observables::density::calculate (density.hpp:78-101), non-spinor: out host or device
 * [npoint] float64 = sum over sets and states of occ |phi|^2; occupations host, per set [nst]. */
int inqb_density(inqb_orbitals *const *phis, int nsets, const double *const *occupations, double *density_host);
/* kick::zero_step (kick.hpp:58-70): phi *= exp(i E_cov . r_contra), E cartesian. */
int inqb_kick(inqb_orbitals *phi, const double efield_cart[3]);
/* observables::dipole(density) (dipole.hpp:24-40) of a host density [npoint]: dV sum r n(r). */
int inqb_dipole(const inqb_basis *basis, const double *density_host, double dipole[3]);
/* One ETRS step (real_time/etrs.hpp:22-79): all sets advanced by dt; returns the density [npoint]
 * (host or device memory of the context's device, may be NULL), the electronic dipole (may be NULL)
 * and the number of SCF iterations taken.  A Hamiltonian with an interaction
 * (inqb_hamiltonian_set_interaction) is rebuilt from every density the step forms. */
int inqb_etrs_step(const inqb_hamiltonian *ham, inqb_orbitals *const *phis, int nsets,
                   const double *const *occupations, double dt, int nscf_max, double scf_threshold,
                   double *density_host, double dipole[3], int *iterations);

#ifdef __cplusplus
}
#endif
#endif /* INQB_H */
