// Host-side setup of libinqb200: cell metric, FFT plans and twiddles, atom-centred
// spheres and the packed projector tables.  Compiled without floating-point
// contraction (-ffp-contract=off) so the sphere point selection reproduces the
// reference's arithmetic (spherical_grid.hpp:96-135) bit for bit.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <unordered_map>

#include "inqb_internal.h"

namespace inqb {

// ------------------------------------------------------------------ metric (systems/cell.hpp:37-53,146-215)

static inline void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

void basis_metric(const double lattice[9], double lat[3][3], double rec[3][3], double rlat[3][3], double &volume) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) lat[i][j] = lattice[3 * i + j];
  double c[3];
  cross3(lat[1], lat[2], c);
  volume = dot3(lat[0], c);
  INQB_REQUIRE(volume >= 1e-10, INQB_ERR_ARG, "the lattice volume is not positive");
  const double two_pi = 2.0 * M_PI;
  const double pref = two_pi / volume;
  cross3(lat[1], lat[2], c);
  for (int j = 0; j < 3; j++) rec[0][j] = pref * c[j];
  cross3(lat[2], lat[0], c);
  for (int j = 0; j < 3; j++) rec[1][j] = pref * c[j];
  cross3(lat[0], lat[1], c);
  for (int j = 0; j < 3; j++) rec[2][j] = pref * c[j];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) rlat[i][j] = rec[i][j] / two_pi;
}

// ------------------------------------------------------------------ FFT plans

std::vector<int> fft_radices(int n) {
  INQB_REQUIRE(n >= 1, INQB_ERR_ARG, "grid size must be positive");
  std::vector<int> r;
  int m = n;
  while (m % 8 == 0) { r.push_back(8); m /= 8; }
  while (m % 4 == 0) { r.push_back(4); m /= 4; }
  while (m % 2 == 0) { r.push_back(2); m /= 2; }
  for (int p : {3, 5, 7})
    while (m % p == 0) { r.push_back(p); m /= p; }
  INQB_REQUIRE(m == 1, INQB_ERR_UNSUPPORTED,
               "grid size " + std::to_string(n) + " is not a product of 2, 3, 5 and 7");
  return r;
}

// ------------------------------------------------------------------ kernel attributes

// Raise a kernel's dynamic shared-memory limit to at least `bytes`.  Host threads driving
// different contexts may launch the same kernel; the limit only ever grows, under a lock, so a
// launch never finds it lowered by another thread.
void ensure_smem_attr(const void *kernel, size_t bytes) {
  static std::mutex mtx;
  static std::unordered_map<const void *, size_t> current;
  std::lock_guard<std::mutex> lock(mtx);
  size_t &cur = current[kernel];
  if (bytes > cur) {
    INQB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    cur = bytes;
  }
}

// volume element of a set's basis: Omega / N in real space (real_space.hpp:216-218), Omega / N^2 in
// Fourier space (fourier_space.hpp:48-50, the forward transform being unnormalised)
double set_volume_element(const Orbitals &o) {
  const double n = double(o.basis->npoints);
  return o.space == INQB_FOURIER_SPACE ? o.basis->volume / (n * n) : o.basis->volume / n;
}

// ------------------------------------------------------------------ scratch memory

namespace {
std::atomic<long long> g_device_allocs{0};
}

void note_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }
long long device_alloc_count() { return g_device_allocs.load(std::memory_order_relaxed); }

void *dev_alloc(Ctx &ctx, size_t bytes) {
  void *p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = counted_malloc_async(&p, bytes, ctx.stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw Error(INQB_ERR_MEMORY, std::string("device allocation of ") + std::to_string(bytes) +
                                     " bytes failed: " + cudaGetErrorString(e));
  }
  return p;
}

void dev_free(Ctx &ctx, void *p) {
  if (p) INQB_CUDA(cudaFreeAsync(p, ctx.stream));
}

}  // namespace inqb
