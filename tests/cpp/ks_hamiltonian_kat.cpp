// The reference's ks_hamiltonian unit test (ks_hamiltonian.hpp:297-445) written against the C++
// facade of libinqb200: 10 bohr cube, 20^3 grid, no atoms.  Prints the checks (and that wrapped
// caller-owned device buffers give the same H|psi>) and returns non-zero when one fails.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "inq_b200.hpp"

using namespace inq;

int main() {
  b200::context ctx(0);
  basis::real_space rs(ctx, systems::cell::cubic(10.0), {20, 20, 20});
  const int nst = 6;
  const long np = rs.size();
  hamiltonian::ks_hamiltonian ham(rs);
  std::vector<double> V(np, 0.0);
  ham.scalar_potential(V);
  states::orbital_set phi(rs, nst);
  std::vector<std::complex<double>> m(size_t(np) * nst);
  auto r_of = [](int i) { return (i >= 10 ? i - 20 : i) * 0.5; };  // symmetric range, spacing 0.5

  // constant -> 0
  for (auto &x : m) x = 1.0;
  phi.upload(m);
  auto h = ham(phi).matrix();
  double diff = 0;
  for (auto &x : h) diff += std::abs(x);
  diff /= double(h.size());
  std::printf("constant: %.3e\n", diff);
  int fail = !(diff < 1e-14);

  // plane waves e^{i s k x} -> (s k)^2 / 2
  const double kk = 2.0 * M_PI / 10.0;
  for (int ix = 0; ix < 20; ix++)
    for (int iy = 0; iy < 20; iy++)
      for (int iz = 0; iz < 20; iz++)
        for (int s = 0; s < nst; s++)
          m[((size_t(ix) * 20 + iy) * 20 + iz) * nst + s] = std::polar(1.0, s * kk * r_of(ix));
  phi.upload(m);
  h = ham(phi).matrix();
  diff = 0;
  for (size_t e = 0; e < h.size(); e++) {
    const int s = int(e % nst);
    diff += std::abs(h[e] - 0.5 * (s * kk) * (s * kk) * m[e]);
  }
  diff /= double(h.size());
  std::printf("plane wave: %.3e\n", diff);
  fail |= !(diff < 1e-14);

  // harmonic oscillator: mean |H phi - 1.5 w phi| = 0.0051420503
  const double ww = 2.0;
  for (int ix = 0; ix < 20; ix++)
    for (int iy = 0; iy < 20; iy++)
      for (int iz = 0; iz < 20; iz++) {
        const double r2 = r_of(ix) * r_of(ix) + r_of(iy) * r_of(iy) + r_of(iz) * r_of(iz);
        const long p = (long(ix) * 20 + iy) * 20 + iz;
        V[p] = 0.5 * ww * ww * r2;
        for (int s = 0; s < nst; s++) m[p * nst + s] = std::exp(-ww * r2);
      }
  ham.scalar_potential(V);
  phi.upload(m);
  h = ham(phi).matrix();
  diff = 0;
  for (size_t e = 0; e < h.size(); e++) diff += std::abs(h[e] - 1.5 * ww * m[e]);
  diff /= double(h.size());
  std::printf("harmonic oscillator: %.10f (reference 0.0051420503)\n", diff);
  fail |= !(std::abs(diff - 0.0051420503) < 1.2e-5 * 0.0051420503);

  // round trip through the Fourier-space operator form
  auto hf = operations::transform::to_real(ham(operations::transform::to_fourier(phi))).matrix();
  diff = 0;
  for (size_t e = 0; e < hf.size(); e++) diff += std::abs(hf[e] - 1.5 * ww * m[e]);
  diff /= double(hf.size());
  std::printf("harmonic oscillator, fourier form: %.10f\n", diff);
  fail |= !(std::abs(diff - 0.0051420503) < 1.2e-5 * 0.0051420503);

  // zero-copy boundary: the same operator on caller-owned device buffers wrapped as orbital sets
  // gives bitwise the result of the owned sets
  const size_t bytes = size_t(np) * nst * sizeof(std::complex<double>);
  void *din = nullptr, *dout = nullptr;
  if (cudaMalloc(&din, bytes) != cudaSuccess || cudaMalloc(&dout, bytes) != cudaSuccess) {
    std::printf("cudaMalloc failed\n");
    return 1;
  }
  cudaMemcpy(din, m.data(), bytes, cudaMemcpyHostToDevice);
  {
    auto win = states::orbital_set::wrap(rs, din, nst);
    auto wout = states::orbital_set::wrap(rs, dout, nst);
    ham.apply(win, wout);
    ctx.synchronize();
  }
  std::vector<std::complex<double>> hw(size_t(np) * nst);
  cudaMemcpy(hw.data(), dout, bytes, cudaMemcpyDeviceToHost);
  size_t ndiff = 0;
  for (size_t e = 0; e < hw.size(); e++) ndiff += (hw[e] != h[e]);
  std::printf("wrapped device buffers: %zu values differ from the owned sets\n", ndiff);
  fail |= ndiff != 0;
  cudaFree(din);
  cudaFree(dout);
  return fail;
}
