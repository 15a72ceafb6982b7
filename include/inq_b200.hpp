// inq_b200.hpp -- header-only C++ facade over the C ABI of libinqb200.so (inqb.h), with the
// names and value-returning signatures of the reference's operator API:
//
//   inq::basis::real_space          (src/basis/real_space.hpp:25-230)
//   inq::states::orbital_set        (src/states/orbital_set.hpp:18-192)
//   inq::hamiltonian::ks_hamiltonian (src/hamiltonian/ks_hamiltonian.hpp:35-275)
//   inq::operations::transform::to_fourier / to_real (src/operations/transform.hpp:186-249)
//   inq::operations::overlap_diagonal, orthogonalize, exponential (operations/*.hpp)
//   inq::real_time::etrs            (src/real_time/etrs.hpp:22-79)
//   inq::operations::io::save/load  (src/operations/io.hpp:172-215)
//   inq::eigensolvers::steepest_descent (src/eigensolvers/steepest_descent.hpp:23-86)
//
// Handles are RAII and move-only; failures throw inq::b200::error with the library's message.
// Orbital data cross the boundary as [npoint][nst] std::complex<double> (field_set::matrix()).
#pragma once

#include <array>
#include <complex>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "inqb.h"

namespace inq {
namespace b200 {

struct error : std::runtime_error {
  int code;
  error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int status, const inqb_ctx *ctx) {
  if (status != INQB_OK) throw error(status, std::string("libinqb200: ") + inqb_last_error(ctx));
}

// One device and its stream (shared by everything created from it).
class context {
  std::shared_ptr<inqb_ctx> ctx_;

 public:
  explicit context(int device = 0) {
    inqb_ctx *c = nullptr;
    check(inqb_ctx_create(device, &c), nullptr);
    ctx_.reset(c, [](inqb_ctx *p) { inqb_ctx_destroy(p); });
  }
  inqb_ctx *get() const { return ctx_.get(); }
  void synchronize() const { check(inqb_ctx_synchronize(get()), get()); }
};

}  // namespace b200

namespace systems {
// cell lattice vectors as rows, cartesian bohr (systems::cell)
struct cell {
  std::array<std::array<double, 3>, 3> lattice;
  static cell cubic(double a) { return cell{{{{a, 0, 0}, {0, a, 0}, {0, 0, a}}}}; }
};
}  // namespace systems

namespace basis {

class real_space {
  b200::context ctx_;
  std::shared_ptr<inqb_basis> b_;
  std::array<int, 3> sizes_;
  systems::cell cell_;

 public:
  real_space(b200::context ctx, systems::cell const &cell, std::array<int, 3> sizes)
      : ctx_(std::move(ctx)), sizes_(sizes), cell_(cell) {
    double lat[9];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) lat[3 * i + j] = cell.lattice[i][j];
    inqb_basis *p = nullptr;
    b200::check(inqb_basis_create(ctx_.get(), lat, sizes[0], sizes[1], sizes[2], &p), ctx_.get());
    b_.reset(p, [](inqb_basis *q) { inqb_basis_destroy(q); });
  }
  long size() const { return long(sizes_[0]) * sizes_[1] * sizes_[2]; }
  std::array<int, 3> const &sizes() const { return sizes_; }
  systems::cell const &cell() const { return cell_; }
  double volume_element() const {
    double dv = 0;
    b200::check(inqb_basis_volume_element(b_.get(), &dv), ctx_.get());
    return dv;
  }
  b200::context const &ctx() const { return ctx_; }
  inqb_basis *get() const { return b_.get(); }
};

}  // namespace basis

namespace states {

enum class space { real = INQB_REAL_SPACE, fourier = INQB_FOURIER_SPACE };

// orbital_set<real_space|fourier_space, complex>: device-resident [npoint][nst]
class orbital_set {
  basis::real_space basis_;
  std::unique_ptr<inqb_orbitals, int (*)(inqb_orbitals *)> o_;
  int nst_;
  std::array<double, 3> kpoint_;
  int spin_;
  int precision_;

  orbital_set(basis::real_space const &basis, inqb_orbitals *p, int nst, std::array<double, 3> kpoint, int spin_index,
              int precision)
      : basis_(basis), o_(p, inqb_orbitals_destroy), nst_(nst), kpoint_(kpoint), spin_(spin_index),
        precision_(precision) {}

 public:
  orbital_set(basis::real_space const &basis, int nst, std::array<double, 3> kpoint = {0, 0, 0}, int spin_index = 0,
              space sp = space::real, int precision = INQB_F64)
      : basis_(basis), o_(nullptr, inqb_orbitals_destroy), nst_(nst), kpoint_(kpoint), spin_(spin_index),
        precision_(precision) {
    inqb_orbitals *p = nullptr;
    b200::check(inqb_orbitals_create(basis_.ctx().get(), basis_.get(), nst, 1, kpoint.data(), spin_index, int(sp),
                                     precision, &p),
                basis_.ctx().get());
    o_.reset(p);
  }
  orbital_set(orbital_set &&) = default;
  orbital_set &operator=(orbital_set &&) = default;

  // A set over caller-owned storage of nst complex numbers per point, [npoint][nst], already on the
  // device (device memory of the context's device, or managed memory such as the reference's
  // gpu::array): no copy, and the storage is not freed with the set (inqb_orbitals_wrap).
  static orbital_set wrap(basis::real_space const &basis, void *device_data, int nst,
                          std::array<double, 3> kpoint = {0, 0, 0}, int spin_index = 0, space sp = space::real,
                          int precision = INQB_F64) {
    inqb_orbitals *p = nullptr;
    b200::check(inqb_orbitals_wrap(basis.ctx().get(), basis.get(), device_data, nst, 1, kpoint.data(), spin_index,
                                   int(sp), precision, &p),
                basis.ctx().get());
    return orbital_set(basis, p, nst, kpoint, spin_index, precision);
  }

  // a new set with the same basis, size, k-point, spin and space (orbital_set::skeleton)
  orbital_set skeleton() const { return orbital_set(basis_, nst_, kpoint_, spin_, current_space(), precision_); }
  space current_space() const {
    int sp = 0;
    b200::check(inqb_orbitals_info(o_.get(), nullptr, &sp, nullptr, nullptr), basis_.ctx().get());
    return space(sp);
  }
  int set_size() const { return nst_; }
  int local_set_size() const { return nst_; }
  std::array<double, 3> const &kpoint() const { return kpoint_; }
  int spin_index() const { return spin_; }
  basis::real_space const &basis() const { return basis_; }

  // host <-> device copies of matrix() ([npoint][nst], state fastest)
  void upload(std::vector<std::complex<double>> const &m) {
    if (precision_ != INQB_F64) throw b200::error(INQB_ERR_ARG, "upload of complex<double> needs an F64 set");
    b200::check(inqb_orbitals_upload(o_.get(), m.data()), basis_.ctx().get());
  }
  std::vector<std::complex<double>> matrix() const {
    if (precision_ != INQB_F64) throw b200::error(INQB_ERR_ARG, "matrix() of complex<double> needs an F64 set");
    std::vector<std::complex<double>> m(size_t(basis_.size()) * nst_);
    b200::check(inqb_orbitals_download(o_.get(), m.data()), basis_.ctx().get());
    return m;
  }
  void fill(std::complex<double> v) { b200::check(inqb_orbitals_fill(o_.get(), v.real(), v.imag()), basis_.ctx().get()); }
  inqb_orbitals *get() const { return o_.get(); }
};

}  // namespace states

namespace hamiltonian {

// ks_hamiltonian<PotentialType> with exchange disabled and scalar-relativistic KB projectors
class ks_hamiltonian {
  basis::real_space basis_;
  std::unique_ptr<inqb_hamiltonian, int (*)(inqb_hamiltonian *)> h_;
  std::array<double, 3> A_{{0, 0, 0}};

 public:
  explicit ks_hamiltonian(basis::real_space const &basis, int nspin = 1)
      : basis_(basis), h_(nullptr, inqb_hamiltonian_destroy) {
    inqb_hamiltonian *p = nullptr;
    b200::check(inqb_hamiltonian_create(basis_.ctx().get(), basis_.get(), nspin, &p), basis_.ctx().get());
    h_.reset(p);
  }
  // scalar_potential() assignment: [npoint][nspin]
  void scalar_potential(std::vector<double> const &v) {
    b200::check(inqb_potential_set(h_.get(), v.data()), basis_.ctx().get());
  }
  std::array<double, 3> const &uniform_vector_potential() const { return A_; }
  void uniform_vector_potential(std::array<double, 3> const &A) {
    A_ = A;
    b200::check(inqb_vector_potential_set(h_.get(), A.data()), basis_.ctx().get());
  }
  // update_projectors with the synthetic Gaussian Kleinman-Bylander projectors (l = 0, 1)
  void update_projectors_gaussian(std::vector<std::array<double, 3>> const &positions, double radius, double rc,
                                  std::vector<double> const &kb /* [natoms][4][4] */) {
    b200::check(inqb_projectors_build_gaussian(h_.get(), int(positions.size()), positions.empty() ? nullptr
                                                                                                    : positions[0].data(),
                                               radius, rc, kb.data()),
                basis_.ctx().get());
  }
  // operator()(orbital_set) -> new orbital_set (ks_hamiltonian.hpp:137-180)
  states::orbital_set operator()(states::orbital_set const &phi) const {
    states::orbital_set hphi = phi.skeleton();
    b200::check(inqb_apply(h_.get(), phi.get(), hphi.get()), basis_.ctx().get());
    return hphi;
  }
  // hphi = H phi into an existing set of the same shape (with wrapped sets: no allocation, no copy)
  void apply(states::orbital_set const &phi, states::orbital_set &hphi) const {
    b200::check(inqb_apply(h_.get(), phi.get(), hphi.get()), basis_.ctx().get());
  }
  double non_local_energy(states::orbital_set const &phi, std::vector<double> const &occupations) const {
    double e = 0;
    b200::check(inqb_non_local_energy(h_.get(), phi.get(), occupations.data(), &e), basis_.ctx().get());
    return e;
  }
  std::vector<double> kinetic_expectation_value(states::orbital_set const &phi) const {
    std::vector<double> out(phi.set_size());
    b200::check(inqb_kinetic_expectation_value(h_.get(), phi.get(), out.data()), basis_.ctx().get());
    return out;
  }
  inqb_hamiltonian *get() const { return h_.get(); }
};

}  // namespace hamiltonian

namespace operations {
namespace transform {
inline states::orbital_set to_fourier(states::orbital_set const &phi) {
  states::orbital_set f = phi.skeleton();
  b200::check(inqb_to_fourier(phi.get(), f.get()), phi.basis().ctx().get());
  return f;
}
inline states::orbital_set to_real(states::orbital_set const &fphi, bool normalize = true) {
  states::orbital_set r = fphi.skeleton();
  b200::check(inqb_to_real(fphi.get(), r.get(), normalize ? 1 : 0), fphi.basis().ctx().get());
  return r;
}
}  // namespace transform

inline std::vector<std::complex<double>> overlap_diagonal(states::orbital_set const &a, states::orbital_set const &b) {
  std::vector<std::complex<double>> out(a.set_size());
  b200::check(inqb_overlap_diagonal(a.get(), b.get(), reinterpret_cast<double *>(out.data())), a.basis().ctx().get());
  return out;
}
inline void orthogonalize(states::orbital_set &phi) {
  b200::check(inqb_orthogonalize(phi.get()), phi.basis().ctx().get());
}
namespace io {
// operations::io::save / load (io.hpp:172-215): one complex128 file per state in dirname
inline void save(std::string const &dirname, states::orbital_set const &phi) {
  b200::check(inqb_orbitals_save(phi.get(), dirname.c_str()), phi.basis().ctx().get());
}
inline void load(std::string const &dirname, states::orbital_set &phi) {
  b200::check(inqb_orbitals_load(phi.get(), dirname.c_str()), phi.basis().ctx().get());
}
}  // namespace io
inline void exponential_in_place(hamiltonian::ks_hamiltonian const &ham, std::complex<double> factor,
                                 states::orbital_set &phi, int order = 4) {
  b200::check(inqb_exponential_in_place(ham.get(), factor.real(), factor.imag(), phi.get(), order),
              phi.basis().ctx().get());
}
}  // namespace operations

namespace eigensolvers {
// eigensolvers::steepest_descent with the TPA preconditioner, then orthogonalize (steepest_descent.hpp:23-86);
// fphi is a Fourier-space set
inline void steepest_descent(hamiltonian::ks_hamiltonian const &ham, states::orbital_set &fphi) {
  b200::check(inqb_steepest_descent(ham.get(), fphi.get()), fphi.basis().ctx().get());
}
}  // namespace eigensolvers

namespace real_time {
// one ETRS step of one orbital set with a fixed Hamiltonian; returns the electronic dipole
inline std::array<double, 3> etrs(hamiltonian::ks_hamiltonian const &ham, states::orbital_set &phi,
                                  std::vector<double> const &occupations, double dt) {
  inqb_orbitals *sets[1] = {phi.get()};
  const double *occ[1] = {occupations.data()};
  std::array<double, 3> dip{};
  int iters = 0;
  b200::check(inqb_etrs_step(ham.get(), sets, 1, occ, dt, 5, 5e-5, nullptr, dip.data(), &iters),
              phi.basis().ctx().get());
  return dip;
}
}  // namespace real_time

}  // namespace inq
