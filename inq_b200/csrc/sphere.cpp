// Atom-centred sphere point lists and the synthetic Kleinman-Bylander projectors.
//
// spherical_grid_build follows basis/spherical_grid.hpp:59-160 (with
// basis/containing_cube.hpp:20-45 and ionic/periodic_replicas.hpp:22-60): the
// centre is folded into the cell, its periodic images within the grid diagonal
// are scanned over their containing cubes (x-major, z fastest), and a grid point
// is kept when |r - R|^2 <= radius^2 with r the point's symmetric-range position.
// Distances and contravariant offsets are stored as float32 as in point_data
// (spherical_grid.hpp:41-43).  The arithmetic is written in the reference's order
// and this file is compiled without FMA contraction, so the kept points match.

#include <cmath>

#include "inqb_internal.h"
#include "sphere.h"

namespace inqb {

static inline long lround_c(double x) { return std::lround(x); }

// cell_metric::to_cartesian of a contravariant vector: lat0*v0 + lat1*v1 + lat2*v2
static inline void contra_to_cart(const double lat[3][3], const double v[3], double out[3]) {
  for (int j = 0; j < 3; j++) out[j] = (lat[0][j] * v[0] + lat[1][j] * v[1]) + lat[2][j] * v[2];
}
// cell_metric::to_contravariant of a cartesian vector: rlat_k . v
static inline void cart_to_contra(const double rlat[3][3], const double v[3], double out[3]) {
  for (int k = 0; k < 3; k++) out[k] = rlat[k][0] * v[0] + rlat[k][1] * v[1] + rlat[k][2] * v[2];
}

void sphere_cubes(const Basis &b, const double center[3], double radius, std::vector<SphereCube> &cubes) {
  cubes.clear();
  const double(*lat)[3] = b.lat;
  const double(*rlat)[3] = b.rlat;
  double rlen[3];
  for (int i = 0; i < 3; i++) rlen[i] = std::sqrt(lat[i][0] * lat[i][0] + lat[i][1] * lat[i][1] + lat[i][2] * lat[i][2]);
  const double range = std::sqrt(rlen[0] * rlen[0] + rlen[1] * rlen[1] + rlen[2] * rlen[2]);

  // periodic_replicas: fold the centre into the cell (cell.hpp:236-250)
  double crys[3], pos[3];
  cart_to_contra(rlat, center, crys);
  for (int d = 0; d < 3; d++) {
    crys[d] -= std::floor(crys[d]);
    if (crys[d] >= 0.5) crys[d] -= 1.0;
  }
  contra_to_cart(lat, crys, pos);
  std::vector<std::array<double, 3>> reps;
  reps.push_back({pos[0], pos[1], pos[2]});
  int nmax[3];
  for (int d = 0; d < 3; d++)
    nmax[d] = 1 + int(lround_c(range / std::sqrt(lat[d][0] * lat[d][0] + lat[d][1] * lat[d][1] + lat[d][2] * lat[d][2])));
  for (int ix = -nmax[0]; ix <= nmax[0]; ix++)
    for (int iy = -nmax[1]; iy <= nmax[1]; iy++)
      for (int iz = -nmax[2]; iz <= nmax[2]; iz++) {
        if (ix == 0 && iy == 0 && iz == 0) continue;
        std::array<double, 3> r;
        for (int j = 0; j < 3; j++) r[j] = ((pos[j] + ix * lat[0][j]) + iy * lat[1][j]) + iz * lat[2][j];
        reps.push_back(r);
      }

  const double conspacing[3] = {1.0 / b.n[0], 1.0 / b.n[1], 1.0 / b.n[2]};
  for (const auto &re : reps) {
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
      // containing_cube (containing_cube.hpp:23-43) with the stored reciprocal vector
      const double *recv = b.rec[d];
      const double lrec = std::sqrt(recv[0] * recv[0] + recv[1] * recv[1] + recv[2] * recv[2]);
      const double sc = radius / lrec;
      double lointer[3], hiinter[3];
      for (int j = 0; j < 3; j++) {
        lointer[j] = re[j] - sc * recv[j];
        hiinter[j] = re[j] + sc * recv[j];
      }
      const double dlo = rlat[d][0] * lointer[0] + rlat[d][1] * lointer[1] + rlat[d][2] * lointer[2];
      const double dhi = rlat[d][0] * hiinter[0] + rlat[d][1] * hiinter[1] + rlat[d][2] * hiinter[2];
      lo[d] = int(lround_c(std::floor(dlo / conspacing[d])));
      hi[d] = int(lround_c(std::ceil(dhi / conspacing[d]))) + 1;
      const int n = b.n[d];
      const int rb = -(n / 2), rend = n / 2 + n % 2;
      lo[d] = std::min(std::max(lo[d], rb), rend);
      hi[d] = std::min(std::max(hi[d], rb), rend);
    }
    if ((hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]) <= 0) continue;
    SphereCube c;
    for (int d = 0; d < 3; d++) {
      c.re[d] = re[d];
      c.lo[d] = lo[d];
      c.dim[d] = hi[d] - lo[d];
    }
    cubes.push_back(c);
  }
}

void spherical_grid_build(const Basis &b, const double center[3], double radius, SphereList &out) {
  out.points.clear();
  out.distance.clear();
  out.relpos.clear();
  const double(*lat)[3] = b.lat;
  const double(*rlat)[3] = b.rlat;
  const double conspacing[3] = {1.0 / b.n[0], 1.0 / b.n[1], 1.0 / b.n[2]};
  std::vector<SphereCube> cubes;
  sphere_cubes(b, center, radius, cubes);
  for (const SphereCube &cb : cubes) {
    const double *re = cb.re;
    const int lo[3] = {cb.lo[0], cb.lo[1], cb.lo[2]};
    const int hi[3] = {cb.lo[0] + cb.dim[0], cb.lo[1] + cb.dim[1], cb.lo[2] + cb.dim[2]};
    for (int ix = lo[0]; ix < hi[0]; ix++)
      for (int iy = lo[1]; iy < hi[1]; iy++)
        for (int iz = lo[2]; iz < hi[2]; iz++) {
          int ii[3] = {ix, iy, iz};
          int g[3];
          double contra[3];
          for (int d = 0; d < 3; d++) {
            const int n = b.n[d];
            g[d] = ii[d] < 0 ? ii[d] + n : ii[d];                       // from_symmetric_range
            const int s = g[d] >= (n + 1) / 2 ? g[d] - n : g[d];          // to_symmetric_range
            contra[d] = s * conspacing[d];
          }
          double rp[3];
          contra_to_cart(lat, contra, rp);
          double df[3] = {rp[0] - re[0], rp[1] - re[1], rp[2] - re[2]};
          const double n2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2];
          if (n2 > radius * radius) continue;
          double cp[3];
          cart_to_contra(rlat, df, cp);
          out.points.push_back({g[0], g[1], g[2]});
          out.distance.push_back(float(std::sqrt(n2)));
          out.relpos.push_back({float(cp[0]), float(cp[1]), float(cp[2])});
        }
  }
}

// Real spherical harmonics of the synthetic projectors: Y00 = 1/(2 sqrt pi),
// Y1m = sqrt(3/4pi) {y, z, x}/r for m = -1, 0, 1 (zero at r = 0).
static double ylm(int l, int m, const double c[3]) {
  if (l == 0) return 0.5 / std::sqrt(M_PI);
  const double r = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  if (!(r > 0.0)) return 0.0;
  const int comp = (m == -1) ? 1 : (m == 0 ? 2 : 0);
  return std::sqrt(3.0 / (4.0 * M_PI)) * c[comp] / r;
}

void gaussian_projector_values(const Basis &b, const SphereList &sph, double rc, std::vector<double> &mat /*[4][n]*/) {
  const size_t n = sph.points.size();
  mat.assign(4 * n, 0.0);
  for (size_t i = 0; i < n; i++) {
    const double d = double(sph.distance[i]);
    const double rad = std::exp(-(d * d) / (rc * rc));
    double v[3] = {double(sph.relpos[i][0]), double(sph.relpos[i][1]), double(sph.relpos[i][2])};
    double c[3];
    contra_to_cart(b.lat, v, c);
    // ilm order of projector.hpp:48-66: l = 0, then l = 1 with m = -1, 0, 1
    mat[0 * n + i] = rad * ylm(0, 0, c);
    mat[1 * n + i] = rad * ylm(1, -1, c);
    mat[2 * n + i] = rad * ylm(1, 0, c);
    mat[3 * n + i] = rad * ylm(1, 1, c);
  }
}

}  // namespace inqb
