// Sphere point lists and synthetic projector values (sphere.cpp).
#pragma once

#include <array>
#include <vector>

#include "inqb_internal.h"

namespace inqb {

struct SphereList {
  std::vector<std::array<int, 3>> points;     // grid indices in [0, n)
  std::vector<float> distance;                // |r - R| (float32, spherical_grid.hpp:41)
  std::vector<std::array<float, 3>> relpos;   // contravariant r - R (float32, spherical_grid.hpp:42)
};

// One periodic image of a sphere centre and the cube of grid points (symmetric-range indices
// lo .. lo + dim - 1 per axis, x-major, z fastest) that contains its sphere.
struct SphereCube {
  double re[3];
  int lo[3];
  int dim[3];
};

// The images of `center` within the grid diagonal and their containing cubes (empty cubes dropped),
// in the order the sphere's points are listed.
void sphere_cubes(const Basis &b, const double center[3], double radius, std::vector<SphereCube> &cubes);
void spherical_grid_build(const Basis &b, const double center[3], double radius, SphereList &out);
void gaussian_projector_values(const Basis &b, const SphereList &sph, double rc, std::vector<double> &mat);

}  // namespace inqb
