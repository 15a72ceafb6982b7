// Device-side construction of the nonlocal projector tables for atoms that move
// (ks_hamiltonian::update_projectors, called from etrs.hpp:45-48 when ions move).
//
// The host only folds each atom into the cell and lists the periodic images with their
// containing cubes (sphere.cpp: a few dozen numbers per atom).  Everything per grid point runs
// here:
//   1. sphere_flag_kernel: every cell of every cube, |r - R|^2 <= radius^2
//      (spherical_grid.hpp:59-133), with the host's operation order and no contraction
//      (__dmul_rn / __dadd_rn), so the kept points are the host construction's;
//   2. sphere_rank_kernel: one CTA per atom scans its cells in cube order; a kept cell's rank is
//      its index in the sphere (the stable compaction of spherical_grid.hpp:135-146);
//   3. sphere_fill_kernel: grid index, float32 distance and contravariant offset
//      (spherical_grid.hpp:41-43) and the projector values radial(d) * Y_lm
//      (projector.hpp:57-66) into the padded tables;
//   4. the per-grid-point hit lists of the owner-computes scatter: hit counts, an exclusive scan
//      (CSR offsets), placement, and a sort of every point's short list by (projector, sphere
//      index), so the lists are the same as a stable sort by point of the hits in projector order;
//      then the list of hit points (scan of the non-empty points) and one record per hit point.
// Two small reads go back to the host: the sphere sizes (to size the padded tables) and the number
// of hit points.

#include <algorithm>
#include <cmath>

#include "inqb_internal.h"
#include "sphere.h"

namespace inqb {

namespace {

struct CubeJob {
  double re[3];      // image of the atom (cartesian)
  double r2;         // squared sphere radius of the atom
  int lo[3];         // first symmetric-range index of the cube per axis
  int dim[3];        // cube extent per axis
  long long off;     // first cell of this cube in the concatenated cell range
  int atom;
};

struct SetupGeom {
  double lat[3][3], rlat[3][3];
  double cons[3];    // 1 / n per axis
  int n[3];
};

__device__ __forceinline__ int find_job(const CubeJob *jobs, int njobs, long long c) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (jobs[mid].off <= c) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Grid index of cell c of a cube and its offset df = r - R from the image, with |df|^2, in the
// host construction's order of operations (sphere.cpp), each product and sum rounded on its own.
__device__ __forceinline__ double eval_cell(const SetupGeom &G, const CubeJob &J, long long c, int g[3], double df[3]) {
  const long long loc = c - J.off;
  const int iz = int(loc % J.dim[2]);
  const int iy = int((loc / J.dim[2]) % J.dim[1]);
  const int ix = int(loc / ((long long)J.dim[2] * J.dim[1]));
  const int ii[3] = {J.lo[0] + ix, J.lo[1] + iy, J.lo[2] + iz};
  double contra[3];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int n = G.n[d];
    g[d] = ii[d] < 0 ? ii[d] + n : ii[d];
    const int s = g[d] >= (n + 1) / 2 ? g[d] - n : g[d];
    contra[d] = __dmul_rn(double(s), G.cons[d]);
  }
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const double rp = __dadd_rn(__dadd_rn(__dmul_rn(G.lat[0][j], contra[0]), __dmul_rn(G.lat[1][j], contra[1])),
                                __dmul_rn(G.lat[2][j], contra[2]));
    df[j] = __dsub_rn(rp, J.re[j]);
  }
  return __dadd_rn(__dadd_rn(__dmul_rn(df[0], df[0]), __dmul_rn(df[1], df[1])), __dmul_rn(df[2], df[2]));
}

__global__ void sphere_flag_kernel(SetupGeom G, const CubeJob *__restrict__ jobs, int njobs, long long ncells,
                                   unsigned char *__restrict__ flag) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells; c += (long long)gridDim.x * blockDim.x) {
    const CubeJob &J = jobs[find_job(jobs, njobs, c)];
    int g[3];
    double df[3];
    const double n2 = eval_cell(G, J, c, g, df);
    flag[c] = (n2 > J.r2) ? 0 : 1;
  }
}

// Exclusive scan of one value per thread over the block (blockDim.x a multiple of 32, <= 1024);
// `total` receives the block's sum.  Uses `ws` (32 ints of shared memory).
__device__ __forceinline__ int block_exclusive_scan(int v, int *ws, int &total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s = lane < nw ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) ws[lane] = s;
  }
  __syncthreads();
  const int excl = x - v + (wid > 0 ? ws[wid - 1] : 0);
  total = ws[nw - 1];
  __syncthreads();
  return excl;
}

__global__ void sphere_rank_kernel(const long long *__restrict__ aoff, const unsigned char *__restrict__ flag,
                                   int *__restrict__ rank, int *__restrict__ count) {
  __shared__ int ws[32];
  const int a = blockIdx.x;
  const long long end = aoff[a + 1];
  int carry = 0;
  for (long long base = aoff[a]; base < end; base += blockDim.x) {
    const long long c = base + threadIdx.x;
    const int f = c < end ? flag[c] : 0;
    int tot;
    const int excl = block_exclusive_scan(f, ws, tot);
    if (f) rank[c] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0) count[a] = carry;
}

// Real spherical harmonics Y_l^m (m index mm = m + l) at a cartesian offset, zero at the origin for
// l > 0: l = 1 is (y, z, x) sqrt(3 / 4 pi) / r, l = 2 and 3 the tesseral harmonics without the
// Condon-Shortley phase (the same table as the host construction).
__device__ __forceinline__ double ylm(int l, int mm, const double c[3]) {
  const double x = c[0], y = c[1], z = c[2];
  if (l == 0) return 0.5 / sqrt(M_PI);
  const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
  if (!(r2 > 0.0)) return 0.0;
  const double r = sqrt(r2);
  if (l == 1) {
    const double k1 = sqrt(3.0 / (4.0 * M_PI));
    const double v = mm == 0 ? y : (mm == 1 ? z : x);
    return __dmul_rn(k1, v) / r;
  }
  if (l == 2) {
    const double c1 = 0.5 * sqrt(15.0 / M_PI);
    switch (mm) {
      case 0: return c1 * x * y / r2;
      case 1: return c1 * y * z / r2;
      case 2: return 0.25 * sqrt(5.0 / M_PI) * (3.0 * z * z - r2) / r2;
      case 3: return c1 * x * z / r2;
      default: return 0.25 * sqrt(15.0 / M_PI) * (x * x - y * y) / r2;
    }
  }
  const double r3 = r2 * r;
  const double a = 0.25 * sqrt(35.0 / (2.0 * M_PI)), b = 0.5 * sqrt(105.0 / M_PI);
  const double cc = 0.25 * sqrt(21.0 / (2.0 * M_PI)), d = 0.25 * sqrt(7.0 / M_PI);
  switch (mm) {
    case 0: return a * y * (3.0 * x * x - y * y) / r3;
    case 1: return b * x * y * z / r3;
    case 2: return cc * y * (5.0 * z * z - r2) / r3;
    case 3: return d * z * (5.0 * z * z - 3.0 * r2) / r3;
    case 4: return cc * x * (5.0 * z * z - r2) / r3;
    case 5: return 0.5 * b * z * (x * x - y * y) / r3;
    default: return a * x * (x * x - 3.0 * y * y) / r3;
  }
}

// Cubic convolution (Catmull-Rom) of a uniform radial table at distance d: the point before r = 0
// mirrors the table with the parity of r^l, points past the end are zero.
__device__ __forceinline__ double radial_value(const double *__restrict__ tab, int nr, double dr, int l, double d) {
  const double xx = d / dr;
  const double fk = floor(xx);
  const int k = int(fk);
  const double t = xx - fk;
  if (k >= nr) return 0.0;
  const double sg = (l & 1) ? -1.0 : 1.0;
  auto f = [&](int i) -> double {
    if (i < 0) return sg * tab[min(-i, nr - 1)];
    return i < nr ? tab[i] : 0.0;
  };
  const double fm = f(k - 1), f0 = f(k), f1 = f(k + 1), f2 = f(k + 2);
  return 0.5 * (2.0 * f0 + (f1 - fm) * t + (2.0 * fm - 5.0 * f0 + 4.0 * f1 - f2) * t * t +
                (3.0 * f0 - fm - 3.0 * f1 + f2) * t * t * t);
}

// What the projector values of a species are made of.  Gaussian mode: one projector per atom with
// exp(-d^2 / rc^2) Y_00, Y_1m.  Radial mode: ngroups projectors per atom, each with up to four
// functions (radial table index, l, m index) taken from the uniform tables.
struct FillSpec {
  int gaussian;
  double rc2;                        // Gaussian: rc^2
  const int *first_proj;             // [natoms] index of the atom's first projector
  const int *species;                // [natoms]
  const int *ngroups;                // [nspecies] projectors per atom
  const int *group_base;             // [nspecies] first group of the species in fn
  const int *fn;                     // [groups][4][3] (table, l, mm), table -1 = unused
  const double *tables;              // [ntables][nr]
  int nr;
  double dr;
};

__global__ void sphere_fill_kernel(SetupGeom G, const CubeJob *__restrict__ jobs, int njobs, long long ncells,
                                   const unsigned char *__restrict__ flag, const int *__restrict__ rank, int maxsph,
                                   FillSpec F, int *__restrict__ pt, float *__restrict__ pos, double *__restrict__ mat) {
  const double y00 = 0.5 / sqrt(M_PI);
  const double k1 = sqrt(3.0 / (4.0 * M_PI));
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < ncells; c += (long long)gridDim.x * blockDim.x) {
    if (!flag[c]) continue;
    const CubeJob &J = jobs[find_job(jobs, njobs, c)];
    int g[3];
    double df[3];
    const double n2 = eval_cell(G, J, c, g, df);
    const int a = J.atom, i = rank[c];
    const int gpt = int((static_cast<long long>(g[0]) * G.n[1] + g[1]) * G.n[2] + g[2]);
    float rel[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double cp = __dadd_rn(__dadd_rn(__dmul_rn(G.rlat[k][0], df[0]), __dmul_rn(G.rlat[k][1], df[1])),
                                  __dmul_rn(G.rlat[k][2], df[2]));
      rel[k] = float(cp);
    }
    // projector values from the stored float32 distance and offset, as the host construction does
    const double d = double(float(sqrt(n2)));
    double cc[3];
#pragma unroll
    for (int j = 0; j < 3; j++)
      cc[j] = __dadd_rn(__dadd_rn(__dmul_rn(G.lat[0][j], double(rel[0])), __dmul_rn(G.lat[1][j], double(rel[1]))),
                        __dmul_rn(G.lat[2][j], double(rel[2])));
    const int p0 = F.first_proj[a];
    const int ng = F.gaussian ? 1 : F.ngroups[F.species[a]];
    for (int gi = 0; gi < ng; gi++) {
      const size_t slot = size_t(p0 + gi) * maxsph + i;
      pt[slot] = gpt;
#pragma unroll
      for (int k = 0; k < 3; k++) pos[slot * 3 + k] = rel[k];
      const size_t mb = size_t(p0 + gi) * 4 * maxsph + i;
      if (F.gaussian) {
        const double rad = exp(-__dmul_rn(d, d) / F.rc2);
        const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(cc[0], cc[0]), __dmul_rn(cc[1], cc[1])), __dmul_rn(cc[2], cc[2])));
        const bool on = r > 0.0;
        // ilm order of projector.hpp:48-66: l = 0, then l = 1 with m = -1, 0, 1 (components y, z, x)
        mat[mb] = __dmul_rn(rad, y00);
        mat[mb + maxsph] = __dmul_rn(rad, on ? __dmul_rn(k1, cc[1]) / r : 0.0);
        mat[mb + 2 * size_t(maxsph)] = __dmul_rn(rad, on ? __dmul_rn(k1, cc[2]) / r : 0.0);
        mat[mb + 3 * size_t(maxsph)] = __dmul_rn(rad, on ? __dmul_rn(k1, cc[0]) / r : 0.0);
      } else {
        const int *fg = F.fn + size_t(F.group_base[F.species[a]] + gi) * 12;
        for (int f = 0; f < 4; f++) {
          const int ti = fg[3 * f], l = fg[3 * f + 1], mm = fg[3 * f + 2];
          mat[mb + size_t(f) * maxsph] =
              ti < 0 ? 0.0 : radial_value(F.tables + size_t(ti) * F.nr, F.nr, F.dr, l, d) * ylm(l, mm, cc);
        }
      }
    }
  }
}

__global__ void hit_count_kernel(int nproj, int maxsph, const int *__restrict__ npts, const int *__restrict__ pt,
                                 int *__restrict__ cnt) {
  const long long total = (long long)nproj * maxsph;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int p = int(e / maxsph), i = int(e % maxsph);
    if (i < npts[p]) atomicAdd(&cnt[pt[e]], 1);
  }
}

__global__ void hit_place_kernel(int nproj, int maxsph, const int *__restrict__ npts, const int *__restrict__ pt,
                                 const int *__restrict__ offs, int *__restrict__ cursor, int *__restrict__ hit) {
  const long long total = (long long)nproj * maxsph;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const int p = int(e / maxsph), i = int(e % maxsph);
    if (i < npts[p]) {
      const int q = pt[e];
      hit[offs[q] + atomicAdd(&cursor[q], 1)] = int(e);
    }
  }
}

// every point's hits in increasing (projector, sphere index) order, and the projector of each hit
__global__ void hit_sort_kernel(long long npoints, const int *__restrict__ offs, int maxsph, int *__restrict__ hit,
                                int *__restrict__ hitp, int *__restrict__ nonempty) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npoints; q += (long long)gridDim.x * blockDim.x) {
    const int b = offs[q], e = offs[q + 1];
    for (int k = b + 1; k < e; k++) {
      const int v = hit[k];
      int j = k - 1;
      while (j >= b && hit[j] > v) {
        hit[j + 1] = hit[j];
        j--;
      }
      hit[j + 1] = v;
    }
    for (int k = b; k < e; k++) hitp[k] = hit[k] / maxsph;
    nonempty[q] = e > b ? 1 : 0;
  }
}

__global__ void hit_records_kernel(long long npoints, const int *__restrict__ offs, const int *__restrict__ hitp,
                                   const int *__restrict__ nonempty, const int *__restrict__ slot,
                                   int *__restrict__ hitpts, int4 *__restrict__ hrec) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npoints; q += (long long)gridDim.x * blockDim.x) {
    if (!nonempty[q]) continue;
    const int r = slot[q], h0 = offs[q];
    hitpts[r] = int(q);
    hrec[r] = make_int4(int(q), h0, offs[q + 1] - h0, hitp[h0]);
  }
}

// ---- exclusive scan of an int array: out[0..n] (out[n] = total), three passes over 4096-element chunks
constexpr int SCAN_T = 1024, SCAN_V = 4, SCAN_CHUNK = SCAN_T * SCAN_V;

__global__ void scan_chunk_sums(const int *__restrict__ in, long long n, int *__restrict__ sums) {
  __shared__ int ws[32];
  const long long base = blockIdx.x * (long long)SCAN_CHUNK + threadIdx.x * (long long)SCAN_V;
  int s = 0;
#pragma unroll
  for (int v = 0; v < SCAN_V; v++)
    if (base + v < n) s += in[base + v];
  int tot;
  block_exclusive_scan(s, ws, tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void scan_sums(int *__restrict__ sums, int nchunks, int *__restrict__ total) {
  __shared__ int ws[32];
  int carry = 0;
  for (int base = 0; base < nchunks; base += SCAN_T) {
    const int i = base + threadIdx.x;
    const int v = i < nchunks ? sums[i] : 0;
    int tot;
    const int excl = block_exclusive_scan(v, ws, tot);
    if (i < nchunks) sums[i] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_chunks(const int *__restrict__ in, long long n, const int *__restrict__ sums, int *__restrict__ out) {
  __shared__ int ws[32];
  const long long base = blockIdx.x * (long long)SCAN_CHUNK + threadIdx.x * (long long)SCAN_V;
  int x[SCAN_V];
  int s = 0;
#pragma unroll
  for (int v = 0; v < SCAN_V; v++) {
    x[v] = base + v < n ? in[base + v] : 0;
    s += x[v];
  }
  int tot;
  int run = sums[blockIdx.x] + block_exclusive_scan(s, ws, tot);
#pragma unroll
  for (int v = 0; v < SCAN_V; v++) {
    if (base + v < n) out[base + v] = run;
    run += x[v];
  }
}

// out[0..n]: exclusive prefix sums of in[0..n-1], out[n] the total
void exclusive_scan(Ctx &ctx, const int *in, long long n, int *out) {
  const int nchunks = int((n + SCAN_CHUNK - 1) / SCAN_CHUNK);
  int *sums = static_cast<int *>(dev_alloc(ctx, sizeof(int) * std::max(1, nchunks)));
  if (nchunks > 0) {
    scan_chunk_sums<<<nchunks, SCAN_T, 0, ctx.stream>>>(in, n, sums);
    INQB_CUDA(cudaGetLastError());
  }
  scan_sums<<<1, SCAN_T, 0, ctx.stream>>>(sums, nchunks, out + n);
  INQB_CUDA(cudaGetLastError());
  if (nchunks > 0) {
    scan_chunks<<<nchunks, SCAN_T, 0, ctx.stream>>>(in, n, sums, out);
    INQB_CUDA(cudaGetLastError());
  }
  ctx.launches += nchunks > 0 ? 3 : 1;
  dev_free(ctx, sums);
}

unsigned blocks_for(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  return unsigned(std::max<long long>(1, std::min<long long>(g, 148LL * 32)));
}

}  // namespace

void build_projectors_device(Hamiltonian &h, int natoms, const double *positions, const DeviceProjectorSpec &spec) {
  Ctx &ctx = *h.ctx;
  const Basis &b = *h.basis;
  cudaStream_t st = ctx.stream;
  free_projectors(h.proj, st);
  Projectors &P = h.proj;
  P.device_built = true;
  if (natoms == 0) return;
  const bool gauss = spec.gaussian != 0;
  const int nspecies = gauss ? 0 : int(spec.ngroups.size());
  if (!gauss) {
    INQB_REQUIRE(int(spec.species.size()) == natoms, INQB_ERR_ARG, "one species index per atom expected");
    for (int a = 0; a < natoms; a++)
      INQB_REQUIRE(spec.species[a] >= 0 && spec.species[a] < nspecies, INQB_ERR_ARG, "species index out of range");
  }
  auto radius_of = [&](int a) { return gauss ? spec.radius : spec.sradius[spec.species[a]]; };
  auto groups_of = [&](int a) { return gauss ? 1 : spec.ngroups[spec.species[a]]; };

  // host: images and containing cubes of every atom; projectors (atom-major, group-minor)
  std::vector<CubeJob> jobs;
  std::vector<long long> aoff(size_t(natoms) + 1, 0);
  std::vector<int> first_proj(natoms), proj_atom;
  std::vector<SphereCube> cubes;
  long long ncells = 0;
  for (int a = 0; a < natoms; a++) {
    const double rad = radius_of(a);
    sphere_cubes(b, positions + 3 * a, rad, cubes);
    for (const SphereCube &c : cubes) {
      CubeJob j;
      for (int d = 0; d < 3; d++) {
        j.re[d] = c.re[d];
        j.lo[d] = c.lo[d];
        j.dim[d] = c.dim[d];
      }
      j.r2 = rad * rad;
      j.off = ncells;
      j.atom = a;
      jobs.push_back(j);
      ncells += (long long)c.dim[0] * c.dim[1] * c.dim[2];
    }
    aoff[size_t(a) + 1] = ncells;
    first_proj[a] = int(proj_atom.size());
    for (int g = 0; g < groups_of(a); g++) proj_atom.push_back(a);
  }
  const int nproj = int(proj_atom.size());
  SetupGeom G;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      G.lat[i][j] = b.lat[i][j];
      G.rlat[i][j] = b.rlat[i][j];
    }
  for (int d = 0; d < 3; d++) {
    G.n[d] = b.n[d];
    G.cons[d] = 1.0 / b.n[d];
  }

  const int njobs = int(jobs.size());
  CubeJob *d_jobs = static_cast<CubeJob *>(dev_alloc(ctx, sizeof(CubeJob) * std::max(1, njobs)));
  long long *d_aoff = static_cast<long long *>(dev_alloc(ctx, sizeof(long long) * aoff.size()));
  unsigned char *d_flag = static_cast<unsigned char *>(dev_alloc(ctx, std::max<long long>(1, ncells)));
  int *d_rank = static_cast<int *>(dev_alloc(ctx, sizeof(int) * std::max<long long>(1, ncells)));
  int *d_count = static_cast<int *>(dev_alloc(ctx, sizeof(int) * natoms));
  if (njobs) INQB_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(CubeJob) * njobs, cudaMemcpyHostToDevice, st));
  INQB_CUDA(cudaMemcpyAsync(d_aoff, aoff.data(), sizeof(long long) * aoff.size(), cudaMemcpyHostToDevice, st));
  if (ncells > 0) {
    sphere_flag_kernel<<<blocks_for(ncells, 256), 256, 0, st>>>(G, d_jobs, njobs, ncells, d_flag);
    INQB_CUDA(cudaGetLastError());
    ctx.launches++;
  }
  sphere_rank_kernel<<<natoms, 1024, 0, st>>>(d_aoff, d_flag, d_rank, d_count);
  INQB_CUDA(cudaGetLastError());
  ctx.launches++;
  std::vector<int> counts(natoms);
  INQB_CUDA(cudaMemcpyAsync(counts.data(), d_count, sizeof(int) * natoms, cudaMemcpyDeviceToHost, st));
  INQB_CUDA(cudaStreamSynchronize(st));
  int maxsph = 0;
  long long total = 0;
  std::vector<int> npts(nproj);
  for (int p = 0; p < nproj; p++) {
    npts[p] = counts[proj_atom[p]];
    maxsph = std::max(maxsph, npts[p]);
    total += npts[p];
  }
  INQB_REQUIRE(total < (1LL << 31), INQB_ERR_UNSUPPORTED, "too many sphere points");

  // KB blocks per projector
  std::vector<double> coeff(size_t(nproj) * 16, 0.0);
  std::vector<int> group_base(std::max(1, nspecies), 0);
  for (int s = 1; s < nspecies; s++) group_base[s] = group_base[s - 1] + spec.ngroups[s - 1];
  for (int p = 0; p < nproj; p++) {
    const int a = proj_atom[p];
    const double *src = gauss ? spec.kb.data() + size_t(a) * 16
                              : spec.gkb.data() + size_t(group_base[spec.species[a]] + (p - first_proj[a])) * 16;
    std::copy(src, src + 16, coeff.begin() + size_t(p) * 16);
  }
  P.nproj = nproj;
  P.maxsph = maxsph;
  P.maxnlm = 4;
  P.total = total;
  P.h_npts = npts;
  P.h_nlm.assign(nproj, 4);
  P.h_coeff = coeff;
  std::vector<float> coeff32(coeff.size());
  for (size_t i = 0; i < coeff.size(); i++) coeff32[i] = float(coeff[i]);
  const size_t slots = std::max<size_t>(1, size_t(nproj) * maxsph);
  INQB_CUDA(counted_malloc_async(&P.d_pt, sizeof(int) * slots, st));
  INQB_CUDA(counted_malloc_async(&P.d_pos, sizeof(float) * 3 * slots, st));
  INQB_CUDA(counted_malloc_async(&P.d_mat, sizeof(double) * 4 * slots, st));
  INQB_CUDA(counted_malloc_async(&P.d_coeff, sizeof(double) * 16 * nproj, st));
  INQB_CUDA(counted_malloc_async(&P.d_coeff32, sizeof(float) * 16 * nproj, st));
  INQB_CUDA(counted_malloc_async(&P.d_npts, sizeof(int) * nproj, st));
  INQB_CUDA(cudaMemsetAsync(P.d_pt, 0xff, sizeof(int) * slots, st));  // -1 padding
  INQB_CUDA(cudaMemsetAsync(P.d_pos, 0, sizeof(float) * 3 * slots, st));
  INQB_CUDA(cudaMemsetAsync(P.d_mat, 0, sizeof(double) * 4 * slots, st));
  INQB_CUDA(cudaMemcpyAsync(P.d_coeff, coeff.data(), sizeof(double) * 16 * nproj, cudaMemcpyHostToDevice, st));
  INQB_CUDA(cudaMemcpyAsync(P.d_coeff32, coeff32.data(), sizeof(float) * 16 * nproj, cudaMemcpyHostToDevice, st));
  INQB_CUDA(cudaMemcpyAsync(P.d_npts, npts.data(), sizeof(int) * nproj, cudaMemcpyHostToDevice, st));

  // what the values are made of
  int *d_first = static_cast<int *>(dev_alloc(ctx, sizeof(int) * natoms));
  INQB_CUDA(cudaMemcpyAsync(d_first, first_proj.data(), sizeof(int) * natoms, cudaMemcpyHostToDevice, st));
  FillSpec F{};
  F.gaussian = gauss ? 1 : 0;
  F.rc2 = spec.rc * spec.rc;
  F.first_proj = d_first;
  std::vector<void *> spec_dev;
  auto upload = [&](const void *src, size_t bytes) {
    void *d = dev_alloc(ctx, std::max<size_t>(bytes, 16));
    if (bytes) INQB_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, st));
    spec_dev.push_back(d);
    return d;
  };
  if (!gauss) {
    INQB_REQUIRE(spec.nr > 0 && spec.dr > 0.0 && spec.tables.size() % size_t(spec.nr) == 0, INQB_ERR_ARG,
                 "radial tables must hold whole rows of nr points");
    const int ntab = int(spec.tables.size() / size_t(spec.nr));
    for (size_t k = 0; k < spec.fn.size(); k += 3)
      INQB_REQUIRE(spec.fn[k] < ntab && spec.fn[k + 1] >= 0 && spec.fn[k + 1] <= 3 && spec.fn[k + 2] >= 0 &&
                       spec.fn[k + 2] <= 2 * spec.fn[k + 1],
                   INQB_ERR_ARG, "projector function (table, l, m) out of range");
    F.species = static_cast<const int *>(upload(spec.species.data(), sizeof(int) * spec.species.size()));
    F.ngroups = static_cast<const int *>(upload(spec.ngroups.data(), sizeof(int) * spec.ngroups.size()));
    F.group_base = static_cast<const int *>(upload(group_base.data(), sizeof(int) * group_base.size()));
    F.fn = static_cast<const int *>(upload(spec.fn.data(), sizeof(int) * spec.fn.size()));
    F.tables = static_cast<const double *>(upload(spec.tables.data(), sizeof(double) * spec.tables.size()));
    F.nr = spec.nr;
    F.dr = spec.dr;
  }
  if (ncells > 0) {
    sphere_fill_kernel<<<blocks_for(ncells, 256), 256, 0, st>>>(G, d_jobs, njobs, ncells, d_flag, d_rank, maxsph, F,
                                                                 P.d_pt, P.d_pos, P.d_mat);
    INQB_CUDA(cudaGetLastError());
    ctx.launches++;
  }

  // per-grid-point hit lists
  const long long np = b.npoints;
  int *d_cnt = static_cast<int *>(dev_alloc(ctx, sizeof(int) * np));
  int *d_nonempty = static_cast<int *>(dev_alloc(ctx, sizeof(int) * np));
  int *d_slot = static_cast<int *>(dev_alloc(ctx, sizeof(int) * (np + 1)));
  INQB_CUDA(counted_malloc_async(&P.d_offs, sizeof(int) * (np + 1), st));
  INQB_CUDA(counted_malloc_async(&P.d_hit, sizeof(int) * std::max<long long>(1, total), st));
  INQB_CUDA(counted_malloc_async(&P.d_hitp, sizeof(int) * std::max<long long>(1, total), st));
  INQB_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int) * np, st));
  const long long nslots = (long long)nproj * maxsph;
  hit_count_kernel<<<blocks_for(nslots, 256), 256, 0, st>>>(nproj, maxsph, P.d_npts, P.d_pt, d_cnt);
  INQB_CUDA(cudaGetLastError());
  exclusive_scan(ctx, d_cnt, np, P.d_offs);
  INQB_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int) * np, st));
  hit_place_kernel<<<blocks_for(nslots, 256), 256, 0, st>>>(nproj, maxsph, P.d_npts, P.d_pt, P.d_offs, d_cnt, P.d_hit);
  INQB_CUDA(cudaGetLastError());
  hit_sort_kernel<<<blocks_for(np, 256), 256, 0, st>>>(np, P.d_offs, maxsph, P.d_hit, P.d_hitp, d_nonempty);
  INQB_CUDA(cudaGetLastError());
  exclusive_scan(ctx, d_nonempty, np, d_slot);
  int nhit = 0;
  INQB_CUDA(cudaMemcpyAsync(&nhit, d_slot + np, sizeof(int), cudaMemcpyDeviceToHost, st));
  INQB_CUDA(cudaStreamSynchronize(st));
  P.nhitpts = nhit;
  INQB_CUDA(counted_malloc_async(&P.d_hitpts, sizeof(int) * std::max(1, nhit), st));
  INQB_CUDA(counted_malloc_async(&P.d_hrec, sizeof(int4) * std::max(1, nhit), st));
  hit_records_kernel<<<blocks_for(np, 256), 256, 0, st>>>(np, P.d_offs, P.d_hitp, d_nonempty, d_slot, P.d_hitpts,
                                                          P.d_hrec);
  INQB_CUDA(cudaGetLastError());
  ctx.launches += 4;
  INQB_CUDA(counted_malloc_async(&P.d_gcoef, sizeof(double2) * slots * 4, st));
  INQB_CUDA(counted_malloc_async(&P.d_gcoef32, sizeof(float2) * slots * 4, st));
  INQB_CUDA(counted_malloc_async(&P.d_hcoef, sizeof(double2) * std::max<long long>(1, total) * 4, st));
  INQB_CUDA(counted_malloc_async(&P.d_hcoef32, sizeof(float2) * std::max<long long>(1, total) * 4, st));
  for (void *p : {static_cast<void *>(d_jobs), static_cast<void *>(d_aoff), static_cast<void *>(d_flag),
                  static_cast<void *>(d_rank), static_cast<void *>(d_count), static_cast<void *>(d_cnt),
                  static_cast<void *>(d_nonempty), static_cast<void *>(d_slot), static_cast<void *>(d_first)})
    dev_free(ctx, p);
  for (void *p : spec_dev) dev_free(ctx, p);
  P.kA[0] = P.kA[1] = P.kA[2] = 1e300;  // (k + A) tables are built on first use
}

}  // namespace inqb
