// binning.cuh -- particle binning shared by the mesh and grid depositors.
//
// A deposition sums, for every target point (mesh node position or brick
// point), the contributions of the particles within the shape radius. The
// particles are binned on a uniform grid, radix-sorted by bin (stable) and
// packed into a 64-byte payload per particle in bin order; a target tile
// then streams the particles of the bins within reach of its box.
#pragma once

#include "common.cuh"
#include "handles.cuh"

namespace prt_dep {

constexpr int CHUNK = 128;    // particles staged per shared-memory round
constexpr int PAYLOAD = 8;    // doubles per staged particle
constexpr int BLOCK = 128;    // threads per deposition CTA
// particle bin width as a fraction of the shape radius: smaller bins cull
// the candidates closer to the tile grown by the radius
constexpr double BIN_FRACTION = 0.5;

struct BinGrid {
  double origin[3];
  double inv_w[3];
  double w[3];      // bin widths
  double slack[3];  // rounding allowance when culling bins by distance
  int dims[3];
  int periodic[3];
  double period[3];
  long long nbins;
};

// Particle payload: x, y, z, w, w vx, w vy, w vz, tag (tag: brick id or 0).
struct DepParticles {
  const double *__restrict__ payload;   // [count][8], bin order
  const uint32_t *__restrict__ starts;  // [nbins + 1]
};

enum Weight { W_SHAPE2 = 0, W_SHAPE_POW = 1, W_TRILINEAR = 2 };

struct ShapeParams {
  double radius, radius2, inv_radius, alpha;
  double reach[3];  // candidate reach per axis (radius, or h for trilinear)
};

__device__ __forceinline__ int bin_coord(const BinGrid &G, int d, double x) {
  double u = (x - G.origin[d]) * G.inv_w[d];
  if (!(u >= 0.0)) return 0;
  if (u >= (double)G.dims[d]) return G.dims[d] - 1;
  return min((int)u, G.dims[d] - 1);
}

// unwrapped bin index of a coordinate, unclamped (for candidate ranges)
__device__ __forceinline__ int bin_floor(const BinGrid &G, int d, double x) {
  double u = floor((x - G.origin[d]) * G.inv_w[d]);
  u = fmax(fmin(u, 1e9), -1e9);
  return (int)u;
}

__device__ __forceinline__ int floor_div(int a, int b) {
  int q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return q;
}

// Uniform bins of about `bin_width` over the box [lo, hi] (exactly one period
// on the mesh's periodic axes); `radius` (a particle's reach) must stay below
// half a period so that a ball never meets its own image.
int choose_bins(const prt_mesh *m, const double lo[3], const double hi[3], double bin_width,
                double radius, BinGrid &G, int *rc);

// Bins, sorts and packs the live particles into P (workspace scratch).
// `scale` (or NULL: q) times `normalizer` is the payload weight; `tag` (or
// NULL) fills the last payload slot.
int stage_particles(prt_workspace *ws, const BinGrid &G, long long n, const double *x,
                    const double *q, const double *v, const uint32_t *el,
                    const double *scale, double normalizer, const uint32_t *tag,
                    DepParticles &P, cudaStream_t s);

}  // namespace prt_dep
