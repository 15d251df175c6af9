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

struct TileBinsDev {
  double origin[3], inv_w[3];
  int dims[3];
  const uint32_t *__restrict__ starts;
  const uint32_t *__restrict__ tiles;
};

// Particle-centric traversal of the node positions within the shape radius
// of the particle at (px, py, pz) and of its periodic images (one warp per
// particle; lanes split each position tile): calls
// f(u, e0, e1, e2, r2) with e = x_u - image and r2 = |e|^2 <= radius^2. Tiles
// are found through the uniform tile bins; a tile is visited once, in the
// first bin of the overlap of its bin range and the particle's.
template <class Fn>
__device__ __forceinline__ void visit_positions_in_reach(
    const DevMesh &M, const TileBinsDev &TB, const double *__restrict__ pos, long long npos,
    const double *__restrict__ boxes, const ShapeParams &S, double px, double py, double pz,
    int lane, Fn &&f) {
  int lo_img[3], hi_img[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo_img[d] = hi_img[d] = 0;
    if (M.pmin[d] != M.pmax[d]) {
      const double pd = d == 0 ? px : (d == 1 ? py : pz);
      if (pd - S.radius < M.pmin[d]) hi_img[d] = 1;
      if (pd + S.radius > M.pmax[d]) lo_img[d] = -1;
    }
  }
  for (int iz = lo_img[2]; iz <= hi_img[2]; ++iz)
    for (int iy = lo_img[1]; iy <= hi_img[1]; ++iy)
      for (int ix = lo_img[0]; ix <= hi_img[0]; ++ix) {
        const double cc[3] = {px + ix * (M.pmax[0] - M.pmin[0]),
                              py + iy * (M.pmax[1] - M.pmin[1]),
                              pz + iz * (M.pmax[2] - M.pmin[2])};
        int b0[3], b1[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double l = floor((cc[d] - S.radius - TB.origin[d]) * TB.inv_w[d]);
          const double h = floor((cc[d] + S.radius - TB.origin[d]) * TB.inv_w[d]);
          b0[d] = (int)fmax(0.0, fmin(l, TB.dims[d] - 1.0));
          b1[d] = (int)fmax(0.0, fmin(h, TB.dims[d] - 1.0));
        }
        for (int bz = b0[2]; bz <= b1[2]; ++bz)
          for (int by = b0[1]; by <= b1[1]; ++by)
            for (int bx = b0[0]; bx <= b1[0]; ++bx) {
              const long long bid = bx + (long long)TB.dims[0] * (by + (long long)TB.dims[1] * bz);
              for (uint32_t k = TB.starts[bid]; k < TB.starts[bid + 1]; ++k) {
                const uint32_t tile = TB.tiles[k];
                const double *bx6 = boxes + 6 * (size_t)tile;
                // a tile is visited in the first bin of the overlap of its
                // bin range and the particle's bin range only
                int first[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  const double l = floor((bx6[d] - TB.origin[d]) * TB.inv_w[d]);
                  first[d] = max((int)fmax(0.0, fmin(l, TB.dims[d] - 1.0)), b0[d]);
                }
                if (bx != first[0] || by != first[1] || bz != first[2]) continue;
                double d2 = 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  const double e = fmax(0.0, fmax(bx6[d] - cc[d], cc[d] - bx6[3 + d]));
                  d2 += e * e;
                }
                if (d2 > S.radius2) continue;
                const long long p0 = (long long)tile * PRT_NODE_TILE;
                const long long p1 = min(p0 + PRT_NODE_TILE, npos);
                for (long long uu = p0 + lane; uu < p1; uu += 32) {
                  const double e0 = pos[3 * uu] - cc[0], e1 = pos[3 * uu + 1] - cc[1],
                               e2 = pos[3 * uu + 2] - cc[2];
                  const double r2 = e0 * e0 + e1 * e1 + e2 * e2;
                  if (r2 <= S.radius2) f(uu, e0, e1, e2, r2);
                }
              }
            }
      }
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
