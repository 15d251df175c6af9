// deposit.cu -- shape-function deposition onto DG nodes and onto brick grids,
// and the grid -> mesh remap.
//
// The reference deposits particle by particle: a face-connected walk from
// the particle's element visits every element its shape ball reaches and
// scatters q S(x_node - x_p) into rho/j (dep_shape.hpp:128-149,
// element_finder.hpp:239-293). The walk reaches exactly the elements that
// intersect the ball (on a convex mesh), and S vanishes at and beyond the
// radius, so the result is the sum, over every node, of the contributions of
// every particle within one radius of it. This file computes that sum as a
// gather, which needs no floating-point atomics and is deterministic:
//
//   1. bin the particles on a uniform grid (bin width >= radius), radix sort
//      by bin (stable), gather a 64-byte payload per particle in bin order;
//   2. one CTA per tile of consecutive elements (<= 128 nodes, one node per
//      thread): stream the particles of the bins that overlap the tile box
//      grown by the radius through shared memory, cull each against the
//      bounding sphere of each element of the tile, and accumulate
//      rho, j_x, j_y, j_z in registers in fixed (bin, particle) order;
//   3. write the node sums once (coalesced).
//
// Periodic axes are handled with particle images shifted by the period, the
// same images the walk uses when it crosses a periodic face.

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "handles.cuh"

namespace {

constexpr int CHUNK = 128;      // particles staged per shared-memory round
constexpr int PAYLOAD = 8;      // doubles per staged particle
constexpr int BLOCK = 128;      // threads per deposition CTA

struct BinGrid {
  double origin[3];
  double inv_w[3];
  int dims[3];
  int periodic[3];
  double period[3];
  long long nbins;
};

// Particle payload: x, y, z, w, w vx, w vy, w vz, tag (tag: brick id or 0).
struct DepParticles {
  const double *__restrict__ payload;  // [count][8], bin order
  const uint32_t *__restrict__ starts; // [nbins + 1]
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

__global__ void bin_keys_kernel(BinGrid G, long long n, const double *__restrict__ x,
                                const uint32_t *__restrict__ el,
                                uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t key = (uint32_t)G.nbins;
  if (!el || el[i] != PRT_INVALID) {
    int b0 = bin_coord(G, 0, x[i]);
    int b1 = bin_coord(G, 1, x[n + i]);
    int b2 = bin_coord(G, 2, x[2 * n + i]);
    key = (uint32_t)(b0 + (long long)G.dims[0] * (b1 + (long long)G.dims[1] * b2));
  }
  keys[i] = key;
  vals[i] = (uint32_t)i;
}

__global__ void bin_starts_kernel(long long nbins, long long n,
                                  const uint32_t *__restrict__ sorted_keys,
                                  uint32_t *__restrict__ starts) {
  long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (b > nbins) return;
  // lower_bound of b in sorted_keys
  long long lo = 0, hi = n;
  while (lo < hi) {
    long long mid = (lo + hi) >> 1;
    if ((long long)sorted_keys[mid] < b)
      lo = mid + 1;
    else
      hi = mid;
  }
  starts[b] = (uint32_t)lo;
}

// payload in bin order; weight[i] multiplies q (plain: normaliser; normalised:
// normaliser / integral, zero for a zero integral).
__global__ void payload_kernel(long long count, const uint32_t *__restrict__ perm,
                               long long n, const double *__restrict__ x,
                               const double *__restrict__ q,
                               const double *__restrict__ v,
                               const double *__restrict__ scale, double normalizer,
                               const uint32_t *__restrict__ tag,
                               double *__restrict__ out) {
  long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= count) return;
  uint32_t i = perm[s];
  double w = scale ? scale[i] * normalizer : q[i] * normalizer;
  double *o = out + PAYLOAD * s;
  o[0] = x[i];
  o[1] = x[n + i];
  o[2] = x[2 * n + i];
  o[3] = w;
  if (v) {
    o[4] = w * v[i];
    o[5] = w * v[n + i];
    o[6] = w * v[2 * n + i];
  } else {
    o[4] = o[5] = o[6] = 0;
  }
  o[7] = tag ? (double)tag[i] : 0.0;
}

// ---------------------------------------------------------------- targets

// Tile of consecutive mesh elements; groups = elements (bounding-sphere cull).
struct MeshTarget {
  const double *__restrict__ nodes;    // [Nn][3]
  const double *__restrict__ boxes;    // [tiles][6]
  const double *__restrict__ spheres;  // [E][4]
  long long E;
  int Np;
  int tile_elements;
  long long node_count;

  __device__ int groups(long long tile) const {
    long long e0 = tile * tile_elements;
    return (int)min((long long)tile_elements, E - e0);
  }
  __device__ int items(long long tile) const { return groups(tile) * Np; }
  __device__ long long out_index(long long tile, int t) const {
    return tile * tile_elements * Np + t;
  }
  __device__ void point(long long tile, int t, double &x0, double &x1, double &x2) const {
    const double *p = nodes + 3 * out_index(tile, t);
    x0 = p[0];
    x1 = p[1];
    x2 = p[2];
  }
  __device__ int group_of(int t) const { return t / Np; }
  __device__ void box(long long tile, double lo[3], double hi[3]) const {
    const double *b = boxes + 6 * tile;
    lo[0] = b[0]; lo[1] = b[1]; lo[2] = b[2];
    hi[0] = b[3]; hi[1] = b[4]; hi[2] = b[5];
  }
  // sphere of group g: centre and squared cull radius (radius + R_e)^2
  __device__ void group_sphere(long long tile, int g, double radius, double s[4]) const {
    const double *sp = spheres + 4 * (tile * tile_elements + g);
    s[0] = sp[0];
    s[1] = sp[1];
    s[2] = sp[2];
    double r = radius + sp[3];
    s[3] = r * r;
  }
  __device__ bool tag_ok(long long, double) const { return true; }
};

// Tile of 8 x 4 x 4 points of one brick; one group (the tile box).
struct BrickTarget {
  const prt_brick *__restrict__ bricks;
  const long long *__restrict__ tile_starts;  // [bricks+1] cumulative tile counts
  int brick_count;
  int check_tag;

  __device__ int find_brick(long long tile) const {
    int b = 0;
    while (b + 1 < brick_count && tile_starts[b + 1] <= tile) ++b;
    return b;
  }
  __device__ void tile_origin(long long tile, int &b, int i0[3]) const {
    b = find_brick(tile);
    const prt_brick &B = bricks[b];
    long long local = tile - tile_starts[b];
    int tx = (B.dims[0] + 7) / 8, ty = (B.dims[1] + 3) / 4;
    i0[0] = (int)(local % tx) * 8;
    i0[1] = (int)((local / tx) % ty) * 4;
    i0[2] = (int)(local / ((long long)tx * ty)) * 4;
  }
  __device__ int groups(long long) const { return 1; }
  __device__ int items(long long) const { return 128; }
  __device__ bool valid(long long tile, int t, int &b, int idx[3]) const {
    int i0[3];
    tile_origin(tile, b, i0);
    idx[0] = i0[0] + (t & 7);
    idx[1] = i0[1] + ((t >> 3) & 3);
    idx[2] = i0[2] + (t >> 5);
    const prt_brick &B = bricks[b];
    return idx[0] < B.dims[0] && idx[1] < B.dims[1] && idx[2] < B.dims[2];
  }
  __device__ long long out_index(long long tile, int t) const {
    int b, idx[3];
    if (!valid(tile, t, b, idx)) return -1;
    const prt_brick &B = bricks[b];
    return B.start_index + idx[0] + (long long)B.dims[0] * (idx[1] + (long long)B.dims[1] * idx[2]);
  }
  __device__ void point(long long tile, int t, double &x0, double &x1, double &x2) const {
    int b, idx[3];
    valid(tile, t, b, idx);
    const prt_brick &B = bricks[b];
    x0 = B.origin[0] + B.stepwidths[0] / 2 + idx[0] * B.stepwidths[0];
    x1 = B.origin[1] + B.stepwidths[1] / 2 + idx[1] * B.stepwidths[1];
    x2 = B.origin[2] + B.stepwidths[2] / 2 + idx[2] * B.stepwidths[2];
  }
  __device__ int group_of(int) const { return 0; }
  __device__ void box(long long tile, double lo[3], double hi[3]) const {
    int b, i0[3];
    tile_origin(tile, b, i0);
    const prt_brick &B = bricks[b];
    for (int d = 0; d < 3; ++d) {
      int cnt = d == 0 ? 8 : 4;
      int last = min(i0[d] + cnt, B.dims[d]) - 1;
      lo[d] = B.origin[d] + B.stepwidths[d] / 2 + i0[d] * B.stepwidths[d];
      hi[d] = B.origin[d] + B.stepwidths[d] / 2 + last * B.stepwidths[d];
    }
  }
  __device__ void group_sphere(long long tile, int, double radius, double s[4]) const {
    double lo[3], hi[3];
    box(tile, lo, hi);
    double hx = 0.5 * (hi[0] - lo[0]), hy = 0.5 * (hi[1] - lo[1]), hz = 0.5 * (hi[2] - lo[2]);
    s[0] = lo[0] + hx;
    s[1] = lo[1] + hy;
    s[2] = lo[2] + hz;
    double r = radius + sqrt(hx * hx + hy * hy + hz * hz);
    s[3] = r * r;
  }
  __device__ bool tag_ok(long long tile, double tag) const {
    if (!check_tag) return true;
    return (long long)tag == (long long)find_brick(tile);
  }
};

enum Weight { W_SHAPE2 = 0, W_SHAPE_POW = 1, W_TRILINEAR = 2 };

struct ShapeParams {
  double radius, radius2, inv_radius, alpha;
  double reach[3];  // candidate reach per axis (radius, or h for trilinear)
};

// The gather kernel. One CTA per tile, one target point per thread.
template <class Target, int WEIGHT, bool COUNT = false>
__global__ void __launch_bounds__(BLOCK)
    gather_kernel(Target T, BinGrid G, DepParticles P, ShapeParams S,
                  double *__restrict__ rho, double *__restrict__ j, long long j_stride,
                  const prt_brick *__restrict__ tri_bricks,
                  unsigned long long *__restrict__ pair_counter) {
  __shared__ double sp[PAYLOAD][CHUNK + 1];
  __shared__ uint32_t smask[CHUNK];
  __shared__ double sph[32][4];

  const long long tile = blockIdx.x;
  const int t = threadIdx.x;
  const int ng = T.groups(tile);
  const int ni = T.items(tile);
  const bool mine = t < ni;
  long long oidx = mine ? T.out_index(tile, t) : -1;
  const bool live = mine && oidx >= 0;
  double x0 = 0, x1 = 0, x2 = 0;
  if (live) T.point(tile, t, x0, x1, x2);
  const int grp = live ? T.group_of(t) : 0;
  if (t < ng) T.group_sphere(tile, t, S.radius, sph[t]);

  // trilinear: the point's brick and index for the clamped hat weights
  int tb = 0, tidx[3] = {0, 0, 0};
  double th[3] = {1, 1, 1};
  if constexpr (WEIGHT == W_TRILINEAR) {
    if (live) {
      T.valid(tile, t, tb, tidx);
      for (int d = 0; d < 3; ++d) th[d] = tri_bricks[tb].stepwidths[d];
    }
  }

  double a_rho = 0, a_jx = 0, a_jy = 0, a_jz = 0;
  unsigned long long npairs = 0;

  double lo[3], hi[3];
  T.box(tile, lo, hi);
  int u0[3], u1[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    u0[d] = bin_floor(G, d, lo[d] - S.reach[d]);
    u1[d] = bin_floor(G, d, hi[d] + S.reach[d]);
    if (G.periodic[d]) {
      u0[d] -= 1;
      u1[d] += 1;
    } else {
      u0[d] = max(u0[d], 0);
      u1[d] = min(u1[d], G.dims[d] - 1);
    }
  }
  __syncthreads();

  for (int bz = u0[2]; bz <= u1[2]; ++bz) {
    int wz = bz, qz = 0;
    if (G.periodic[2]) { qz = floor_div(bz, G.dims[2]); wz = bz - qz * G.dims[2]; }
    const double sz = qz * G.period[2];
    for (int by = u0[1]; by <= u1[1]; ++by) {
      int wy = by, qy = 0;
      if (G.periodic[1]) { qy = floor_div(by, G.dims[1]); wy = by - qy * G.dims[1]; }
      const double sy = qy * G.period[1];
      // the x-row splits into segments of constant shift
      int bx = u0[0];
      while (bx <= u1[0]) {
        int wx = bx, qx = 0, seg_end = u1[0];
        if (G.periodic[0]) {
          qx = floor_div(bx, G.dims[0]);
          wx = bx - qx * G.dims[0];
          seg_end = min(u1[0], (qx + 1) * G.dims[0] - 1);
        }
        const double sx = qx * G.period[0];
        const long long row = (long long)G.dims[0] * (wy + (long long)G.dims[1] * wz);
        const uint32_t s0 = P.starts[row + wx];
        const uint32_t s1 = P.starts[row + wx + (seg_end - bx) + 1];
        bx = seg_end + 1;
        for (uint32_t c0 = s0; c0 < s1; c0 += CHUNK) {
          const int cnt = (int)min((uint32_t)CHUNK, s1 - c0);
          __syncthreads();
          for (int k = t; k < cnt * PAYLOAD; k += BLOCK) {
            double val = P.payload[(size_t)c0 * PAYLOAD + k];
            const int comp = k % PAYLOAD;
            if (comp == 0) val += sx;
            if (comp == 1) val += sy;
            if (comp == 2) val += sz;
            sp[comp][k / PAYLOAD] = val;
          }
          __syncthreads();
          for (int k = t; k < cnt; k += BLOCK) {
            const double px = sp[0][k], py = sp[1][k], pz = sp[2][k];
            uint32_t m = 0;
            if (T.tag_ok(tile, sp[7][k])) {
              for (int g = 0; g < ng; ++g) {
                double dx = px - sph[g][0], dy = py - sph[g][1], dz = pz - sph[g][2];
                if (dx * dx + dy * dy + dz * dz <= sph[g][3]) m |= 1u << g;
              }
            }
            smask[k] = m;
          }
          __syncthreads();
          if (live) {
            const uint32_t bit = 1u << grp;
            for (int k = 0; k < cnt; ++k) {
              if (!(smask[k] & bit)) continue;
              const double dx = x0 - sp[0][k];
              const double dy = x1 - sp[1][k];
              const double dz = x2 - sp[2][k];
              double s;
              if constexpr (WEIGHT == W_TRILINEAR) {
                // clamped hat weight per axis (edge points absorb the outside)
                double wgt = 1.0;
                const double dd[3] = {dx, dy, dz};
                const prt_brick &B = tri_bricks[tb];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  const double u = -dd[d] / th[d];  // (x_p - pt) / h
                  // edge points also take the weight of the missing neighbour
                  const bool edge = (tidx[d] == 0 && u < 0) || (tidx[d] == B.dims[d] - 1 && u > 0);
                  wgt *= edge ? 1.0 : fmax(0.0, 1.0 - fabs(u));
                }
                if (wgt == 0) continue;
                s = wgt;
              } else {
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 > S.radius2) continue;
                if (COUNT) ++npairs;
                const double rt = S.radius - r2 * S.inv_radius;
                s = WEIGHT == W_SHAPE2 ? rt * rt : pow(rt, S.alpha);
              }
              a_rho = fma(sp[3][k], s, a_rho);
              a_jx = fma(sp[4][k], s, a_jx);
              a_jy = fma(sp[5][k], s, a_jy);
              a_jz = fma(sp[6][k], s, a_jz);
            }
          }
        }
      }
    }
  }
  if (COUNT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) npairs += __shfl_down_sync(0xffffffffu, npairs, o);
    if ((t & 31) == 0 && npairs) atomicAdd(pair_counter, npairs);
  }
  if (live) {
    if (rho) rho[oidx] = a_rho;
    if (j) {
      j[oidx] = a_jx;
      j[j_stride + oidx] = a_jy;
      j[2 * j_stride + oidx] = a_jz;
    }
  }
}

// Normalising pre-pass (dep_normshape.hpp:125-199): per particle, the
// integral sum_e |J_e| sum_i w_i S(x_i - x_p) over every element with a node
// inside the ball, gathered one warp per particle over the element bins of
// the tiles; scale = q / integral (0 and a warning for a zero integral).
struct TileBins {
  double origin[3], inv_w[3];
  int dims[3];
  const uint32_t *__restrict__ starts;
  const uint32_t *__restrict__ tiles;
};

template <bool ALPHA2>
__global__ void normalize_kernel(DevMesh M, TileBins TB, const double *__restrict__ boxes,
                                 const double *__restrict__ spheres, int tile_elements,
                                 const double *__restrict__ iw, ShapeParams S,
                                 double normalizer, long long n,
                                 const double *__restrict__ x, const double *__restrict__ q,
                                 const uint32_t *__restrict__ el,
                                 double *__restrict__ scale_out,
                                 double *__restrict__ elcount_out, DevStatus *st) {
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const long long i = warp;
  if (el && el[i] == PRT_INVALID) {
    if (lane == 0) {
      scale_out[i] = 0;
      elcount_out[i] = -1;
    }
    return;
  }
  const double px = x[i], py = x[n + i], pz = x[2 * n + i];
  const int Np = M.Np;
  double integral = 0;
  int elements_hit = 0;
  // images on periodic axes
  int lo_img[3], hi_img[3];
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
        const double cx = px + ix * (M.pmax[0] - M.pmin[0]);
        const double cy = py + iy * (M.pmax[1] - M.pmin[1]);
        const double cz = pz + iz * (M.pmax[2] - M.pmin[2]);
        const double c[3] = {cx, cy, cz};
        int b0[3], b1[3];
        for (int d = 0; d < 3; ++d) {
          double l = floor((c[d] - S.radius - TB.origin[d]) * TB.inv_w[d]);
          double h = floor((c[d] + S.radius - TB.origin[d]) * TB.inv_w[d]);
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
                // dedupe: a tile is handled in the first bin of the overlap
                // of its bin range and the particle's bin range
                int first[3];
                for (int d = 0; d < 3; ++d) {
                  double l = floor((bx6[d] - TB.origin[d]) * TB.inv_w[d]);
                  int tl = (int)fmax(0.0, fmin(l, TB.dims[d] - 1.0));
                  first[d] = max(tl, b0[d]);
                }
                if (bx != first[0] || by != first[1] || bz != first[2]) continue;
                // box-ball test
                double d2 = 0;
                for (int d = 0; d < 3; ++d) {
                  double e = fmax(0.0, fmax(bx6[d] - c[d], c[d] - bx6[3 + d]));
                  d2 += e * e;
                }
                if (d2 > S.radius2) continue;
                const long long e0 = (long long)tile * tile_elements;
                const long long e1 = min(e0 + tile_elements, M.E);
                for (long long e = e0; e < e1; ++e) {
                  const double *sph = spheres + 4 * e;
                  double dx = cx - sph[0], dy = cy - sph[1], dz = cz - sph[2];
                  double rr = S.radius + sph[3];
                  if (dx * dx + dy * dy + dz * dz > rr * rr) continue;
                  double el_int = 0;
                  bool any = false;
                  for (int nd = lane; nd < Np; nd += 32) {
                    const double *xn = M.nodes + 3 * (e * Np + nd);
                    double ex = xn[0] - cx, ey = xn[1] - cy, ez = xn[2] - cz;
                    double r2 = ex * ex + ey * ey + ez * ez;
                    if (r2 <= S.radius2) {
                      double rt = S.radius - r2 * S.inv_radius;
                      double s = normalizer * (ALPHA2 ? rt * rt : pow(rt, S.alpha));
                      el_int = fma(s, iw[nd], el_int);
                      any = any || s != 0;
                    }
                  }
                  integral = fma(el_int, M.jacobians[e], integral);
                  if (__any_sync(0xffffffffu, any)) ++elements_hit;
                }
              }
            }
      }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) integral += __shfl_xor_sync(0xffffffffu, integral, o);
  if (lane == 0) {
    if (integral == 0) {
      scale_out[i] = 0;
      record_warning(st, PRT_WARN_ZERO_MASS, i);
    } else {
      scale_out[i] = q[i] / integral;
    }
    elcount_out[i] = elements_hit;
  }
}

int choose_bins(const prt_mesh *m, double reach_x, BinGrid &G, int *rc) {
  *rc = PRT_OK;
  long long nb = 1;
  for (int d = 0; d < 3; ++d) {
    const bool per = m->dev.pmin[d] != m->dev.pmax[d];
    G.periodic[d] = per;
    double lo = per ? m->dev.pmin[d] : m->box_lo[d];
    double hi = per ? m->dev.pmax[d] : m->box_hi[d];
    double ext = hi - lo;
    double w = reach_x > 0 ? reach_x : ext;
    int dims = ext > 0 ? (int)std::max(1.0, std::floor(ext / w)) : 1;
    dims = std::min(dims, 1024);
    double width = ext > 0 ? ext / dims : 1.0;
    if (per && reach_x * 2 >= ext) {
      *rc = PRT_ERR_INVALID_ARGUMENT;  // ball reaches its own image
      return 0;
    }
    G.origin[d] = lo;
    G.inv_w[d] = 1.0 / width;
    G.dims[d] = dims;
    G.period[d] = per ? ext : 0.0;
    nb *= dims;
  }
  if (nb >= (1ll << 31) - 2) {
    *rc = PRT_ERR_INVALID_ARGUMENT;
    return 0;
  }
  G.nbins = nb;
  return 1;
}

// Bins, sorts and packs the live particles; fills P. `scale` (or NULL) and
// `tag` (or NULL) feed the payload.
int stage_particles(prt_workspace *ws, const BinGrid &G, long long n, const double *x,
                    const double *q, const double *v, const uint32_t *el,
                    const double *scale, double normalizer, const uint32_t *tag,
                    DepParticles &P, long long *live_count, cudaStream_t s) {
  int rc;
  uint32_t *keys = (uint32_t *)ws_buffer(ws, PRT_WS_DEP_KEYS, 8 * (size_t)n, &rc);
  if (!keys) return rc;
  uint32_t *vals = (uint32_t *)ws_buffer(ws, PRT_WS_DEP_VALS, 8 * (size_t)n, &rc);
  if (!vals) return rc;
  uint32_t *keys_out = keys + n, *vals_out = vals + n;
  bin_keys_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(G, n, x, el, keys, vals);
  PRT_CHECK_CUDA(cudaGetLastError());
  int bits = 1;
  while ((1ll << bits) <= G.nbins) ++bits;
  size_t temp_bytes = 0;
  PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_out, vals,
                                                 vals_out, (int)n, 0, bits, s));
  void *temp = ws_buffer(ws, PRT_WS_CUB, temp_bytes, &rc);
  if (!temp) return rc;
  PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_out, vals,
                                                 vals_out, (int)n, 0, bits, s));
  uint32_t *starts =
      (uint32_t *)ws_buffer(ws, PRT_WS_DEP_BINSTARTS, 4 * (size_t)(G.nbins + 2), &rc);
  if (!starts) return rc;
  bin_starts_kernel<<<prt_grid_blocks(G.nbins + 1, 256), 256, 0, s>>>(G.nbins, n, keys_out,
                                                                      starts);
  PRT_CHECK_CUDA(cudaGetLastError());
  double *payload =
      (double *)ws_buffer(ws, PRT_WS_DEP_PARTICLES, sizeof(double) * PAYLOAD * (size_t)n, &rc);
  if (!payload) return rc;
  // all n rows are packed; rows past starts[nbins] (dead particles) are never read
  payload_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(n, vals_out, n, x, q, v, scale,
                                                         normalizer, tag, payload);
  PRT_CHECK_CUDA(cudaGetLastError());
  P.payload = payload;
  P.starts = starts;
  if (live_count) *live_count = n;
  return PRT_OK;
}

__global__ void stats_kernel(long long n, const double *__restrict__ scale,
                             const double *__restrict__ elc, double *__restrict__ out) {
  // single block: deterministic tree reduction of count/sum/sumsq/min/max
  __shared__ double sh[10][256];
  double acc[10] = {0, 0, 0, INFINITY, -INFINITY, 0, 0, 0, INFINITY, -INFINITY};
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    double c = elc[i];
    if (c < 0) continue;  // dead particle
    acc[5] += 1;
    acc[6] += c;
    acc[7] += c * c;
    acc[8] = fmin(acc[8], c);
    acc[9] = fmax(acc[9], c);
    double s = scale[i];
    if (s == 0) continue;  // zero-mass particle: skipped by the depositor
    acc[0] += 1;
    acc[1] += s;
    acc[2] += s * s;
    acc[3] = fmin(acc[3], s);
    acc[4] = fmax(acc[4], s);
  }
  for (int k = 0; k < 10; ++k) sh[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int k = 0; k < 10; ++k) {
        double a = sh[k][threadIdx.x], b = sh[k][threadIdx.x + o];
        sh[k][threadIdx.x] = (k == 3 || k == 8) ? fmin(a, b)
                             : (k == 4 || k == 9) ? fmax(a, b)
                                                  : a + b;
      }
    __syncthreads();
  }
  if (threadIdx.x < 10) out[threadIdx.x] = sh[threadIdx.x][0];
}

}  // namespace

// ------------------------------------------------------------------ tiles

int prt_mesh_build_tiles(prt_mesh *m, const prt_mesh_desc *d) {
  const long long E = d->element_count;
  const int Np = d->nodes_per_element;
  const int te = std::max(1, std::min(32, PRT_TILE_NODES / Np));
  const long long tiles = (E + te - 1) / te;
  std::vector<double> boxes(6 * (size_t)tiles), spheres(4 * (size_t)E);
  for (int a = 0; a < 3; ++a) {
    m->box_lo[a] = INFINITY;
    m->box_hi[a] = -INFINITY;
  }
  for (long long e = 0; e < E; ++e) {
    double c[3] = {0, 0, 0};
    const double *xn = d->nodes + 3 * (size_t)e * Np;
    for (int i = 0; i < Np; ++i)
      for (int a = 0; a < 3; ++a) c[a] += xn[3 * i + a];
    for (int a = 0; a < 3; ++a) c[a] /= Np;
    double r2 = 0;
    for (int i = 0; i < Np; ++i) {
      double s = 0;
      for (int a = 0; a < 3; ++a) s += (xn[3 * i + a] - c[a]) * (xn[3 * i + a] - c[a]);
      r2 = std::max(r2, s);
    }
    for (int a = 0; a < 3; ++a) spheres[4 * e + a] = c[a];
    // a little slack so that rounding never culls a node inside the ball
    spheres[4 * e + 3] = std::sqrt(r2) * (1 + 1e-9) + 1e-300;
    const long long t = e / te;
    double *b = &boxes[6 * t];
    if (e % te == 0)
      for (int a = 0; a < 3; ++a) {
        b[a] = INFINITY;
        b[3 + a] = -INFINITY;
      }
    for (int i = 0; i < Np; ++i)
      for (int a = 0; a < 3; ++a) {
        b[a] = std::min(b[a], xn[3 * i + a]);
        b[3 + a] = std::max(b[3 + a], xn[3 * i + a]);
        m->box_lo[a] = std::min(m->box_lo[a], xn[3 * i + a]);
        m->box_hi[a] = std::max(m->box_hi[a], xn[3 * i + a]);
      }
  }
  m->tile_elements = te;
  m->tile_count = tiles;
  double *db;
  PRT_CHECK_CUDA(cudaMalloc(&db, boxes.size() * sizeof(double)));
  PRT_CHECK_CUDA(cudaMemcpy(db, boxes.data(), boxes.size() * sizeof(double), cudaMemcpyHostToDevice));
  m->tile_boxes = db;
  PRT_CHECK_CUDA(cudaMalloc(&db, spheres.size() * sizeof(double)));
  PRT_CHECK_CUDA(cudaMemcpy(db, spheres.data(), spheres.size() * sizeof(double), cudaMemcpyHostToDevice));
  m->el_spheres = db;

  // tile bins for the normalising pre-pass: uniform bins of about one tile
  double ext[3], mean[3] = {0, 0, 0};
  for (long long t = 0; t < tiles; ++t)
    for (int a = 0; a < 3; ++a) mean[a] += boxes[6 * t + 3 + a] - boxes[6 * t + a];
  TileBinsHost &H = m->tile_bins;
  long long nb = 1;
  for (int a = 0; a < 3; ++a) {
    mean[a] = std::max(mean[a] / tiles, 1e-300);
    ext[a] = m->box_hi[a] - m->box_lo[a];
    int dims = ext[a] > 0 ? (int)std::max(1.0, std::min(512.0, std::floor(ext[a] / mean[a]))) : 1;
    H.dims[a] = dims;
    H.origin[a] = m->box_lo[a];
    H.inv_w[a] = ext[a] > 0 ? dims / ext[a] : 0.0;
    nb *= dims;
  }
  std::vector<uint32_t> counts(nb + 1, 0);
  auto brange = [&](long long t, int a, int &b0, int &b1) {
    double l = std::floor((boxes[6 * t + a] - H.origin[a]) * H.inv_w[a]);
    double h = std::floor((boxes[6 * t + 3 + a] - H.origin[a]) * H.inv_w[a]);
    b0 = (int)std::max(0.0, std::min(l, H.dims[a] - 1.0));
    b1 = (int)std::max(0.0, std::min(h, H.dims[a] - 1.0));
  };
  for (int pass = 0; pass < 2; ++pass) {
    std::vector<uint32_t> fill;
    std::vector<uint32_t> list;
    if (pass == 1) {
      for (long long b = 0; b < nb; ++b) counts[b + 1] += counts[b];
      list.resize(counts[nb]);
      fill.assign(counts.begin(), counts.end() - 1);
    }
    for (long long t = 0; t < tiles; ++t) {
      int r0[3], r1[3];
      for (int a = 0; a < 3; ++a) brange(t, a, r0[a], r1[a]);
      for (int z = r0[2]; z <= r1[2]; ++z)
        for (int y = r0[1]; y <= r1[1]; ++y)
          for (int x = r0[0]; x <= r1[0]; ++x) {
            long long b = x + (long long)H.dims[0] * (y + (long long)H.dims[1] * z);
            if (pass == 0)
              ++counts[b + 1];
            else
              list[fill[b]++] = (uint32_t)t;
          }
    }
    if (pass == 1) {
      uint32_t *dp;
      PRT_CHECK_CUDA(cudaMalloc(&dp, counts.size() * 4));
      PRT_CHECK_CUDA(cudaMemcpy(dp, counts.data(), counts.size() * 4, cudaMemcpyHostToDevice));
      H.starts = dp;
      PRT_CHECK_CUDA(cudaMalloc(&dp, std::max<size_t>(1, list.size()) * 4));
      if (!list.empty())
        PRT_CHECK_CUDA(cudaMemcpy(dp, list.data(), list.size() * 4, cudaMemcpyHostToDevice));
      H.tiles = dp;
    }
  }
  return PRT_OK;
}

// -------------------------------------------------------------- C ABI: mesh

extern "C" int prt_deposit_shape(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                                 prt_shape_function shape, const double *iw, int64_t n,
                                 const double *x, const double *q, const double *v,
                                 const uint32_t *el, double *rho, double *j,
                                 int32_t precision, prt_deposit_stats *stats,
                                 void *stream) {
  if (!mesh || !ws || n < 0 || n >= (1ll << 31) || precision != 0) return PRT_ERR_INVALID_ARGUMENT;
  if (!(shape.radius > 0) || (mode != PRT_DEPOSIT_PLAIN && mode != PRT_DEPOSIT_NORMALIZED))
    return PRT_ERR_INVALID_ARGUMENT;
  if (mode == PRT_DEPOSIT_NORMALIZED && !iw) return PRT_ERR_INVALID_ARGUMENT;
  if (n > 0 && (!x || !q || (j && !v))) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const long long nn = mesh->dev.E * (long long)mesh->dev.Np;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (n == 0) {
    if (rho) PRT_CHECK_CUDA(cudaMemsetAsync(rho, 0, nn * sizeof(double), s));
    if (j) PRT_CHECK_CUDA(cudaMemsetAsync(j, 0, 3 * nn * sizeof(double), s));
    return PRT_OK;
  }
  ShapeParams S;
  S.radius = shape.radius;
  S.radius2 = shape.radius * shape.radius;
  S.inv_radius = 1.0 / shape.radius;
  S.alpha = shape.alpha;
  for (int d = 0; d < 3; ++d) S.reach[d] = shape.radius;
  int rc;
  BinGrid G;
  if (!choose_bins(mesh, shape.radius, G, &rc)) return rc;

  const double *scale = nullptr;
  double normalizer = shape.normalizer;
  if (mode == PRT_DEPOSIT_NORMALIZED) {
    double *sc = (double *)ws_buffer(ws, PRT_WS_DEP_SCALE, 2 * sizeof(double) * (size_t)n, &rc);
    if (!sc) return rc;
    int rc2;
    double *iwd = (double *)ws_buffer(ws, PRT_WS_DEP_STATS, sizeof(double) * (64 + mesh->dev.Np), &rc2);
    if (!iwd) return rc2;
    PRT_CHECK_CUDA(cudaMemcpyAsync(iwd + 16, iw, sizeof(double) * mesh->dev.Np,
                                   cudaMemcpyHostToDevice, s));
    TileBins TB;
    for (int d = 0; d < 3; ++d) {
      TB.origin[d] = mesh->tile_bins.origin[d];
      TB.inv_w[d] = mesh->tile_bins.inv_w[d];
      TB.dims[d] = mesh->tile_bins.dims[d];
    }
    TB.starts = mesh->tile_bins.starts;
    TB.tiles = mesh->tile_bins.tiles;
    const long long threads = 32 * (long long)n;
    if (shape.alpha == 2)
      normalize_kernel<true><<<prt_grid_blocks(threads, 128), 128, 0, s>>>(
          mesh->dev, TB, mesh->tile_boxes, mesh->el_spheres, mesh->tile_elements, iwd + 16, S,
          shape.normalizer, n, x, q, el, sc, sc + n, ws->status);
    else
      normalize_kernel<false><<<prt_grid_blocks(threads, 128), 128, 0, s>>>(
          mesh->dev, TB, mesh->tile_boxes, mesh->el_spheres, mesh->tile_elements, iwd + 16, S,
          shape.normalizer, n, x, q, el, sc, sc + n, ws->status);
    PRT_CHECK_CUDA(cudaGetLastError());
    if (stats) {
      stats_kernel<<<1, 256, 0, s>>>(n, sc, sc + n, iwd);
      PRT_CHECK_CUDA(cudaGetLastError());
      double h[10];
      PRT_CHECK_CUDA(cudaMemcpyAsync(h, iwd, sizeof(h), cudaMemcpyDeviceToHost, s));
      PRT_CHECK_CUDA(cudaStreamSynchronize(s));
      stats->norm_count = h[0];
      stats->norm_sum = h[1];
      stats->norm_sum_sq = h[2];
      stats->norm_min = h[3];
      stats->norm_max = h[4];
      stats->el_count = h[5];
      stats->el_sum = h[6];
      stats->el_sum_sq = h[7];
      stats->el_min = h[8];
      stats->el_max = h[9];
    }
    scale = sc;
  }

  DepParticles P;
  {
    ScopedTimer timer(ws, PRT_TIME_DEPOSIT_STAGE, s);
    if ((rc = stage_particles(ws, G, n, x, q, v, el, scale, normalizer, nullptr, P, nullptr, s)))
      return rc;
  }
  unsigned long long *counter = nullptr;
  if (stats) {
    counter = (unsigned long long *)ws_buffer(ws, PRT_WS_DEP_COUNT, 64, &rc);
    if (!counter) return rc;
    PRT_CHECK_CUDA(cudaMemsetAsync(counter, 0, 8, s));
  }
  MeshTarget T;
  T.nodes = mesh->dev.nodes;
  T.boxes = mesh->tile_boxes;
  T.spheres = mesh->el_spheres;
  T.E = mesh->dev.E;
  T.Np = mesh->dev.Np;
  T.tile_elements = mesh->tile_elements;
  T.node_count = nn;
  const bool a2 = shape.alpha == 2;
  {
    ScopedTimer timer(ws, PRT_TIME_DEPOSIT_GATHER, s);
    const unsigned nb = (unsigned)mesh->tile_count;
    if (counter) {
      if (a2)
        gather_kernel<MeshTarget, W_SHAPE2, true><<<nb, BLOCK, 0, s>>>(T, G, P, S, rho, j, nn,
                                                                       nullptr, counter);
      else
        gather_kernel<MeshTarget, W_SHAPE_POW, true><<<nb, BLOCK, 0, s>>>(T, G, P, S, rho, j,
                                                                          nn, nullptr, counter);
    } else if (a2) {
      gather_kernel<MeshTarget, W_SHAPE2><<<nb, BLOCK, 0, s>>>(T, G, P, S, rho, j, nn, nullptr,
                                                               nullptr);
    } else {
      gather_kernel<MeshTarget, W_SHAPE_POW><<<nb, BLOCK, 0, s>>>(T, G, P, S, rho, j, nn,
                                                                  nullptr, nullptr);
    }
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  if (counter) {
    unsigned long long h = 0;
    PRT_CHECK_CUDA(cudaMemcpyAsync(&h, counter, 8, cudaMemcpyDeviceToHost, s));
    PRT_CHECK_CUDA(cudaStreamSynchronize(s));
    stats->pair_count = (double)h;
  }
  return PRT_OK;
}

// ------------------------------------------------------------------- grid

struct prt_grid {
  const prt_mesh *mesh;
  int brick_count;
  int np;
  std::vector<prt_brick> host_bricks;
  prt_brick *bricks = nullptr;
  long long *tile_starts = nullptr;
  long long tiles = 0;
  long long grid_nodes = 0;
  long long eog_count = 0;
  uint32_t *eog_elements = nullptr;
  uint64_t *eog_starts = nullptr;
  uint32_t *eog_nodes = nullptr;
  double *eog_weights = nullptr;
  uint64_t *eog_mstarts = nullptr;
  double *eog_matrices = nullptr;
  int max_points = 0;
  long long avg_count = 0;
  uint32_t *avg_starts = nullptr;
  uint32_t *avg_nodes = nullptr;
};

extern "C" int prt_grid_create(const prt_mesh *mesh, const prt_grid_desc *d, prt_grid **out) {
  if (!mesh || !d || !out || d->brick_count <= 0 || !d->bricks ||
      d->nodes_per_element != mesh->dev.Np)
    return PRT_ERR_INVALID_ARGUMENT;
  prt_grid *g = new prt_grid();
  g->mesh = mesh;
  g->brick_count = d->brick_count;
  g->np = d->nodes_per_element;
  g->host_bricks.assign(d->bricks, d->bricks + d->brick_count);
  std::vector<long long> ts(d->brick_count + 1, 0);
  long long gn = 0;
  for (int b = 0; b < d->brick_count; ++b) {
    const prt_brick &B = d->bricks[b];
    for (int a = 0; a < 3; ++a)
      if (B.dims[a] <= 0 || !(B.stepwidths[a] > 0)) {
        delete g;
        return PRT_ERR_INVALID_ARGUMENT;
      }
    long long t = (long long)((B.dims[0] + 7) / 8) * ((B.dims[1] + 3) / 4) * ((B.dims[2] + 3) / 4);
    ts[b + 1] = ts[b] + t;
    gn = std::max(gn, B.start_index + (long long)B.dims[0] * B.dims[1] * B.dims[2]);
  }
  g->tiles = ts.back();
  g->grid_nodes = gn;
  auto up = [&](auto **dst, const auto *src, size_t cnt) -> int {
    using T = std::remove_pointer_t<std::remove_reference_t<decltype(*dst)>>;
    *dst = nullptr;
    if (cnt == 0) return PRT_OK;
    if (!src) return PRT_ERR_INVALID_ARGUMENT;
    PRT_CHECK_CUDA(cudaMalloc((void **)dst, cnt * sizeof(T)));
    PRT_CHECK_CUDA(cudaMemcpy((void *)*dst, src, cnt * sizeof(T), cudaMemcpyHostToDevice));
    return PRT_OK;
  };
  int rc = up(&g->bricks, d->bricks, d->brick_count);
  if (!rc) rc = up(&g->tile_starts, ts.data(), ts.size());
  g->eog_count = d->eog_count;
  if (d->eog_count > 0) {
    // one element-on-grid per element: the remap owns its nodes
    std::vector<char> seen(mesh->dev.E, 0);
    for (long long e = 0; e < d->eog_count && !rc; ++e) {
      uint32_t el = d->eog_elements[e];
      if (el >= mesh->dev.E || seen[el]) rc = PRT_ERR_INVALID_ARGUMENT;
      else seen[el] = 1;
      g->max_points = std::max<int>(g->max_points, (int)(d->eog_starts[e + 1] - d->eog_starts[e]));
      if (d->eog_matrix_starts[e + 1] - d->eog_matrix_starts[e] !=
          (uint64_t)g->np * (d->eog_starts[e + 1] - d->eog_starts[e]))
        rc = PRT_ERR_INVALID_ARGUMENT;
    }
    const size_t tot = d->eog_starts[d->eog_count];
    const size_t mtot = d->eog_matrix_starts[d->eog_count];
    if (!rc) rc = up(&g->eog_elements, d->eog_elements, d->eog_count);
    if (!rc) rc = up(&g->eog_starts, d->eog_starts, d->eog_count + 1);
    if (!rc) rc = up(&g->eog_nodes, d->eog_grid_nodes, tot);
    if (!rc) rc = up(&g->eog_weights, d->eog_weights, tot);
    if (!rc) rc = up(&g->eog_mstarts, d->eog_matrix_starts, d->eog_count + 1);
    if (!rc) rc = up(&g->eog_matrices, d->eog_matrices, mtot);
  }
  g->avg_count = d->avg_group_count;
  if (!rc && d->avg_group_count > 0) {
    rc = up(&g->avg_starts, d->avg_group_starts, d->avg_group_count + 1);
    if (!rc) rc = up(&g->avg_nodes, d->avg_group_nodes, d->avg_group_starts[d->avg_group_count]);
  }
  if (rc) {
    prt_grid_destroy(g);
    return rc;
  }
  *out = g;
  return PRT_OK;
}

extern "C" int prt_grid_destroy(prt_grid *g) {
  if (!g) return PRT_OK;
  void *ptrs[] = {g->bricks, g->tile_starts, g->eog_elements, g->eog_starts, g->eog_nodes,
                  g->eog_weights, g->eog_mstarts, g->eog_matrices, g->avg_starts, g->avg_nodes};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete g;
  return PRT_OK;
}

__global__ void brick_tag_kernel(const prt_brick *__restrict__ bricks, int nb, long long n,
                                 const double *__restrict__ x, const uint32_t *__restrict__ el,
                                 uint32_t *__restrict__ tag) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t t = 0xffffffffu;
  if (!el || el[i] != PRT_INVALID) {
    const double p[3] = {x[i], x[n + i], x[2 * n + i]};
    for (int b = 0; b < nb && t == 0xffffffffu; ++b) {
      bool in = true;
      for (int d = 0; d < 3; ++d)
        in = in && p[d] >= bricks[b].origin[d] &&
             p[d] < bricks[b].origin[d] + bricks[b].dims[d] * bricks[b].stepwidths[d];
      if (in) t = (uint32_t)b;
    }
  }
  tag[i] = t;
}

extern "C" int prt_deposit_grid(const prt_grid *g, prt_workspace *ws, int32_t weights,
                                prt_shape_function shape, int64_t n, const double *x,
                                const double *q, const double *v, const uint32_t *el,
                                double *grid_rho, double *grid_j, void *stream) {
  if (!g || !ws || n < 0 || n >= (1ll << 31)) return PRT_ERR_INVALID_ARGUMENT;
  if (weights != PRT_GRID_SHAPE && weights != PRT_GRID_TRILINEAR) return PRT_ERR_INVALID_ARGUMENT;
  if (weights == PRT_GRID_SHAPE && !(shape.radius > 0)) return PRT_ERR_INVALID_ARGUMENT;
  if (n > 0 && (!x || !q || (grid_j && !v))) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const long long G_n = g->grid_nodes;
  if (n == 0) {
    if (grid_rho) PRT_CHECK_CUDA(cudaMemsetAsync(grid_rho, 0, G_n * sizeof(double), s));
    if (grid_j) PRT_CHECK_CUDA(cudaMemsetAsync(grid_j, 0, 3 * G_n * sizeof(double), s));
    return PRT_OK;
  }
  ShapeParams S;
  int rc;
  BinGrid G;
  double reach_bins;
  const uint32_t *tag = nullptr;
  double normalizer;
  if (weights == PRT_GRID_SHAPE) {
    S.radius = shape.radius;
    S.radius2 = shape.radius * shape.radius;
    S.inv_radius = 1.0 / shape.radius;
    S.alpha = shape.alpha;
    for (int d = 0; d < 3; ++d) S.reach[d] = shape.radius;
    reach_bins = shape.radius;
    normalizer = shape.normalizer;
  } else {
    // trilinear: a point receives from particles within one cell; the
    // payload weight is q / dV (dV of the particle's brick, via the tag).
    double hmax = 0;
    for (const prt_brick &B : g->host_bricks)
      for (int d = 0; d < 3; ++d) hmax = std::max(hmax, B.stepwidths[d]);
    // a point receives from particles within one cell per axis, i.e. within
    // sqrt(3) h: the cull sphere uses that radius
    S.radius = hmax * std::sqrt(3.0) * (1 + 1e-12);
    S.radius2 = S.radius * S.radius;
    S.inv_radius = 1.0 / hmax;
    S.alpha = 1;
    for (int d = 0; d < 3; ++d) S.reach[d] = hmax;
    reach_bins = hmax;
    normalizer = 1.0;
    if (g->brick_count > 1) {
      // distinct cell volumes per brick are not supported in one payload
      for (const prt_brick &B : g->host_bricks)
        for (int d = 0; d < 3; ++d)
          if (B.stepwidths[d] != g->host_bricks[0].stepwidths[d]) return PRT_ERR_INVALID_ARGUMENT;
    }
    const prt_brick &B0 = g->host_bricks[0];
    normalizer = 1.0 / (B0.stepwidths[0] * B0.stepwidths[1] * B0.stepwidths[2]);
    uint32_t *tg = (uint32_t *)ws_buffer(ws, PRT_WS_SORT_TMP, 4 * (size_t)n, &rc);
    if (!tg) return rc;
    brick_tag_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(g->bricks, g->brick_count, n, x, el, tg);
    PRT_CHECK_CUDA(cudaGetLastError());
    tag = tg;
  }
  // bins must cover the bricks as well as the mesh box
  prt_mesh tmp = *g->mesh;
  for (const prt_brick &B : g->host_bricks)
    for (int d = 0; d < 3; ++d) {
      tmp.box_lo[d] = std::min(tmp.box_lo[d], B.origin[d]);
      tmp.box_hi[d] = std::max(tmp.box_hi[d], B.origin[d] + B.dims[d] * B.stepwidths[d]);
    }
  if (!choose_bins(&tmp, reach_bins, G, &rc)) return rc;
  DepParticles P;
  if ((rc = stage_particles(ws, G, n, x, q, v, el, nullptr, normalizer, tag, P, nullptr, s)))
    return rc;
  BrickTarget T;
  T.bricks = g->bricks;
  T.tile_starts = g->tile_starts;
  T.brick_count = g->brick_count;
  T.check_tag = weights == PRT_GRID_TRILINEAR;
  if (grid_rho) PRT_CHECK_CUDA(cudaMemsetAsync(grid_rho, 0, G_n * sizeof(double), s));
  if (grid_j) PRT_CHECK_CUDA(cudaMemsetAsync(grid_j, 0, 3 * G_n * sizeof(double), s));
  if (weights == PRT_GRID_TRILINEAR)
    gather_kernel<BrickTarget, W_TRILINEAR><<<(unsigned)g->tiles, BLOCK, 0, s>>>(
        T, G, P, S, grid_rho, grid_j, G_n, g->bricks, nullptr);
  else if (shape.alpha == 2)
    gather_kernel<BrickTarget, W_SHAPE2><<<(unsigned)g->tiles, BLOCK, 0, s>>>(
        T, G, P, S, grid_rho, grid_j, G_n, g->bricks, nullptr);
  else
    gather_kernel<BrickTarget, W_SHAPE_POW><<<(unsigned)g->tiles, BLOCK, 0, s>>>(
        T, G, P, S, grid_rho, grid_j, G_n, g->bricks, nullptr);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

// Remap (dep_grid.hpp:270-358): one warp per element-on-grid; lanes own the
// element's nodes, the weighted grid values are staged in shared memory.
__global__ void remap_kernel(long long eog_count, int np, const uint32_t *__restrict__ els,
                             const uint64_t *__restrict__ starts,
                             const uint32_t *__restrict__ gnodes,
                             const double *__restrict__ weights,
                             const uint64_t *__restrict__ mstarts,
                             const double *__restrict__ mats, const double *__restrict__ from,
                             double *__restrict__ to, long long offset, long long inc) {
  extern __shared__ double gv_all[];
  const int warps = blockDim.x >> 5;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long e = blockIdx.x * (long long)warps + wid;
  if (e >= eog_count) return;
  const uint64_t s = starts[e];
  const int cnt = (int)(starts[e + 1] - s);
  // stage at most 256 points per pass
  double *gv = gv_all + wid * 256;
  double acc[2] = {0, 0};
  bool any = false;
  const double *M = mats + mstarts[e];
  for (int base = 0; base < cnt; base += 256) {
    const int m = min(256, cnt - base);
    for (int k = lane; k < m; k += 32) {
      double w = weights[s + base + k] * from[offset + (long long)gnodes[s + base + k] * inc];
      gv[k] = w;
      any = any || w != 0;
    }
    __syncwarp();
    for (int k = 0; k < m; ++k) {
      const double g = gv[k];
      for (int r = 0; r < 2; ++r) {
        int i = lane + 32 * r;
        if (i < np) acc[r] = fma(M[i + (size_t)np * (base + k)], g, acc[r]);
      }
    }
    __syncwarp();
  }
  if (!__any_sync(0xffffffffu, any)) return;
  double *y = to + (long long)els[e] * np * inc + offset;
  for (int r = 0; r < 2; ++r) {
    int i = lane + 32 * r;
    if (i < np) y[i * inc] += acc[r];
  }
}

__global__ void average_kernel(long long groups, const uint32_t *__restrict__ starts,
                               const uint32_t *__restrict__ nodes, double *__restrict__ to,
                               long long offset, long long inc) {
  long long gi = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (gi >= groups) return;
  uint32_t s = starts[gi], t = starts[gi + 1];
  if (s == t) return;
  double avg = 0;
  for (uint32_t k = s; k < t; ++k) avg += to[offset + (long long)nodes[k] * inc];
  avg /= (t - s);
  for (uint32_t k = s; k < t; ++k) to[offset + (long long)nodes[k] * inc] = avg;
}

extern "C" int prt_remap_grid_to_mesh(const prt_grid *g, const double *from, double *to,
                                      int64_t offset, int64_t inc, void *stream) {
  if (!g || !from || !to || inc <= 0 || offset < 0 || g->np > 64) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  if (g->eog_count > 0) {
    const int warps = 4;
    remap_kernel<<<prt_grid_blocks(g->eog_count, warps), 32 * warps,
                   warps * 256 * sizeof(double), s>>>(
        g->eog_count, g->np, g->eog_elements, g->eog_starts, g->eog_nodes, g->eog_weights,
        g->eog_mstarts, g->eog_matrices, from, to, offset, inc);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  if (g->avg_count > 0) {
    average_kernel<<<prt_grid_blocks(g->avg_count, 128), 128, 0, s>>>(
        g->avg_count, g->avg_starts, g->avg_nodes, to, offset, inc);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  return PRT_OK;
}
