// grid.cu -- deposition onto brick grids and the element-local remap onto
// the DG nodes (dep_grid_base.hpp:175-382, dep_grid.hpp:220-358, grid.hpp).
//
// Deposition is the same deterministic gather as the mesh depositor (see
// deposit.cu): particles binned and sorted, one CTA per tile of 8 x 4 x 4
// brick points, one point per thread, the staged particles culled against
// the tile's bounding sphere. Weights: the shape function at the point (the
// reference's grid depositor) or trilinear weights (cell-centred hat
// functions, clamped at the brick edge so that they always sum to one).
// Jiggly bricks (grid.hpp:345-449) take their points from three jittered
// point origins; the tile boxes grow by the largest jitter.

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "binning.cuh"

namespace {

using namespace prt_dep;

#ifndef PRT_GRID_MIN_BLOCKS
#define PRT_GRID_MIN_BLOCKS 6
#endif

// ---------------------------------------------------------------- targets

// Per brick of a jiggly grid: the three point origins and, per axis, the
// largest distance of a point from its cell centre.
struct JiggleDev {
  double origins[3][3];
  double pad[3];
};

// Tile of 8 x 4 x 4 points of one brick; one group (the tile box).
struct BrickTarget {
  const prt_brick *__restrict__ bricks;
  const long long *__restrict__ tile_starts;  // [bricks+1] cumulative tile counts
  const JiggleDev *__restrict__ jiggle;       // [bricks] or NULL (regular points)
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
    if (jiggle) {
      // jiggly_brick::point (grid.hpp:386-396)
      const double *o = jiggle[b].origins[(idx[0] + idx[1] + idx[2]) % 3];
      x0 = o[0] + idx[0] * B.stepwidths[0];
      x1 = o[1] + idx[1] * B.stepwidths[1];
      x2 = o[2] + idx[2] * B.stepwidths[2];
      return;
    }
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
      if (jiggle) {
        lo[d] -= jiggle[b].pad[d];
        hi[d] += jiggle[b].pad[d];
      }
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


// One CTA per tile of brick points, one point per thread. Per chunk of
// staged particles every thread stages one particle and tests it against the
// tile's bounding sphere (grown by the reach); the survivors are compacted
// into a shared index list that every point walks. Bin rows are culled
// against the tile box with the sphere of the shape radius.
template <class Target, int WEIGHT, bool COUNT = false>
__global__ void __launch_bounds__(BLOCK, PRT_GRID_MIN_BLOCKS)
    deposit_grid_kernel(Target T, BinGrid G, DepParticles P, ShapeParams S,
                  double *__restrict__ rho, double *__restrict__ j, long long j_stride,
                  const prt_brick *__restrict__ tri_bricks,
                  unsigned long long *__restrict__ pair_counter) {
  static_assert(BLOCK == CHUNK, "one staged particle per thread");
  constexpr int WARPS = BLOCK / 32;
  __shared__ double sp[PAYLOAD][CHUNK];
  __shared__ uint8_t lists[32][CHUNK];
  __shared__ int warp_cnt[32][WARPS];
  __shared__ int list_len[32];
  __shared__ double sph[32][4];

  const long long tile = blockIdx.x;
  const int t = threadIdx.x;
  const int lane = t & 31, wid = t >> 5;
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
  // sphere culling of bin rows (not for the per-axis trilinear reach)
  constexpr bool SPHERE = WEIGHT != W_TRILINEAR;
  const double reach = S.reach[0] * (1 + 1e-6);
  const double reach2 = reach * reach;
  __syncthreads();

  for (int bz = u0[2]; bz <= u1[2]; ++bz) {
    int wz = bz, qz = 0;
    if (G.periodic[2]) { qz = floor_div(bz, G.dims[2]); wz = bz - qz * G.dims[2]; }
    const double sz = qz * G.period[2];
    double dz2 = 0;
    if (SPHERE) {
      const double blo = G.origin[2] + bz * G.w[2], bhi = blo + G.w[2];
      const double e = fmax(0.0, fmax(blo - hi[2], lo[2] - bhi)) - G.slack[2];
      dz2 = e > 0 ? e * e : 0.0;
      if (dz2 > reach2) continue;
    }
    for (int by = u0[1]; by <= u1[1]; ++by) {
      int wy = by, qy = 0;
      if (G.periodic[1]) { qy = floor_div(by, G.dims[1]); wy = by - qy * G.dims[1]; }
      const double sy = qy * G.period[1];
      int bx0 = u0[0], bx1 = u1[0];
      if (SPHERE) {
        const double blo = G.origin[1] + by * G.w[1], bhi = blo + G.w[1];
        const double e = fmax(0.0, fmax(blo - hi[1], lo[1] - bhi)) - G.slack[1];
        const double dyz2 = dz2 + (e > 0 ? e * e : 0.0);
        if (dyz2 > reach2) continue;
        const double rem = sqrt(reach2 - dyz2);
        int c0 = bin_floor(G, 0, lo[0] - rem), c1 = bin_floor(G, 0, hi[0] + rem);
        if (G.periodic[0]) {
          c0 -= 1;
          c1 += 1;
        }
        bx0 = max(bx0, c0);
        bx1 = min(bx1, c1);
      }
      // the x-row splits into segments of constant shift
      int bx = bx0;
      while (bx <= bx1) {
        int wx = bx, qx = 0, seg_end = bx1;
        if (G.periodic[0]) {
          qx = floor_div(bx, G.dims[0]);
          wx = bx - qx * G.dims[0];
          seg_end = min(bx1, (qx + 1) * G.dims[0] - 1);
        }
        const double sx = qx * G.period[0];
        const long long row = (long long)G.dims[0] * (wy + (long long)G.dims[1] * wz);
        const uint32_t s0 = P.starts[row + wx];
        const uint32_t s1 = P.starts[row + wx + (seg_end - bx) + 1];
        bx = seg_end + 1;
        for (uint32_t c0 = s0; c0 < s1; c0 += CHUNK) {
          const int cnt = (int)min((uint32_t)CHUNK, s1 - c0);
          __syncthreads();  // previous chunk fully consumed
          uint32_t m = 0;
          if (t < cnt) {
            const double2 *src = reinterpret_cast<const double2 *>(P.payload) +
                                 (size_t)(c0 + t) * (PAYLOAD / 2);
            const double2 a = src[0], b = src[1], c = src[2], d = src[3];
            const double px = a.x + sx, py = a.y + sy, pz = b.x + sz;
            sp[0][t] = px;
            sp[1][t] = py;
            sp[2][t] = pz;
            sp[3][t] = b.y;
            sp[4][t] = c.x;
            sp[5][t] = c.y;
            sp[6][t] = d.x;
            sp[7][t] = d.y;
            if (T.tag_ok(tile, d.y)) {
              for (int g = 0; g < ng; ++g) {
                const double dx = px - sph[g][0], dy = py - sph[g][1], dz = pz - sph[g][2];
                if (dx * dx + dy * dy + dz * dz <= sph[g][3]) m |= 1u << g;
              }
            }
          }
          for (int g = 0; g < ng; ++g) {
            const unsigned b = __ballot_sync(0xffffffffu, (m >> g) & 1u);
            if (lane == 0) warp_cnt[g][wid] = __popc(b);
          }
          __syncthreads();
          for (int g = 0; g < ng; ++g) {
            const unsigned b = __ballot_sync(0xffffffffu, (m >> g) & 1u);
            if ((m >> g) & 1u) {
              int off = __popc(b & ((1u << lane) - 1u));
              for (int w = 0; w < wid; ++w) off += warp_cnt[g][w];
              lists[g][off] = (uint8_t)t;
            }
          }
          if (t < ng) {
            int tot = 0;
            for (int w = 0; w < WARPS; ++w) tot += warp_cnt[t][w];
            list_len[t] = tot;
          }
          __syncthreads();
          if (live) {
            const int len = list_len[grp];
            const uint8_t *L = lists[grp];
            for (int i = 0; i < len; ++i) {
              const int k = L[i];
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
    if (lane == 0 && npairs) atomicAdd(pair_counter, npairs);
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


}  // namespace

// ------------------------------------------------------------------- grid

struct prt_grid {
  const prt_mesh *mesh;
  int brick_count;
  int np;
  std::vector<prt_brick> host_bricks;
  prt_brick *bricks = nullptr;
  JiggleDev *jiggle = nullptr;
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
  // host copy of the jiggled point origins [bricks][3][3] (or empty)
  std::vector<double> host_origins;
  // the grid's points in grid-node order, for the tensor-core deposition
  // (made on its first call)
  mutable unsigned long long uid = 0;
  mutable std::vector<double> pt_host;
  mutable double *pt_dev = nullptr;
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
  if (!rc && d->point_origins) {
    g->host_origins.assign(d->point_origins, d->point_origins + 9 * d->brick_count);
    std::vector<JiggleDev> jg(d->brick_count);
    for (int b = 0; b < d->brick_count && !rc; ++b) {
      const prt_brick &B = d->bricks[b];
      for (int a = 0; a < 3; ++a) {
        const double centre = B.origin[a] + B.stepwidths[a] / 2;
        double pad = 0;
        for (int i = 0; i < 3; ++i) {
          const double o = d->point_origins[9 * b + 3 * i + a];
          jg[b].origins[i][a] = o;
          pad = std::max(pad, std::fabs(o - centre));
        }
        // points stay within their cells (the reference's index ranges
        // assume it); the margin covers the rounding of idx * h
        if (!(pad <= 0.5 * B.stepwidths[a] * (1 + 1e-12))) rc = PRT_ERR_INVALID_ARGUMENT;
        jg[b].pad[a] = pad * (1 + 1e-9) + 1e-12 * B.stepwidths[a];
      }
    }
    if (!rc) rc = up(&g->jiggle, jg.data(), jg.size());
  }
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
  void *ptrs[] = {g->bricks,      g->tile_starts, g->jiggle,      g->eog_elements,
                  g->eog_starts,  g->eog_nodes,   g->eog_weights, g->eog_mstarts,
                  g->eog_matrices, g->avg_starts, g->avg_nodes,   g->pt_dev};
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
  if (weights == PRT_GRID_TRILINEAR && g->jiggle) return PRT_ERR_INVALID_ARGUMENT;
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
  double blo[3], bhi[3];
  for (int d = 0; d < 3; ++d) {
    blo[d] = g->mesh->box_lo[d];
    bhi[d] = g->mesh->box_hi[d];
  }
  for (const prt_brick &B : g->host_bricks)
    for (int d = 0; d < 3; ++d) {
      blo[d] = std::min(blo[d], B.origin[d]);
      bhi[d] = std::max(bhi[d], B.origin[d] + B.dims[d] * B.stepwidths[d]);
    }
  if (!choose_bins(g->mesh, blo, bhi,
                   weights == PRT_GRID_TRILINEAR ? reach_bins : reach_bins * BIN_FRACTION,
                   weights == PRT_GRID_TRILINEAR ? reach_bins * std::sqrt(3.0) : reach_bins, G,
                   &rc))
    return rc;
  DepParticles P;
  if ((rc = stage_particles(ws, G, n, x, q, v, el, nullptr, normalizer, tag, P, s))) return rc;
  BrickTarget T;
  T.bricks = g->bricks;
  T.tile_starts = g->tile_starts;
  T.jiggle = g->jiggle;
  T.brick_count = g->brick_count;
  T.check_tag = weights == PRT_GRID_TRILINEAR;
  if (grid_rho) PRT_CHECK_CUDA(cudaMemsetAsync(grid_rho, 0, G_n * sizeof(double), s));
  if (grid_j) PRT_CHECK_CUDA(cudaMemsetAsync(grid_j, 0, 3 * G_n * sizeof(double), s));
  ScopedTimer timer(ws, PRT_TIME_DEPOSIT_GATHER, s);
  if (weights == PRT_GRID_TRILINEAR)
    deposit_grid_kernel<BrickTarget, W_TRILINEAR><<<(unsigned)g->tiles, BLOCK, 0, s>>>(
        T, G, P, S, grid_rho, grid_j, G_n, g->bricks, nullptr);
  else if (shape.alpha == 2)
    deposit_grid_kernel<BrickTarget, W_SHAPE2><<<(unsigned)g->tiles, BLOCK, 0, s>>>(
        T, G, P, S, grid_rho, grid_j, G_n, g->bricks, nullptr);
  else
    deposit_grid_kernel<BrickTarget, W_SHAPE_POW><<<(unsigned)g->tiles, BLOCK, 0, s>>>(
        T, G, P, S, grid_rho, grid_j, G_n, g->bricks, nullptr);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

// The grid's points in grid-node order (host and device), made once: the
// positions of BrickTarget::point (regular cell centres, or the jiggled
// points of jiggly_brick::point, grid.hpp:386-396). The bricks must number
// their points contiguously (brick b starts where brick b-1 ends).
int grid_points(const prt_grid *g) {
  if (g->pt_dev) return PRT_OK;
  long long next = 0;
  for (const prt_brick &B : g->host_bricks) {
    if (B.start_index != next) return PRT_ERR_INVALID_ARGUMENT;
    next += (long long)B.dims[0] * B.dims[1] * B.dims[2];
  }
  if (next != g->grid_nodes) return PRT_ERR_INVALID_ARGUMENT;
  std::vector<double> P(3 * (size_t)g->grid_nodes);
  for (int b = 0; b < g->brick_count; ++b) {
    const prt_brick &B = g->host_bricks[b];
    for (int k = 0; k < B.dims[2]; ++k)
      for (int jy = 0; jy < B.dims[1]; ++jy)
        for (int i = 0; i < B.dims[0]; ++i) {
          const int idx[3] = {i, jy, k};
          double *p = &P[3 * (size_t)(B.start_index + i +
                                      (long long)B.dims[0] * (jy + (long long)B.dims[1] * k))];
          for (int a = 0; a < 3; ++a)
            p[a] = g->host_origins.empty()
                       ? B.origin[a] + B.stepwidths[a] / 2 + idx[a] * B.stepwidths[a]
                       : g->host_origins[9 * b + 3 * ((i + jy + k) % 3) + a] +
                             idx[a] * B.stepwidths[a];
        }
  }
  double *d = nullptr;
  PRT_CHECK_CUDA(cudaMalloc((void **)&d, P.size() * sizeof(double)));
  if (cudaMemcpy(d, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return PRT_ERR_CUDA;
  }
  g->pt_host.swap(P);
  g->pt_dev = d;
  g->uid = prt_next_target_uid();
  return PRT_OK;
}

extern "C" int prt_deposit_grid_mixed(const prt_grid *g, prt_workspace *ws,
                                      prt_shape_function shape, int64_t n, const double *x,
                                      const double *q, const double *v, const uint32_t *el,
                                      double *grid_rho, double *grid_j, void *stream) {
  if (!g || !ws || n < 0 || n >= (1ll << 31)) return PRT_ERR_INVALID_ARGUMENT;
  if (shape.alpha != 2 || !(shape.radius > 0)) return PRT_ERR_INVALID_ARGUMENT;
  if (n > 0 && (!x || !q || (grid_j && !v))) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  if ((rc = grid_points(g))) return rc;
  const long long G_n = g->grid_nodes;
  if (n == 0) {
    if (grid_rho) PRT_CHECK_CUDA(cudaMemsetAsync(grid_rho, 0, G_n * sizeof(double), s));
    if (grid_j) PRT_CHECK_CUDA(cudaMemsetAsync(grid_j, 0, 3 * G_n * sizeof(double), s));
    return PRT_OK;
  }
  TcTarget T;
  T.mesh = g->mesh;
  T.uid = g->uid;
  T.npos = G_n;
  T.pos = g->pt_dev;
  T.pos_host = g->pt_host.data();
  // particle bins over the mesh box and the bricks
  for (int d = 0; d < 3; ++d) {
    T.lo[d] = g->mesh->box_lo[d];
    T.hi[d] = g->mesh->box_hi[d];
  }
  for (const prt_brick &B : g->host_bricks)
    for (int d = 0; d < 3; ++d) {
      T.lo[d] = std::min(T.lo[d], B.origin[d]);
      T.hi[d] = std::max(T.hi[d], B.origin[d] + B.dims[d] * B.stepwidths[d]);
    }
  return prt_deposit_points_tc(T, ws, shape, n, x, q, v, el, grid_rho, grid_j, s);
}

// Remap (dep_grid.hpp:270-358): one warp per element-on-grid; lanes own the
// element's nodes, the weighted grid values of NC components are staged in
// shared memory, and each matrix entry is read once for all components. A
// block of grid values that is zero in every component is skipped before the
// matrix is read (fma(M, 0, acc) = acc: the sums are unchanged).
template <int NC>
__global__ void remap_kernel(long long eog_count, int np, const uint32_t *__restrict__ els,
                             const uint64_t *__restrict__ starts,
                             const uint32_t *__restrict__ gnodes,
                             const double *__restrict__ weights,
                             const uint64_t *__restrict__ mstarts,
                             const double *__restrict__ mats, const double *__restrict__ from,
                             long long from_stride, double *__restrict__ to,
                             long long to_stride, long long offset, long long inc) {
  extern __shared__ double gv_all[];
  const int warps = blockDim.x >> 5;
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long e = blockIdx.x * (long long)warps + wid;
  if (e >= eog_count) return;
  const uint64_t s = starts[e];
  const int cnt = (int)(starts[e + 1] - s);
  // stage at most 256 points per pass
  double *gv = gv_all + (size_t)wid * 256 * NC;
  double acc[NC][2];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c][0] = acc[c][1] = 0;
  bool any_total = false;
  const double *M = mats + mstarts[e];
  for (int base = 0; base < cnt; base += 256) {
    const int m = min(256, cnt - base);
    bool any = false;
    for (int k = lane; k < m; k += 32) {
      const double wt = weights[s + base + k];
      const long long gi = offset + (long long)gnodes[s + base + k] * inc;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double w = wt * from[c * from_stride + gi];
        gv[c * 256 + k] = w;
        any = any || w != 0;
      }
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, any)) {
      any_total = true;
      for (int k = 0; k < m; ++k) {
        double g[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) g[c] = gv[c * 256 + k];
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int i = lane + 32 * r;
          if (i < np) {
            const double Mv = M[i + (size_t)np * (base + k)];
#pragma unroll
            for (int c = 0; c < NC; ++c) acc[c][r] = fma(Mv, g[c], acc[c][r]);
          }
        }
      }
    }
    __syncwarp();
  }
  if (!any_total) return;
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    double *y = to + c * to_stride + (long long)els[e] * np * inc + offset;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int i = lane + 32 * r;
      if (i < np) y[i * inc] += acc[c][r];
    }
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

template <int NC>
int launch_remap(const prt_grid *g, const double *from, long long from_stride, double *to,
                 long long to_stride, long long offset, long long inc, cudaStream_t s) {
  if (g->eog_count > 0) {
    const int warps = 4;
    remap_kernel<NC><<<prt_grid_blocks(g->eog_count, warps), 32 * warps,
                       warps * 256 * NC * sizeof(double), s>>>(
        g->eog_count, g->np, g->eog_elements, g->eog_starts, g->eog_nodes, g->eog_weights,
        g->eog_mstarts, g->eog_matrices, from, from_stride, to, to_stride, offset, inc);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  if (g->avg_count > 0)
    for (int c = 0; c < NC; ++c) {
      average_kernel<<<prt_grid_blocks(g->avg_count, 128), 128, 0, s>>>(
          g->avg_count, g->avg_starts, g->avg_nodes, to + c * to_stride, offset, inc);
      PRT_CHECK_CUDA(cudaGetLastError());
    }
  return PRT_OK;
}

extern "C" int prt_remap_grid_to_mesh(const prt_grid *g, const double *from, double *to,
                                      int64_t offset, int64_t inc, void *stream) {
  if (!g || !from || !to || inc <= 0 || offset < 0 || g->np > 64) return PRT_ERR_INVALID_ARGUMENT;
  return launch_remap<1>(g, from, 0, to, 0, offset, inc, (cudaStream_t)stream);
}

extern "C" int prt_remap_grid_to_mesh_components(const prt_grid *g, const double *from,
                                                 double *to, int32_t components,
                                                 void *stream) {
  if (!g || !from || !to || components < 1 || components > 4 || g->np > 64)
    return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const long long G = g->grid_nodes, N = g->mesh->dev.E * (long long)g->np;
  switch (components) {
    case 1: return launch_remap<1>(g, from, G, to, N, 0, 1, s);
    case 2: return launch_remap<2>(g, from, G, to, N, 0, 1, s);
    case 3: return launch_remap<3>(g, from, G, to, N, 0, 1, s);
    default: return launch_remap<4>(g, from, G, to, N, 0, 1, s);
  }
}
