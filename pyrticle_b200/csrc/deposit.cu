// deposit.cu -- shape-function deposition onto DG nodes.
//
// The reference deposits particle by particle: a face-connected walk from
// the particle's element visits every element its shape ball reaches and
// scatters q S(x_node - x_p) into rho/j (dep_shape.hpp:128-149,
// element_finder.hpp:239-293). The walk reaches exactly the elements that
// intersect the ball (on a convex mesh), and S vanishes at and beyond the
// radius, so the result is, for every node, the sum of the contributions of
// every particle within one radius of it. That value depends only on the
// node's position, and DG nodes on shared faces, edges and vertices are
// coincident (order 3: about 4.3 distinct positions per tetrahedron for 20
// nodes). This file computes the sum as a gather over the distinct
// positions, which needs no floating-point atomics and is deterministic:
//
//   1. set-up (host, once per mesh): merge coincident nodes into positions,
//      order them along a Morton curve, cut the order into warp groups
//      (<= 32 positions at Morton cells of ~24) and wide groups (<= 64, two
//      positions per lane), each with its bounding sphere;
//   2. per call: bin the particles (bin width radius/2), radix sort by bin,
//      pack a 64-byte payload per particle in bin order; estimate each
//      group's work (the particles of its bin rows) and launch the groups
//      heaviest first;
//   3. one warp per group, warps independent: the warp streams the
//      particles of the bin rows within the radius of its box straight from
//      L2, culls them against the box grown by the radius, appends the
//      survivors to a private shared-memory ring (ballot), and every 32
//      entries the lanes walk the batch with a branch-free weight, two
//      positions per lane; rho, j accumulate in a fixed order;
//   4. expand: every node takes its position's values.
//
// The chosen form's tensor-core deposition (deposit_tc.cu) shares steps 1,
// 2 and 4 and replaces step 3.
//
// Periodic axes use particle images shifted by the period, the images the
// walk uses when it crosses a periodic face.

#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "binning.cuh"
#include "gather.cuh"

namespace prt_dep {

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
  long long lo = 0, hi = n;  // lower_bound of b
  while (lo < hi) {
    long long mid = (lo + hi) >> 1;
    if ((long long)sorted_keys[mid] < b)
      lo = mid + 1;
    else
      hi = mid;
  }
  starts[b] = (uint32_t)lo;
}

__global__ void payload_kernel(long long n, const uint32_t *__restrict__ perm,
                               const double *__restrict__ x, const double *__restrict__ q,
                               const double *__restrict__ v,
                               const double *__restrict__ scale, double normalizer,
                               const uint32_t *__restrict__ tag, double *__restrict__ out) {
  long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = perm[s];
  double w = scale ? scale[i] * normalizer : q[i] * normalizer;
  double2 *o = reinterpret_cast<double2 *>(out + PAYLOAD * s);
  double v0 = 0, v1 = 0, v2 = 0;
  if (v) {
    v0 = w * v[i];
    v1 = w * v[n + i];
    v2 = w * v[2 * n + i];
  }
  o[0] = make_double2(x[i], x[n + i]);
  o[1] = make_double2(x[2 * n + i], w);
  o[2] = make_double2(v0, v1);
  o[3] = make_double2(v2, tag ? (double)tag[i] : 0.0);
}

int choose_bins(const prt_mesh *m, const double box_lo[3], const double box_hi[3],
                double bin_width, double radius, BinGrid &G, int *rc) {
  *rc = PRT_OK;
  long long nb = 1;
  for (int d = 0; d < 3; ++d) {
    const bool per = m->dev.pmin[d] != m->dev.pmax[d];
    G.periodic[d] = per;
    const double lo = per ? m->dev.pmin[d] : box_lo[d];
    const double hi = per ? m->dev.pmax[d] : box_hi[d];
    const double ext = hi - lo;
    const double w = bin_width > 0 ? bin_width : ext;
    int dims = ext > 0 ? (int)std::max(1.0, std::floor(ext / w)) : 1;
    dims = std::min(dims, 1024);
    const double width = ext > 0 ? ext / dims : 1.0;
    if (per && radius * 2 >= ext) {
      *rc = PRT_ERR_INVALID_ARGUMENT;  // a ball would meet its own image
      return 0;
    }
    G.origin[d] = lo;
    G.inv_w[d] = 1.0 / width;
    G.w[d] = width;
    G.slack[d] = 1e-6 * width + 1e-9 * std::max(std::fabs(lo), std::fabs(hi));
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

int stage_particles(prt_workspace *ws, const BinGrid &G, long long n, const double *x,
                    const double *q, const double *v, const uint32_t *el,
                    const double *scale, double normalizer, const uint32_t *tag,
                    DepParticles &P, cudaStream_t s) {
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
  // rows past starts[nbins] (removed particles) are packed but never read
  payload_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(n, vals_out, x, q, v, scale,
                                                         normalizer, tag, payload);
  PRT_CHECK_CUDA(cudaGetLastError());
  P.payload = payload;
  P.starts = starts;
  return PRT_OK;
}

}  // namespace prt_dep

namespace {

using namespace prt_dep;

constexpr int WARPS = BLOCK / 32;

// resident CTAs per SM the group kernel is compiled for (register budget)
#ifndef PRT_GATHER_MIN_BLOCKS
#define PRT_GATHER_MIN_BLOCKS 6
#endif
// the same for the two-positions-per-lane form (twice the accumulators)
#ifndef PRT_GATHER_MIN_BLOCKS_WIDE
#define PRT_GATHER_MIN_BLOCKS_WIDE 4
#endif
// mixed form, wide groups: 6 CTAs (80 registers, no spills) measured best
// with the heaviest groups first: 8 CTAs cost ~20% on dense bunches
// (config4) and 4 CTAs ~15% on config2
#ifndef PRT_MIXED_MIN_BLOCKS_WIDE
#define PRT_MIXED_MIN_BLOCKS_WIDE 6
#endif
// positions per lane of the FP64 and mixed deposition (2: wide groups)
#ifndef PRT_FP64_PPL
#define PRT_FP64_PPL 2
#endif
#ifndef PRT_MIXED_PPL
#define PRT_MIXED_PPL 2
#endif
// unrolling of the full-batch loops (two entries per step)
#ifndef PRT_FP64_UNROLL
#define PRT_FP64_UNROLL 4
#endif
#ifndef PRT_MIXED_UNROLL
#define PRT_MIXED_UNROLL 4
#endif
constexpr int FP64_UNROLL = PRT_FP64_UNROLL;
// launch the position groups heaviest first (1) or in Morton order (0)
#ifndef PRT_DEPOSIT_HEAVY_FIRST
#define PRT_DEPOSIT_HEAVY_FIRST 1
#endif
constexpr int MIXED_UNROLL = PRT_MIXED_UNROLL;
// per-warp ring of compacted particles (two batches of 32)
constexpr int RING = 64;

// Streams the candidate particles of one warp's position group: the
// particles of the bin rows that can come within `radius` of the group's box
// [c + lo, c + hi], 32 at a time (one per lane, straight from L2/L1). Calls
// visit(in, k, w0, w1, w2) on every lane for every batch (warp-uniform),
// with w the particle's position relative to c (periodic images shifted by
// the period) and `in` set when the particle may lie within the radius of
// the box (never cleared for one that does), hence possibly within the
// radius of a position.
template <class Visit>
__device__ __forceinline__ void stream_box(const BinGrid &G, const DepParticles &P,
                                           const double c[3], const double lo[3],
                                           const double hi[3], double radius, int lane,
                                           Visit &&visit) {
  // The culls only decide which particles are evaluated (a particle beyond
  // the radius gets weight 0 anyway), so they run on few registers: the box
  // as FP32 centre and half-extent (relative to c) grown by 1e-5 of the
  // radius, which covers their FP32 rounding, and the per-particle test in
  // FP32 on the FP64 offsets rounded to FP32.
  const double rr = radius * (1 + 1e-5), rr2 = rr * rr;
  const float rcf = (float)rr;
  const float rc4 = 4.0f * rcf * rcf;
  float midf[3], halff[3];
  int ulo[3], uhi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    midf[d] = (float)(0.5 * (lo[d] + hi[d]));
    halff[d] = (float)(0.5 * (hi[d] - lo[d]) + 1e-5 * radius);
    ulo[d] = bin_floor(G, d, c[d] + lo[d] - radius);
    uhi[d] = bin_floor(G, d, c[d] + hi[d] + radius);
    if (G.periodic[d]) {
      ulo[d] -= 1;
      uhi[d] += 1;
    } else {
      ulo[d] = max(ulo[d], 0);
      uhi[d] = min(uhi[d], G.dims[d] - 1);
    }
  }
  const double2 *__restrict__ pay = reinterpret_cast<const double2 *>(P.payload);
  // distance from the slab [blo, blo + w) of bins to the box along one axis
  auto slab_gap = [&](int d, double blo) {
    const double m = c[d] + (double)midf[d], h = (double)halff[d];
    const double e = fmax(0.0, fmax(blo - (m + h), (m - h) - (blo + G.w[d]))) - G.slack[d];
    return e > 0 ? e * e : 0.0;
  };
  for (int bz = ulo[2]; bz <= uhi[2]; ++bz) {
    int wz = bz, qz = 0;
    if (G.periodic[2]) { qz = floor_div(bz, G.dims[2]); wz = bz - qz * G.dims[2]; }
    const double sz = qz * G.period[2] - c[2];
    const double dz2 = slab_gap(2, G.origin[2] + bz * G.w[2]);
    if (dz2 > rr2) continue;
    for (int by = ulo[1]; by <= uhi[1]; ++by) {
      int wy = by, qy = 0;
      if (G.periodic[1]) { qy = floor_div(by, G.dims[1]); wy = by - qy * G.dims[1]; }
      const double sy = qy * G.period[1] - c[1];
      const double dyz2 = dz2 + slab_gap(1, G.origin[1] + by * G.w[1]);
      if (dyz2 > rr2) continue;
      const double rem = sqrt(rr2 - dyz2);
      const double m0 = c[0] + (double)midf[0], h0 = (double)halff[0];
      int bx0 = bin_floor(G, 0, m0 - h0 - rem);
      int bx1 = bin_floor(G, 0, m0 + h0 + rem);
      if (G.periodic[0]) {
        bx0 -= 1;
        bx1 += 1;
      }
      bx0 = max(bx0, ulo[0]);
      bx1 = min(bx1, uhi[0]);
      int bx = bx0;
      while (bx <= bx1) {
        int wx = bx, qx = 0, seg_end = bx1;
        if (G.periodic[0]) {
          qx = floor_div(bx, G.dims[0]);
          wx = bx - qx * G.dims[0];
          seg_end = min(bx1, (qx + 1) * G.dims[0] - 1);
        }
        const double sx = qx * G.period[0] - c[0];
        const long long row = (long long)G.dims[0] * (wy + (long long)G.dims[1] * wz);
        const uint32_t s0 = P.starts[row + wx];
        const uint32_t s1 = P.starts[row + wx + (seg_end - bx) + 1];
        bx = seg_end + 1;
        for (uint32_t b0 = s0; b0 < s1; b0 += 32) {
          const uint32_t k = b0 + lane;
          bool in = false;
          double w0 = 0, w1 = 0, w2 = 0;
          if (k < s1) {
            const double2 xy = pay[4 * (size_t)k], zq = pay[4 * (size_t)k + 1];
            w0 = xy.x + sx;
            w1 = xy.y + sy;
            w2 = zq.x + sz;
            // per axis 2 max(|w - mid| - half, 0) = d + |d|
            const float d0 = fabsf((float)w0 - midf[0]) - halff[0];
            const float d1 = fabsf((float)w1 - midf[1]) - halff[1];
            const float d2a = fabsf((float)w2 - midf[2]) - halff[2];
            const float e0 = d0 + fabsf(d0), e1 = d1 + fabsf(d1), e2 = d2a + fabsf(d2a);
            in = e0 * e0 + e1 * e1 + e2 * e2 <= rc4;
          }
          visit(in, k, w0, w1, w2);
        }
      }
    }
  }
}

// Bounding box [lo, hi] (relative to c) of the positions a warp holds.
template <int PPL>
__device__ __forceinline__ void warp_box(const double *__restrict__ pos, uint32_t p0, int npg,
                                         int lane, const double c[3], double lo[3],
                                         double hi[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = INFINITY;
    hi[d] = -INFINITY;
  }
#pragma unroll
  for (int h = 0; h < PPL; ++h)
    if (lane + 32 * h < npg) {
      const long long u = p0 + lane + 32 * h;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo[d] = fmin(lo[d], pos[3 * u + d] - c[d]);
        hi[d] = fmax(hi[d], pos[3 * u + d] - c[d]);
      }
    }
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
}

// Work estimate per position group: the particles in the bin rows of its
// sphere grown by the radius (periodic images ignored), keyed for a
// descending sort so that the heaviest groups start first and the light
// ones fill the tail of the launch. Each group is still walked by one warp,
// so the order changes no result.
__global__ void group_work_kernel(long long ngroups, const double *__restrict__ gspheres,
                                  BinGrid G, const uint32_t *__restrict__ starts,
                                  double radius, uint32_t *__restrict__ work,
                                  uint32_t *__restrict__ ids) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const double r = gspheres[4 * g + 3] + radius;
  int lo[3], hi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo[d] = max(0, min(G.dims[d] - 1, bin_floor(G, d, gspheres[4 * g + d] - r)));
    hi[d] = max(0, min(G.dims[d] - 1, bin_floor(G, d, gspheres[4 * g + d] + r)));
  }
  unsigned long long wsum = 0;
  for (int bz = lo[2]; bz <= hi[2]; ++bz)
    for (int by = lo[1]; by <= hi[1]; ++by) {
      const long long row = (long long)G.dims[0] * (by + (long long)G.dims[1] * bz);
      wsum += starts[row + hi[0] + 1] - starts[row + lo[0]];
    }
  work[g] = (uint32_t)min(wsum, 0xffffffffull);
  ids[g] = (uint32_t)g;
}

// One warp per position group (<= 32 positions, one per lane), warps fully
// independent (no block-level barrier). The warp streams the particles of
// the bin rows within its sphere grown by the radius straight from L2/L1:
// each lane tests one particle on the payload's first 32-byte sector
// (x, y, z, q N); the survivors' weights are fetched and appended to the
// warp's shared-memory ring (warp ballot); every 32 entries the lanes walk
// the batch, two particles per iteration. Coordinates are relative to the
// group centre c: r^2 = |u|^2 + |w|^2 - 2 u.w with u = x_position - c,
// w = x_particle - c. Output out[4][npos]: rho, j_x, j_y, j_z per position.
// In COUNT mode counters[0] receives the (particle, position) pairs within
// the radius, counters[1] the (particle, node) pairs (positions weighted by
// their node count) and counters[2] the evaluated pairs.
template <bool ALPHA2, bool COUNT, int PPL = 1>
__global__ void __launch_bounds__(BLOCK, PPL == 1 ? PRT_GATHER_MIN_BLOCKS : PRT_GATHER_MIN_BLOCKS_WIDE)
    deposit_groups_kernel(const double *__restrict__ pos, long long ngroups,
                          const uint32_t *__restrict__ gstarts,
                          const double *__restrict__ gspheres,
                          const uint32_t *__restrict__ run_starts, BinGrid G,
                          DepParticles P, ShapeParams S, long long npos,
                          double *__restrict__ out, unsigned long long *__restrict__ counters,
                          const uint32_t *__restrict__ order = nullptr) {
  // ring entries: (wx, wy), (wz, |w|^2), (q N, q N vx), (q N vy, q N vz)
  __shared__ double2 ring[WARPS][4][RING];

  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long gi = blockIdx.x * (long long)WARPS + wid;
  if (gi >= ngroups) return;  // whole warp
  const long long g = order ? (long long)order[gi] : gi;
  const uint32_t p0 = gstarts[g];
  const int npg = (int)(gstarts[g + 1] - p0);
  double2(*R)[RING] = ring[wid];

  const double c0 = gspheres[4 * g], c1 = gspheres[4 * g + 1], c2 = gspheres[4 * g + 2];
  // lane holds positions p0 + lane + 32 h, h < PPL. With u = x_position - c
  // and w = x_particle - c: a - r^2/a = (a - |u|^2/a) - |w|^2/a + (2/a) u.w,
  // so per pair the weight base is three FMAs and an add: B + e + V . w
  double V0[PPL], V1[PPL], V2[PPL], B[PPL];
  bool live[PPL];
  unsigned mult[PPL];
#pragma unroll
  for (int h = 0; h < PPL; ++h) {
    live[h] = lane + 32 * h < npg;
    V0[h] = V1[h] = V2[h] = B[h] = 0;
    mult[h] = 0;
    if (live[h]) {
      const long long u = p0 + lane + 32 * h;
      const double u0 = pos[3 * u] - c0, u1 = pos[3 * u + 1] - c1, u2 = pos[3 * u + 2] - c2;
      B[h] = S.radius - (u0 * u0 + u1 * u1 + u2 * u2) * S.inv_radius;
      V0[h] = 2 * u0 * S.inv_radius;
      V1[h] = 2 * u1 * S.inv_radius;
      V2[h] = 2 * u2 * S.inv_radius;
      if (COUNT) mult[h] = run_starts[u + 1] - run_starts[u];
    }
  }

  double r0[PPL], x0[PPL], y0[PPL], z0[PPL], r1[PPL], x1[PPL], y1[PPL], z1[PPL];
#pragma unroll
  for (int h = 0; h < PPL; ++h) r0[h] = x0[h] = y0[h] = z0[h] = r1[h] = x1[h] = y1[h] = z1[h] = 0;
  unsigned long long npairs = 0, nnode = 0, nevals = 0;

  // shape weight from tr = a - r^2/a (zero beyond the radius)
  // alpha = 2: (tr + |tr|)^2 = 4 max(tr, 0)^2 exactly (one add with an
  // absolute-value operand and one multiply); the sums are scaled by 1/4 at
  // the end, also exactly, so the result equals that of max(tr, 0)^2
  auto weight = [&](double tr) -> double {
    if (ALPHA2) {
      const double t2 = tr + fabs(tr);
      return t2 * t2;
    }
    return tr > 0 ? pow(tr, S.alpha) : 0.0;
  };
  const double wscale = ALPHA2 ? 0.25 : 1.0;
  // one ring entry against the lane's positions
  auto pair = [&](const double2 p, const double2 q, const double2 wq, const double2 wv,
                  double *r, double *x, double *y, double *z) {
#pragma unroll
    for (int h = 0; h < PPL; ++h) {
      const double tr = fma(V0[h], p.x, fma(V1[h], p.y, fma(V2[h], q.x, B[h] + q.y)));
      const double sw = weight(tr);
      r[h] = fma(wq.x, sw, r[h]);
      x[h] = fma(wq.y, sw, x[h]);
      y[h] = fma(wv.x, sw, y[h]);
      z[h] = fma(wv.y, sw, z[h]);
      if (COUNT) {
        const unsigned in = live[h] && tr >= 0;
        npairs += in;
        nnode += in * mult[h];
      }
    }
  };
  int head = 0, count = 0;
  // walks `k` ring entries from head (warp-uniform k)
  auto drain = [&](int k) {
    for (int i = 0; i < k; ++i) {
      const int e = (head + i) & (RING - 1);
      pair(R[0][e], R[1][e], R[2][e], R[3][e], r0, x0, y0, z0);
    }
    if (COUNT && lane == 0) nevals += (unsigned long long)k * (unsigned)npg;
    head = (head + k) & (RING - 1);
    count -= k;
  };
  // a full batch of 32 from head (0 or 32): constant offsets, two entries
  // per step into two sets of accumulators
  auto drain_full = [&]() {
    const double2 *E0 = &R[0][head], *E1 = &R[1][head], *E2 = &R[2][head], *E3 = &R[3][head];
#pragma unroll FP64_UNROLL
    for (int i = 0; i < 32; i += 2) {
      pair(E0[i], E1[i], E2[i], E3[i], r0, x0, y0, z0);
      pair(E0[i + 1], E1[i + 1], E2[i + 1], E3[i + 1], r1, x1, y1, z1);
    }
    if (COUNT && lane == 0) nevals += 32ull * (unsigned)npg;
    head = (head + 32) & (RING - 1);
    count -= 32;
  };

  const double cc[3] = {c0, c1, c2};
  double blo[3], bhi[3];
  warp_box<PPL>(pos, p0, npg, lane, cc, blo, bhi);
  const double2 *__restrict__ pay = reinterpret_cast<const double2 *>(P.payload);
  stream_box(G, P, cc, blo, bhi, S.radius, lane,
             [&](bool in, uint32_t k, double w0, double w1, double w2) {
               const unsigned bal = __ballot_sync(0xffffffffu, in);
               if (in) {
                 const double d2 = w0 * w0 + w1 * w1 + w2 * w2;
                 const double2 zq = pay[4 * (size_t)k + 1];
                 const double2 jv = pay[4 * (size_t)k + 2], jt = pay[4 * (size_t)k + 3];
                 const int slot =
                     (head + count + __popc(bal & ((1u << lane) - 1u))) & (RING - 1);
                 R[0][slot] = make_double2(w0, w1);
                 R[1][slot] = make_double2(w2, -d2 * S.inv_radius);
                 R[2][slot] = make_double2(zq.y, jv.x);
                 R[3][slot] = make_double2(jv.y, jt.x);
               }
               count += __popc(bal);
               __syncwarp();
               if (count >= 32) {
                 drain_full();
                 __syncwarp();
               }
             });
  if (count > 0) drain(count);
  if (COUNT) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      npairs += __shfl_down_sync(0xffffffffu, npairs, o);
      nnode += __shfl_down_sync(0xffffffffu, nnode, o);
    }
    if (lane == 0) {
      if (npairs) atomicAdd(&counters[0], npairs);
      if (nnode) atomicAdd(&counters[1], nnode);
      if (nevals) atomicAdd(&counters[2], nevals);
    }
  }
#pragma unroll
  for (int h = 0; h < PPL; ++h)
    if (live[h]) {
      const long long u = p0 + lane + 32 * h;
      out[u] = (r0[h] + r1[h]) * wscale;
      out[npos + u] = (x0[h] + x1[h]) * wscale;
      out[2 * npos + u] = (y0[h] + y1[h]) * wscale;
      out[3 * npos + u] = (z0[h] + z1[h]) * wscale;
    }
}

// Mixed-precision form of deposit_groups_kernel: the same culling and order,
// with the particle-to-position geometry and the shape weight in FP32
// (coordinates relative to the group centre, taken from the FP64 positions)
// and the contributions summed in FP32 over each batch of 32 ring entries,
// then combined into FP64 per-position accumulators. A ring entry is 32
// bytes: (wx, wy, wz, |w|^2), (qN, qN vx, qN vy, qN vz).
template <bool ALPHA2, int PPL = 1>
__global__ void __launch_bounds__(BLOCK, PPL == 1 ? PRT_GATHER_MIN_BLOCKS : PRT_MIXED_MIN_BLOCKS_WIDE)
    deposit_groups_mixed_kernel(const double *__restrict__ pos, long long ngroups,
                                const uint32_t *__restrict__ gstarts,
                                const double *__restrict__ gspheres, BinGrid G,
                                DepParticles P, ShapeParams S, long long npos,
                                double *__restrict__ out,
                                const uint32_t *__restrict__ order = nullptr) {
  __shared__ float4 ring[WARPS][2][RING];
  // per lane its positions' FP64 sums (rho, j_x, j_y, j_z per position),
  // kept in shared memory: registers go to the streaming state and the
  // batch arithmetic
  __shared__ double acc64[WARPS][4 * PPL][32];

  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long gi = blockIdx.x * (long long)WARPS + wid;
  if (gi >= ngroups) return;  // whole warp
  const long long g = order ? (long long)order[gi] : gi;
  const uint32_t p0 = gstarts[g];
  const int npg = (int)(gstarts[g + 1] - p0);
  float4(*R)[RING] = ring[wid];
  double(*A64)[32] = acc64[wid];

  const double c0 = gspheres[4 * g], c1 = gspheres[4 * g + 1], c2 = gspheres[4 * g + 2];
  // lane holds positions p0 + lane + 32 h, h < PPL; the weight base
  // a - r^2/a = B + e + V . w as in deposit_groups_kernel, B and V rounded
  // to FP32 from FP64
  float V0[PPL], V1[PPL], V2[PPL], B[PPL];
  bool live[PPL];
#pragma unroll
  for (int h = 0; h < PPL; ++h) {
    live[h] = lane + 32 * h < npg;
    V0[h] = V1[h] = V2[h] = B[h] = 0;
    if (live[h]) {
      const long long u = p0 + lane + 32 * h;
      const double u0 = pos[3 * u] - c0, u1 = pos[3 * u + 1] - c1, u2 = pos[3 * u + 2] - c2;
      B[h] = (float)(S.radius - (u0 * u0 + u1 * u1 + u2 * u2) * S.inv_radius);
      V0[h] = (float)(2 * u0 * S.inv_radius);
      V1[h] = (float)(2 * u1 * S.inv_radius);
      V2[h] = (float)(2 * u2 * S.inv_radius);
    }
  }
#pragma unroll
  for (int k = 0; k < 4 * PPL; ++k) A64[k][lane] = 0;
  const float alpha = (float)S.alpha;
  // alpha = 2: (tr + |tr|)^2 = 4 max(tr, 0)^2, the 1/4 applied to the FP64
  // sums at the end (exact)
  auto weight = [&](float tr) -> float {
    if (ALPHA2) {
      const float t2 = tr + fabsf(tr);
      return t2 * t2;
    }
    return tr > 0 ? powf(tr, alpha) : 0.0f;
  };
  const double wscale = ALPHA2 ? 0.25 : 1.0;
  auto pair = [&](const float4 p, const float4 q, float *r, float *x, float *y, float *z) {
#pragma unroll
    for (int h = 0; h < PPL; ++h) {
      const float sw = weight(fmaf(V0[h], p.x, fmaf(V1[h], p.y, fmaf(V2[h], p.z, B[h] + p.w))));
      r[h] = fmaf(q.x, sw, r[h]);
      x[h] = fmaf(q.y, sw, x[h]);
      y[h] = fmaf(q.z, sw, y[h]);
      z[h] = fmaf(q.w, sw, z[h]);
    }
  };
  // FP32 batch sums into the FP64 accumulators
  auto combine = [&](const float *ra, const float *xa, const float *ya, const float *za) {
#pragma unroll
    for (int h = 0; h < PPL; ++h) {
      A64[4 * h][lane] += (double)ra[h];
      A64[4 * h + 1][lane] += (double)xa[h];
      A64[4 * h + 2][lane] += (double)ya[h];
      A64[4 * h + 3][lane] += (double)za[h];
    }
  };
  int head = 0, count = 0;
  auto drain = [&](int k) {
    float ra[PPL], xa[PPL], ya[PPL], za[PPL];
#pragma unroll
    for (int h = 0; h < PPL; ++h) ra[h] = xa[h] = ya[h] = za[h] = 0;
    for (int i = 0; i < k; ++i) {
      const int e = (head + i) & (RING - 1);
      pair(R[0][e], R[1][e], ra, xa, ya, za);
    }
    combine(ra, xa, ya, za);
    head = (head + k) & (RING - 1);
    count -= k;
  };
  // a full batch of 32 from head (0 or 32): constant offsets, one set of
  // FP32 batch sums (4 PPL independent accumulation chains)
  auto drain_full = [&]() {
    float ra[PPL], xa[PPL], ya[PPL], za[PPL];
#pragma unroll
    for (int h = 0; h < PPL; ++h) ra[h] = xa[h] = ya[h] = za[h] = 0;
    const float4 *E0 = &R[0][head], *E1 = &R[1][head];
#pragma unroll MIXED_UNROLL
    for (int i = 0; i < 32; ++i) pair(E0[i], E1[i], ra, xa, ya, za);
    combine(ra, xa, ya, za);
    head = (head + 32) & (RING - 1);
    count -= 32;
  };

  const double cc[3] = {c0, c1, c2};
  double blo[3], bhi[3];
  warp_box<PPL>(pos, p0, npg, lane, cc, blo, bhi);
  const double2 *__restrict__ pay = reinterpret_cast<const double2 *>(P.payload);
  stream_box(G, P, cc, blo, bhi, S.radius, lane,
             [&](bool in, uint32_t k, double w0, double w1, double w2) {
               const unsigned bal = __ballot_sync(0xffffffffu, in);
               if (in) {
                 const double d2 = w0 * w0 + w1 * w1 + w2 * w2;
                 const double2 zq = pay[4 * (size_t)k + 1];
                 const double2 jv = pay[4 * (size_t)k + 2], jt = pay[4 * (size_t)k + 3];
                 const int slot =
                     (head + count + __popc(bal & ((1u << lane) - 1u))) & (RING - 1);
                 R[0][slot] = make_float4((float)w0, (float)w1, (float)w2,
                                          (float)(-d2 * S.inv_radius));
                 R[1][slot] = make_float4((float)zq.y, (float)jv.x, (float)jv.y, (float)jt.x);
               }
               count += __popc(bal);
               __syncwarp();
               if (count >= 32) {
                 drain_full();
                 __syncwarp();
               }
             });
  if (count > 0) drain(count);
#pragma unroll
  for (int h = 0; h < PPL; ++h)
    if (live[h]) {
      const long long u = p0 + lane + 32 * h;
      out[u] = A64[4 * h][lane] * wscale;
      out[npos + u] = A64[4 * h + 1][lane] * wscale;
      out[2 * npos + u] = A64[4 * h + 2][lane] * wscale;
      out[3 * npos + u] = A64[4 * h + 3][lane] * wscale;
    }
}

// Every node takes the values of its position.
__global__ void expand_kernel(long long nn, long long npos,
                              const uint32_t *__restrict__ node_to_pos,
                              const double *__restrict__ vals, double *__restrict__ rho,
                              double *__restrict__ j) {
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (n >= nn) return;
  const uint32_t u = node_to_pos[n];
  if (rho) rho[n] = vals[u];
  if (j) {
    j[n] = vals[npos + u];
    j[nn + n] = vals[2 * npos + u];
    j[2 * nn + n] = vals[3 * npos + u];
  }
}

// Integration weight of a position: sum over its nodes of w_i |J_e| (the
// normalising depositor's sum_e |J_e| sum_i w_i S_i, dep_normshape.hpp:155-164,
// regrouped by position), in ascending node order.
__global__ void position_weights_kernel(long long npos, const uint32_t *__restrict__ run_starts,
                                        const uint32_t *__restrict__ run_nodes, int np,
                                        const double *__restrict__ iw,
                                        const double *__restrict__ jac,
                                        double *__restrict__ W) {
  long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (u >= npos) return;
  double s = 0;
  for (uint32_t k = run_starts[u]; k < run_starts[u + 1]; ++k) {
    const uint32_t node = run_nodes[k];
    s += iw[node % np] * jac[node / np];
  }
  W[u] = s;
}

// Normalising pre-pass (dep_normshape.hpp:125-199): per particle the
// integral of its deposited shape, sum_u W_u N S(x_u - x_p), over the
// positions within the radius; scale = q / integral, or 0 with a warning for
// a zero integral (the reference skips such a particle). A warp takes 32
// consecutive particles (element-sorted particles are close together), one
// per lane, and walks the position groups near them with the positions and
// W staged in shared memory (gather.cuh); each particle's sum runs in a fixed
// order. hits_out: the positions within the radius (-1 for a dead particle).
constexpr int NORM_WARPS = 4;
template <bool ALPHA2>
__global__ void __launch_bounds__(32 * NORM_WARPS)
    normalize_kernel(DevMesh M, CentreBinsDev CB, const double *__restrict__ pos,
                     long long npos, const double *__restrict__ W, ShapeParams S,
                     double normalizer, long long n, const double *__restrict__ x,
                     const double *__restrict__ q, const uint32_t *__restrict__ el,
                     double *__restrict__ scale_out, double *__restrict__ hits_out,
                     DevStatus *st) {
  __shared__ GatherStage<1> stage[NORM_WARPS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long w0 = (blockIdx.x * (long long)NORM_WARPS + wid) * 32;
  if (w0 >= n) return;  // whole warp
  const long long i = w0 + lane;
  const bool valid = i < n;
  const bool live = valid && !(el && el[i] == PRT_INVALID);
  double p[3] = {0, 0, 0};
  if (live) {
    p[0] = x[i];
    p[1] = x[n + i];
    p[2] = x[2 * n + i];
  }
  double integral = 0, hits = 0;
  warp_gather_positions<1>(M, CB, pos, npos, W, S.radius, live, p, stage[wid],
                           [&](double, double, double, double r2, const double *vals) {
                             const bool in = r2 <= S.radius2;
                             const double rt = S.radius - r2 * S.inv_radius;
                             const double sv =
                                 in ? normalizer * (ALPHA2 ? rt * rt : pow(rt, S.alpha))
                                    : 0.0;
                             integral = fma(sv, vals[0], integral);
                             hits += in ? 1.0 : 0.0;
                           });
  if (!valid) return;
  if (!live) {
    scale_out[i] = 0;
    hits_out[i] = -1;
    return;
  }
  if (integral == 0) {
    scale_out[i] = 0;
    record_warning(st, PRT_WARN_ZERO_MASS, i);
  } else {
    scale_out[i] = q[i] / integral;
  }
  hits_out[i] = hits;
}

// Count / sum / sum of squares / min / max of the applied scales (non-zero
// ones) and of the per-particle position counts (live particles): per block
// partials, then one pass over them in block order (deterministic).
constexpr int STATS_BLOCKS = 592;  // 4 per SM of a 148-SM B200
__device__ __forceinline__ double stats_combine(int k, double a, double b) {
  return (k == 3 || k == 8) ? fmin(a, b) : (k == 4 || k == 9) ? fmax(a, b) : a + b;
}
__global__ void __launch_bounds__(256) stats_kernel(long long n, const double *__restrict__ scale,
                                                    const double *__restrict__ hits,
                                                    double *__restrict__ partials) {
  __shared__ double sh[10][256];
  double acc[10] = {0, 0, 0, INFINITY, -INFINITY, 0, 0, 0, INFINITY, -INFINITY};
  for (long long i = blockIdx.x * 256LL + threadIdx.x; i < n; i += 256LL * gridDim.x) {
    const double c = hits[i];
    if (c < 0) continue;
    acc[5] += 1;
    acc[6] += c;
    acc[7] += c * c;
    acc[8] = fmin(acc[8], c);
    acc[9] = fmax(acc[9], c);
    const double s = scale[i];
    if (s == 0) continue;
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
      for (int k = 0; k < 10; ++k)
        sh[k][threadIdx.x] = stats_combine(k, sh[k][threadIdx.x], sh[k][threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x < 10) partials[10 * (size_t)blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}
__global__ void stats_final_kernel(int blocks, const double *__restrict__ partials,
                                   double *__restrict__ out) {
  const int k = threadIdx.x;
  if (k >= 10) return;
  double a = partials[k];
  for (int b = 1; b < blocks; ++b) a = stats_combine(k, a, partials[10 * (size_t)b + k]);
  out[k] = a;
}

inline uint64_t spread_bits(uint64_t v) {  // 21 bits -> every third bit
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffull;
  v = (v | v << 16) & 0x1f0000ff0000ffull;
  v = (v | v << 8) & 0x100f00f00f00f00full;
  v = (v | v << 4) & 0x10c30c30c30c30c3ull;
  v = (v | v << 2) & 0x1249249249249249ull;
  return v;
}

template <class T>
int upload_vec(const std::vector<T> &v, const T **dst) {
  T *p = nullptr;
  PRT_CHECK_CUDA(cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(T)));
  if (!v.empty()) PRT_CHECK_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  *dst = p;
  return PRT_OK;
}

}  // namespace

// ------------------------------------------------------------ position set

unsigned long long prt_next_target_uid() {
  static std::atomic<unsigned long long> next_uid{1};
  return next_uid++;
}

int prt_mesh_build_positions(prt_mesh *m, const prt_mesh_desc *d) {
  m->uid = prt_next_target_uid();
  const long long E = d->element_count;
  const int Np = d->nodes_per_element;
  const long long nn = E * (long long)Np;
  const double *X = d->nodes;
  for (int a = 0; a < 3; ++a) {
    m->box_lo[a] = INFINITY;
    m->box_hi[a] = -INFINITY;
  }
  for (long long i = 0; i < nn; ++i)
    for (int a = 0; a < 3; ++a) {
      m->box_lo[a] = std::min(m->box_lo[a], X[3 * i + a]);
      m->box_hi[a] = std::max(m->box_hi[a], X[3 * i + a]);
    }
  double ext = 0;
  for (int a = 0; a < 3; ++a) ext = std::max(ext, m->box_hi[a] - m->box_lo[a]);
  if (!(ext > 0)) ext = 1;
  // Morton keys of the nodes quantised to 2^21 cells per axis
  const double scale = (double)((1 << 21) - 1) / ext;
  std::vector<uint64_t> key(nn);
  for (long long i = 0; i < nn; ++i) {
    uint64_t k = 0;
    for (int a = 0; a < 3; ++a) {
      double qv = std::floor((X[3 * i + a] - m->box_lo[a]) * scale);
      qv = std::min(std::max(qv, 0.0), (double)((1 << 21) - 1));
      k |= spread_bits((uint64_t)qv) << a;
    }
    key[i] = k;
  }
  std::vector<uint32_t> order(nn);
  std::iota(order.begin(), order.end(), 0u);
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    return key[a] != key[b] ? key[a] < key[b] : a < b;
  });
  // coincident nodes: same cell and within 1e-9 of the mesh extent
  const double tol2 = (1e-9 * ext) * (1e-9 * ext);
  std::vector<uint32_t> run_starts, node_to_pos(nn);
  std::vector<double> pos;
  run_starts.reserve(nn / 3);
  pos.reserve(nn);
  long long npos = 0;
  for (long long r = 0; r < nn; ++r) {
    const uint32_t i = order[r];
    bool same = false;
    if (r > 0 && key[i] == key[order[r - 1]]) {
      const double *p = &pos[3 * (npos - 1)];
      double s = 0;
      for (int a = 0; a < 3; ++a) s += (X[3 * i + a] - p[a]) * (X[3 * i + a] - p[a]);
      same = s <= tol2;
    }
    if (!same) {
      run_starts.push_back((uint32_t)r);
      for (int a = 0; a < 3; ++a) pos.push_back(X[3 * i + a]);
      ++npos;
    }
    node_to_pos[i] = (uint32_t)(npos - 1);
  }
  run_starts.push_back((uint32_t)nn);
  PositionSet &P = m->positions;
  P.count = npos;
  // host copies for the tensor-core tiles, which are cut per shape radius
  m->pos_host = pos;
  int rc;
  if ((rc = upload_vec(pos, &P.pos))) return rc;
  if ((rc = upload_vec(node_to_pos, &P.node_to_pos))) return rc;
  if ((rc = upload_vec(run_starts, &P.run_starts))) return rc;
  if ((rc = upload_vec(order, &P.run_nodes))) return rc;

  // warp groups: runs of at most 32 positions, cut wherever the Morton cell
  // of about PRT_GROUP_TARGET positions changes, so that no group straddles
  // two cells (compact groups, tight spheres)
  {
    double vol = 1;
    for (int a = 0; a < 3; ++a) vol *= std::max(m->box_hi[a] - m->box_lo[a], 1e-300);
    const double side = std::cbrt(PRT_GROUP_TARGET * vol / std::max<long long>(1, npos));
    int level = (int)std::lround(std::log2(ext / side));
    level = std::min(std::max(level, 0), 21);
    const int shift = 3 * (21 - level);
    // runs of <= maxlen positions cut at Morton cells (key >> cell_shift),
    // with their bounding spheres
    auto build_groups = [&](int cell_shift, long long maxlen, std::vector<uint32_t> &gs,
                            std::vector<double> &sph) {
      gs.clear();
      gs.reserve(npos / 16 + 2);
      uint64_t prev_cell = ~0ull;
      for (long long u = 0; u < npos; ++u) {
        const uint64_t cell = key[order[run_starts[u]]] >> cell_shift;
        if (u == 0 || cell != prev_cell || u - gs.back() >= maxlen) gs.push_back((uint32_t)u);
        prev_cell = cell;
      }
      gs.push_back((uint32_t)npos);
      const long long ng = (long long)gs.size() - 1;
      sph.assign(4 * (size_t)std::max<long long>(1, ng), 0.0);
      for (long long g = 0; g < ng; ++g) {
        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t p = gs[g]; p < gs[g + 1]; ++p)
          for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], pos[3 * p + a]);
            hi[a] = std::max(hi[a], pos[3 * p + a]);
          }
        double c[3], r2 = 0;
        for (int a = 0; a < 3; ++a) c[a] = 0.5 * (lo[a] + hi[a]);
        for (uint32_t p = gs[g]; p < gs[g + 1]; ++p) {
          double s = 0;
          for (int a = 0; a < 3; ++a) s += (pos[3 * p + a] - c[a]) * (pos[3 * p + a] - c[a]);
          r2 = std::max(r2, s);
        }
        for (int a = 0; a < 3; ++a) sph[4 * g + a] = c[a];
        sph[4 * g + 3] = std::sqrt(r2) * (1 + 1e-9) + 1e-300;
      }
    };
    std::vector<uint32_t> gstart;
    std::vector<double> spheres;
    build_groups(shift, PRT_WARP_NODES, gstart, spheres);
    const long long groups = (long long)gstart.size() - 1;
    {
      std::vector<uint32_t> wstart;
      std::vector<double> wsph;
      build_groups(std::min(shift + PRT_WIDE_CELL_BITS, 63), 2 * PRT_WARP_NODES, wstart, wsph);
      P.wide_groups = (long long)wstart.size() - 1;
      if ((rc = upload_vec(wstart, &P.wide_starts))) return rc;
      if ((rc = upload_vec(wsph, &P.wide_spheres))) return rc;
    }
    P.groups = groups;
    if ((rc = upload_vec(gstart, &P.group_starts))) return rc;
    if ((rc = upload_vec(spheres, &P.group_spheres))) return rc;



    // centre bins: width about the mean group radius
    auto &CB = P.centre_bins;
    double rsum = 0, rmax = 0;
    for (long long g = 0; g < groups; ++g) {
      rsum += spheres[4 * g + 3];
      rmax = std::max(rmax, spheres[4 * g + 3]);
    }
    const double wbin = std::max(rsum / std::max<long long>(1, groups), 1e-300);
    long long ncb = 1;
    for (int a = 0; a < 3; ++a) {
      const double e = m->box_hi[a] - m->box_lo[a];
      const int dims = e > 0 ? (int)std::max(1.0, std::min(1024.0, std::floor(e / wbin))) : 1;
      CB.dims[a] = dims;
      CB.origin[a] = m->box_lo[a];
      CB.inv_w[a] = e > 0 ? dims / e : 0.0;
      ncb *= dims;
    }
    CB.max_radius = rmax;
    std::vector<uint32_t> gbin(std::max<long long>(1, groups));
    std::vector<uint32_t> cstarts(ncb + 1, 0);
    for (long long g = 0; g < groups; ++g) {
      long long b = 0, mul = 1;
      for (int a = 0; a < 3; ++a) {
        const double u = std::floor((spheres[4 * g + a] - CB.origin[a]) * CB.inv_w[a]);
        b += mul * (long long)std::max(0.0, std::min(u, CB.dims[a] - 1.0));
        mul *= CB.dims[a];
      }
      gbin[g] = (uint32_t)b;
      ++cstarts[b + 1];
    }
    for (long long b = 0; b < ncb; ++b) cstarts[b + 1] += cstarts[b];
    std::vector<uint32_t> fill(cstarts.begin(), cstarts.end() - 1);
    std::vector<double> csph(4 * (size_t)std::max<long long>(1, groups));
    std::vector<uint32_t> crange(2 * (size_t)std::max<long long>(1, groups));
    for (long long g = 0; g < groups; ++g) {
      const uint32_t k = fill[gbin[g]]++;
      for (int a = 0; a < 4; ++a) csph[4 * k + a] = spheres[4 * g + a];
      crange[2 * k] = gstart[g];
      crange[2 * k + 1] = gstart[g + 1] - gstart[g];
    }
    if ((rc = upload_vec(cstarts, &CB.starts))) return rc;
    if ((rc = upload_vec(csph, &CB.spheres))) return rc;
    if ((rc = upload_vec(crange, &CB.ranges))) return rc;
  }

  return PRT_OK;
}

// ------------------------------------------- pieces shared with deposit_tc.cu

int prt_dep_position_weights(const prt_mesh *mesh, prt_workspace *ws, const double *iw,
                             double *W, cudaStream_t s) {
  int rc;
  double *iwd = (double *)ws_buffer(ws, PRT_WS_DEP_STATS,
                                    sizeof(double) * (64 + mesh->dev.Np + 10 * STATS_BLOCKS), &rc);
  if (!iwd) return rc;
  PRT_CHECK_CUDA(cudaMemcpyAsync(iwd, iw, sizeof(double) * mesh->dev.Np, cudaMemcpyHostToDevice, s));
  const PositionSet &PS = mesh->positions;
  position_weights_kernel<<<prt_grid_blocks(PS.count, 256), 256, 0, s>>>(
      PS.count, PS.run_starts, PS.run_nodes, mesh->dev.Np, iwd, mesh->dev.jacobians, W);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

int prt_dep_norm_stats(prt_workspace *ws, long long n, const double *scale, const double *hits,
                       prt_deposit_stats *stats, cudaStream_t s) {
  int rc;
  double *aux = (double *)ws_buffer(ws, PRT_WS_DEP_COUNT, sizeof(double) * (16 + 10 * STATS_BLOCKS), &rc);
  if (!aux) return rc;
  const long long need = (n + 255) / 256;
  const int sb = (int)(need < 1 ? 1 : need < STATS_BLOCKS ? need : STATS_BLOCKS);
  double *partials = aux + 16;
  stats_kernel<<<sb, 256, 0, s>>>(n, scale, hits, partials);
  PRT_CHECK_CUDA(cudaGetLastError());
  stats_final_kernel<<<1, 32, 0, s>>>(sb, partials, aux);
  PRT_CHECK_CUDA(cudaGetLastError());
  double h[10];
  PRT_CHECK_CUDA(cudaMemcpyAsync(h, aux, sizeof(h), cudaMemcpyDeviceToHost, s));
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
  return PRT_OK;
}

int prt_dep_expand(const prt_mesh *mesh, const double *vals, double *rho, double *j,
                   cudaStream_t s) {
  if (!rho && !j) return PRT_OK;
  const long long nn = mesh->dev.E * (long long)mesh->dev.Np;
  expand_kernel<<<prt_grid_blocks(nn, 256), 256, 0, s>>>(nn, mesh->positions.count,
                                                         mesh->positions.node_to_pos, vals, rho, j);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

// -------------------------------------------------------------- C ABI: mesh

extern "C" int prt_deposit_shape(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                                 prt_shape_function shape, const double *iw, int64_t n,
                                 const double *x, const double *q, const double *v,
                                 const uint32_t *el, double *rho, double *j,
                                 int32_t precision, prt_deposit_stats *stats,
                                 void *stream) {
  if (!mesh || !ws || n < 0 || n >= (1ll << 31)) return PRT_ERR_INVALID_ARGUMENT;
  if (precision != PRT_PRECISION_FP64 && precision != PRT_PRECISION_MIXED &&
      precision != PRT_PRECISION_MIXED_SIMT)
    return PRT_ERR_INVALID_ARGUMENT;
  if (!(shape.radius > 0) || (mode != PRT_DEPOSIT_PLAIN && mode != PRT_DEPOSIT_NORMALIZED))
    return PRT_ERR_INVALID_ARGUMENT;
  if (mode == PRT_DEPOSIT_NORMALIZED && !iw) return PRT_ERR_INVALID_ARGUMENT;
  if (n > 0 && (!x || !q || (j && !v))) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  // the chosen form runs on the tensor cores for the alpha = 2 shape; other
  // exponents take the CUDA-core form
  if (precision == PRT_PRECISION_MIXED && shape.alpha == 2 && n > 0)
    return prt_deposit_shape_tc(mesh, ws, mode, shape, iw, n, x, q, v, el, rho, j, stats, s);
  const long long nn = mesh->dev.E * (long long)mesh->dev.Np;
  const PositionSet &PS = mesh->positions;
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
  if (!choose_bins(mesh, mesh->box_lo, mesh->box_hi, shape.radius * BIN_FRACTION, shape.radius, G, &rc))
    return rc;
  const bool a2 = shape.alpha == 2;

  const double *scale = nullptr;
  if (mode == PRT_DEPOSIT_NORMALIZED) {
    double *sc = (double *)ws_buffer(ws, PRT_WS_DEP_SCALE, 2 * sizeof(double) * (size_t)n, &rc);
    if (!sc) return rc;
    double *aux = (double *)ws_buffer(
        ws, PRT_WS_DEP_STATS,
        sizeof(double) * (64 + mesh->dev.Np + PS.count + 10 * STATS_BLOCKS), &rc);
    if (!aux) return rc;
    double *iwd = aux + 16, *W = aux + 64 + mesh->dev.Np;
    PRT_CHECK_CUDA(cudaMemcpyAsync(iwd, iw, sizeof(double) * mesh->dev.Np,
                                   cudaMemcpyHostToDevice, s));
    position_weights_kernel<<<prt_grid_blocks(PS.count, 256), 256, 0, s>>>(
        PS.count, PS.run_starts, PS.run_nodes, mesh->dev.Np, iwd, mesh->dev.jacobians, W);
    PRT_CHECK_CUDA(cudaGetLastError());
    const CentreBinsDev CB = centre_bins_dev(PS);
    const unsigned nblk = (unsigned)((n + 32 * NORM_WARPS - 1) / (32 * NORM_WARPS));
    {
      ScopedTimer norm_timer(ws, PRT_TIME_DEPOSIT_NORMALIZE, s);
      if (a2)
        normalize_kernel<true><<<nblk, 32 * NORM_WARPS, 0, s>>>(
            mesh->dev, CB, PS.pos, PS.count, W, S, shape.normalizer, n, x, q, el, sc, sc + n,
            ws->status);
      else
        normalize_kernel<false><<<nblk, 32 * NORM_WARPS, 0, s>>>(
            mesh->dev, CB, PS.pos, PS.count, W, S, shape.normalizer, n, x, q, el, sc, sc + n,
            ws->status);
      PRT_CHECK_CUDA(cudaGetLastError());
    }
    if (stats) {
      const long long need = (n + 255) / 256;
      const int sb = (int)(need < STATS_BLOCKS ? need : STATS_BLOCKS);
      double *partials = W + PS.count;
      stats_kernel<<<sb, 256, 0, s>>>(n, sc, sc + n, partials);
      PRT_CHECK_CUDA(cudaGetLastError());
      stats_final_kernel<<<1, 32, 0, s>>>(sb, partials, aux);
      PRT_CHECK_CUDA(cudaGetLastError());
      double h[10];
      PRT_CHECK_CUDA(cudaMemcpyAsync(h, aux, sizeof(h), cudaMemcpyDeviceToHost, s));
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
    if ((rc = stage_particles(ws, G, n, x, q, v, el, scale, shape.normalizer, nullptr, P, s)))
      return rc;
  }
  unsigned long long *counter = nullptr;
  if (stats) {
    counter = (unsigned long long *)ws_buffer(ws, PRT_WS_DEP_COUNT, 64, &rc);
    if (!counter) return rc;
    PRT_CHECK_CUDA(cudaMemsetAsync(counter, 0, 24, s));
  }
  double *vals = (double *)ws_buffer(ws, PRT_WS_DEP_VALUES, 4 * sizeof(double) * PS.count, &rc);
  if (!vals) return rc;
  {
    ScopedTimer timer(ws, PRT_TIME_DEPOSIT_GATHER, s);
    auto groups_for = [&](int ppl, long long &ng, const uint32_t *&gs, const double *&gsp) {
      ng = ppl == 2 ? PS.wide_groups : PS.groups;
      gs = ppl == 2 ? PS.wide_starts : PS.group_starts;
      gsp = ppl == 2 ? PS.wide_spheres : PS.group_spheres;
      return (unsigned)((ng + WARPS - 1) / WARPS);
    };
    long long ng;
    const uint32_t *gs;
    const double *gsp;
    // heaviest groups first (group_work_kernel + a descending radix sort)
    auto heavy_first = [&](long long ngr, const double *sph, const uint32_t **order) -> int {
      *order = nullptr;
      if (!PRT_DEPOSIT_HEAVY_FIRST || ngr < 2) return PRT_OK;
      int rc2;
      uint32_t *buf = (uint32_t *)ws_buffer(ws, PRT_WS_GROUP_ORDER, 16 * (size_t)ngr, &rc2);
      if (!buf) return rc2;
      uint32_t *wk = buf, *ids = buf + ngr, *wk_out = buf + 2 * ngr, *ids_out = buf + 3 * ngr;
      group_work_kernel<<<prt_grid_blocks(ngr, 256), 256, 0, s>>>(ngr, sph, G, P.starts,
                                                                  S.radius, wk, ids);
      PRT_CHECK_CUDA(cudaGetLastError());
      size_t tb = 0;
      PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, wk, wk_out, ids,
                                                               ids_out, (int)ngr, 0, 32, s));
      void *tmp = ws_buffer(ws, PRT_WS_CUB, tb, &rc2);
      if (!tmp) return rc2;
      PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp, tb, wk, wk_out, ids,
                                                               ids_out, (int)ngr, 0, 32, s));
      *order = ids_out;
      return PRT_OK;
    };
    const uint32_t *order = nullptr;
    if (precision != PRT_PRECISION_FP64) {
      constexpr int W = PRT_MIXED_PPL;
      const unsigned nb = groups_for(W, ng, gs, gsp);
      if ((rc = heavy_first(ng, gsp, &order))) return rc;
      if (a2)
        deposit_groups_mixed_kernel<true, W><<<nb, BLOCK, 0, s>>>(PS.pos, ng, gs, gsp, G, P, S,
                                                                  PS.count, vals, order);
      else
        deposit_groups_mixed_kernel<false, W><<<nb, BLOCK, 0, s>>>(PS.pos, ng, gs, gsp, G, P, S,
                                                                   PS.count, vals, order);
    } else {
      constexpr int W = PRT_FP64_PPL;
      const unsigned nb = groups_for(W, ng, gs, gsp);
      if ((rc = heavy_first(ng, gsp, &order))) return rc;
      if (counter) {
        if (a2)
          deposit_groups_kernel<true, true, W><<<nb, BLOCK, 0, s>>>(
              PS.pos, ng, gs, gsp, PS.run_starts, G, P, S, PS.count, vals, counter, order);
        else
          deposit_groups_kernel<false, true, W><<<nb, BLOCK, 0, s>>>(
              PS.pos, ng, gs, gsp, PS.run_starts, G, P, S, PS.count, vals, counter, order);
      } else if (a2) {
        deposit_groups_kernel<true, false, W><<<nb, BLOCK, 0, s>>>(
            PS.pos, ng, gs, gsp, PS.run_starts, G, P, S, PS.count, vals, nullptr, order);
      } else {
        deposit_groups_kernel<false, false, W><<<nb, BLOCK, 0, s>>>(
            PS.pos, ng, gs, gsp, PS.run_starts, G, P, S, PS.count, vals, nullptr, order);
      }
    }
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  if (rho || j) {
    expand_kernel<<<prt_grid_blocks(nn, 256), 256, 0, s>>>(nn, PS.count, PS.node_to_pos, vals,
                                                           rho, j);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  if (counter) {
    unsigned long long h[3] = {0, 0, 0};
    PRT_CHECK_CUDA(cudaMemcpyAsync(h, counter, 24, cudaMemcpyDeviceToHost, s));
    PRT_CHECK_CUDA(cudaStreamSynchronize(s));
    stats->pair_count = (double)h[0];
    stats->node_pair_count = (double)h[1];
    stats->evaluated_pairs = (double)h[2];
  }
  return PRT_OK;
}

// ---------------------------------------------- deposition without allocation
//
// Some callers cannot allocate device memory while they run: an application
// that sizes and reserves all of its GPU memory up front (a fixed memory
// budget, a pool handed to it by a host framework), a real-time loop where a
// cudaMalloc would stall or synchronise the device, or code running where
// allocating is not allowed at all. prt_deposit_shape grows workspace
// buffers on demand, so it cannot serve them. prt_deposit_shape_noalloc runs
// the same plain-form deposition with all of its scratch taken from one
// fixed, file-scope device array instead.

namespace {

// The scratch: PRT_NOALLOC_SCRATCH_BYTES per device, held by every GPU that
// loads this library until the process exits. Host code must not use the
// symbol as an address (it is a host-side stand-in); it asks the runtime for
// the device address once per device (noalloc_scratch_address).
static __device__ __align__(256) unsigned char g_noalloc_scratch[PRT_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
void *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mutex;

// Device address of the scratch for the current device; looked up with
// cudaGetSymbolAddress on the first call per device and cached for the life
// of the process (a cudaDeviceReset, which tears down the context that owns
// the array, leaves the cached address stale).
int noalloc_scratch_address(void **out) {
  int dev = 0;
  PRT_CHECK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return PRT_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    PRT_CHECK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return PRT_ERR_CUDA;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return PRT_OK;
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int prt_deposit_shape_noalloc(const prt_mesh *mesh, prt_shape_function shape,
                                         int64_t n, const double *x, const double *q,
                                         const double *v, const uint32_t *el, double *rho,
                                         double *j, void *stream) {
  if (!mesh || n < 0 || n >= (1ll << 31) || !(shape.radius > 0)) return PRT_ERR_INVALID_ARGUMENT;
  const PositionSet &PS = mesh->positions;
  const long long nn = mesh->dev.E * (long long)mesh->dev.Np;
  int rc;
  BinGrid G;
  if (!choose_bins(mesh, mesh->box_lo, mesh->box_hi, shape.radius * BIN_FRACTION, shape.radius,
                   G, &rc))
    return rc;
  // scratch layout: keys, sorted keys, values, sorted values, bin starts,
  // packed particles, position sums, radix-sort temporary storage
  size_t cub_bytes = 0;
  int bits = 1;
  while ((1ll << bits) <= G.nbins) ++bits;
  PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (uint32_t *)nullptr,
                                                 (uint32_t *)nullptr, (uint32_t *)nullptr,
                                                 (uint32_t *)nullptr, (int)std::max<int64_t>(n, 1),
                                                 0, bits, (cudaStream_t)stream));
  const size_t b_keys = align256(4 * (size_t)n);
  const size_t b_starts = align256(4 * (size_t)(G.nbins + 2));
  const size_t b_payload = align256(sizeof(double) * PAYLOAD * (size_t)n);
  const size_t b_vals = align256(4 * sizeof(double) * (size_t)PS.count);
  const size_t need = 4 * b_keys + b_starts + b_payload + b_vals + align256(cub_bytes);
  if (need > (size_t)PRT_NOALLOC_SCRATCH_BYTES) return PRT_ERR_CAPACITY;
  if (n > 0 && (!x || !q || (j && !v))) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  if (!rho && !j) return PRT_OK;  // nothing requested: no work
  if (n == 0) {
    if (rho) PRT_CHECK_CUDA(cudaMemsetAsync(rho, 0, nn * sizeof(double), s));
    if (j) PRT_CHECK_CUDA(cudaMemsetAsync(j, 0, 3 * nn * sizeof(double), s));
    return PRT_OK;
  }
  void *base = nullptr;
  if ((rc = noalloc_scratch_address(&base))) return rc;
  char *p = (char *)base;
  uint32_t *keys = (uint32_t *)p;
  uint32_t *keys_out = (uint32_t *)(p += b_keys);
  uint32_t *vals = (uint32_t *)(p += b_keys);
  uint32_t *vals_out = (uint32_t *)(p += b_keys);
  uint32_t *starts = (uint32_t *)(p += b_keys);
  double *payload = (double *)(p += b_starts);
  double *posvals = (double *)(p += b_payload);
  void *cub_temp = (void *)(p += b_vals);
  // every region is fully written before it is read, so the contents left
  // by an earlier call need no clearing
  bin_keys_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(G, n, x, el, keys, vals);
  PRT_CHECK_CUDA(cudaGetLastError());
  PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(cub_temp, cub_bytes, keys, keys_out, vals,
                                                 vals_out, (int)n, 0, bits, s));
  bin_starts_kernel<<<prt_grid_blocks(G.nbins + 1, 256), 256, 0, s>>>(G.nbins, n, keys_out,
                                                                      starts);
  PRT_CHECK_CUDA(cudaGetLastError());
  payload_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(n, vals_out, x, q, v, nullptr,
                                                         shape.normalizer, nullptr, payload);
  PRT_CHECK_CUDA(cudaGetLastError());
  DepParticles P;
  P.payload = payload;
  P.starts = starts;
  ShapeParams S;
  S.radius = shape.radius;
  S.radius2 = shape.radius * shape.radius;
  S.inv_radius = 1.0 / shape.radius;
  S.alpha = shape.alpha;
  for (int d = 0; d < 3; ++d) S.reach[d] = shape.radius;
  const unsigned nb = (unsigned)((PS.groups + WARPS - 1) / WARPS);
  if (shape.alpha == 2)
    deposit_groups_kernel<true, false><<<nb, BLOCK, 0, s>>>(
        PS.pos, PS.groups, PS.group_starts, PS.group_spheres, PS.run_starts, G, P, S, PS.count,
        posvals, nullptr);
  else
    deposit_groups_kernel<false, false><<<nb, BLOCK, 0, s>>>(
        PS.pos, PS.groups, PS.group_starts, PS.group_spheres, PS.run_starts, G, P, S, PS.count,
        posvals, nullptr);
  PRT_CHECK_CUDA(cudaGetLastError());
  if (rho || j) {
    expand_kernel<<<prt_grid_blocks(nn, 256), 256, 0, s>>>(nn, PS.count, PS.node_to_pos,
                                                           posvals, rho, j);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  return PRT_OK;
}
