// gather.cuh -- particle-centric gathers over the node positions within the
// shape radius (lane = particle), shared by the deposition adjoint and the
// averaging pusher.
//
// A warp takes 32 consecutive particles (element-sorted particles are
// spatially close) and walks the position groups whose centre bin lies
// within radius + (largest group radius) of the warp's bounding box: the
// lanes test 32 candidate groups at a time against the box (ballot), then
// for each surviving group that reaches some lane's particle the warp stages
// the group's positions and NV per-position values in shared memory and
// every lane visits its particle against all of them with
// f(e0, e1, e2, r2, vals) (e = x_position - x_particle), branch-free: the
// callee gives zero weight beyond the radius. Each particle's sums run in a
// fixed order (deterministic). Periodic axes: the warp also walks the images
// of its box shifted by a period where the box comes within the radius of
// the periodicity interval's end.
#pragma once

#include "binning.cuh"

struct CentreBinsDev {
  double origin[3], inv_w[3];
  int dims[3];
  double max_radius;
  const uint32_t *__restrict__ starts;
  const double *__restrict__ spheres;
  const uint32_t *__restrict__ ranges;
};

inline CentreBinsDev centre_bins_dev(const PositionSet &PS) {
  CentreBinsDev CB;
  for (int d = 0; d < 3; ++d) {
    CB.origin[d] = PS.centre_bins.origin[d];
    CB.inv_w[d] = PS.centre_bins.inv_w[d];
    CB.dims[d] = PS.centre_bins.dims[d];
  }
  CB.max_radius = PS.centre_bins.max_radius;
  CB.starts = PS.centre_bins.starts;
  CB.spheres = PS.centre_bins.spheres;
  CB.ranges = PS.centre_bins.ranges;
  return CB;
}

// Staging per warp: 32 positions x (3 + NV) doubles, rounded up to an even
// count (double2 accesses).
template <int NV>
struct GatherStage {
  static constexpr int W = (3 + NV + 1) / 2;  // double2 per position
  double2 v[32][W];
};

// `live`: this lane has a particle at p[3]; all 32 lanes must call.
template <int NV, class Fn>
__device__ __forceinline__ void warp_gather_positions(const DevMesh &M, const CentreBinsDev &CB,
                                                      const double *__restrict__ pos,
                                                      long long npos,
                                                      const double *__restrict__ G,
                                                      double radius, bool live,
                                                      const double p[3], GatherStage<NV> &stg,
                                                      Fn &&f) {
  const int lane = threadIdx.x & 31;
  if (!__any_sync(0xffffffffu, live)) return;  // warp-uniform
  double blo[3], bhi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    blo[d] = live ? p[d] : INFINITY;
    bhi[d] = live ? p[d] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      blo[d] = fmin(blo[d], __shfl_xor_sync(0xffffffffu, blo[d], o));
      bhi[d] = fmax(bhi[d], __shfl_xor_sync(0xffffffffu, bhi[d], o));
    }
  }
  int lo_img[3], hi_img[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    lo_img[d] = hi_img[d] = 0;
    if (M.pmin[d] != M.pmax[d]) {
      if (blo[d] - radius < M.pmin[d]) hi_img[d] = 1;
      if (bhi[d] + radius > M.pmax[d]) lo_img[d] = -1;
    }
  }
  const double reach = radius + CB.max_radius;
  for (int iz = lo_img[2]; iz <= hi_img[2]; ++iz)
    for (int iy = lo_img[1]; iy <= hi_img[1]; ++iy)
      for (int ix = lo_img[0]; ix <= hi_img[0]; ++ix) {
        const double sh[3] = {ix * (M.pmax[0] - M.pmin[0]), iy * (M.pmax[1] - M.pmin[1]),
                              iz * (M.pmax[2] - M.pmin[2])};
        const double c0 = p[0] + sh[0], c1 = p[1] + sh[1], c2 = p[2] + sh[2];
        double qlo[3], qhi[3];
        int b0[3], b1[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          qlo[d] = blo[d] + sh[d];
          qhi[d] = bhi[d] + sh[d];
          const double l = floor((qlo[d] - reach - CB.origin[d]) * CB.inv_w[d]);
          const double h = floor((qhi[d] + reach - CB.origin[d]) * CB.inv_w[d]);
          b0[d] = (int)fmax(0.0, fmin(l, CB.dims[d] - 1.0));
          b1[d] = (int)fmax(0.0, fmin(h, CB.dims[d] - 1.0));
        }
        for (int bz = b0[2]; bz <= b1[2]; ++bz)
          for (int by = b0[1]; by <= b1[1]; ++by) {
            const long long row = (long long)CB.dims[0] * (by + (long long)CB.dims[1] * bz);
            const uint32_t k0 = CB.starts[row + b0[0]], k1 = CB.starts[row + b1[0] + 1];
            for (uint32_t kb = k0; kb < k1; kb += 32) {
              const uint32_t k = kb + lane;
              bool cand = false;
              if (k < k1) {
                const double *sp = CB.spheres + 4 * (size_t)k;
                double d2 = 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                  const double e = fmax(0.0, fmax(qlo[d] - sp[d], sp[d] - qhi[d]));
                  d2 = fma(e, e, d2);
                }
                const double lim = radius + sp[3];
                cand = d2 <= lim * lim;
              }
              unsigned mask = __ballot_sync(0xffffffffu, cand);
              while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1;
                const uint32_t kk = kb + j;
                const double *sp = CB.spheres + 4 * (size_t)kk;
                const double e0 = sp[0] - c0, e1 = sp[1] - c1, e2 = sp[2] - c2;
                const double lim = radius + sp[3];
                const bool hit = live && e0 * e0 + e1 * e1 + e2 * e2 <= lim * lim;
                if (!__any_sync(0xffffffffu, hit)) continue;
                const uint32_t u0 = CB.ranges[2 * (size_t)kk], cnt = CB.ranges[2 * (size_t)kk + 1];
                if ((uint32_t)lane < cnt) {
                  const long long u = u0 + lane;
                  double row_v[2 * GatherStage<NV>::W];
                  row_v[0] = pos[3 * u];
                  row_v[1] = pos[3 * u + 1];
                  row_v[2] = pos[3 * u + 2];
#pragma unroll
                  for (int k2 = 0; k2 < NV; ++k2) row_v[3 + k2] = G[k2 * npos + u];
#pragma unroll
                  for (int k2 = 3 + NV; k2 < 2 * GatherStage<NV>::W; ++k2) row_v[k2] = 0.0;
#pragma unroll
                  for (int w2 = 0; w2 < GatherStage<NV>::W; ++w2)
                    stg.v[lane][w2] = make_double2(row_v[2 * w2], row_v[2 * w2 + 1]);
                }
                __syncwarp();
                for (uint32_t t = 0; t < cnt; ++t) {
                  double row_v[2 * GatherStage<NV>::W];
#pragma unroll
                  for (int w2 = 0; w2 < GatherStage<NV>::W; ++w2) {
                    const double2 dv = stg.v[t][w2];
                    row_v[2 * w2] = dv.x;
                    row_v[2 * w2 + 1] = dv.y;
                  }
                  const double f0 = row_v[0] - c0, f1 = row_v[1] - c1, f2 = row_v[2] - c2;
                  const double r2 = fma(f0, f0, fma(f1, f1, f2 * f2));
                  f(f0, f1, f2, r2, row_v + 3);
                }
                __syncwarp();
              }
            }
          }
      }
}
