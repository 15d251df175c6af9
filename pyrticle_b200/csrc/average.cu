// average.cu -- the averaging pusher (push_average.hpp:26-420): forces from
// the shape-weighted averages of the fields over the nodes within the
// depositor's radius, and the RK update from given forces.
//
// The reference deposits each particle's shape onto the elements its walk
// reaches and accumulates, per element and node, |J_e| w_i rho_i F_i and
// |J_e| w_i rho_i (rho_i = q S(x_i - x_p), w = M 1 the integration weights);
// the force is q <E> + v x (q <B>) with <F> = sum |J| w S F / sum |J| w S
// (the charge cancels). The same sums regroup by node position:
//   <F> = sum_u S(x_u - x_p) WF_u / sum_u S(x_u - x_p) W_u,
// W_u = sum over the nodes at u of |J| w, WF_u = sum |J| w F. A per-position
// pass builds W, WE, WB and the weighted squares (for the verbose standard
// deviations); a particle-centric gather (gather.cuh, lane = particle) forms
// the averages. No atomics; deterministic.

#include <cmath>

#include "gather.cuh"
#include "push.cuh"

namespace {

constexpr int AVG_BLOCK = 128;
constexpr int AVG_NV = 9;  // W, WE[3], WB[3], W|E|^2, W|B|^2

__global__ void average_prepare_kernel(long long npos, int np,
                                       const uint32_t *__restrict__ run_starts,
                                       const uint32_t *__restrict__ run_nodes,
                                       const double *__restrict__ iw,
                                       const double *__restrict__ jac, Fields6 F,
                                       double *__restrict__ G) {
  const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (u >= npos) return;
  double s[AVG_NV];
#pragma unroll
  for (int k = 0; k < AVG_NV; ++k) s[k] = 0;
  for (uint32_t k = run_starts[u]; k < run_starts[u + 1]; ++k) {
    const uint32_t node = run_nodes[k];
    const double w = iw[node % np] * jac[node / np];
    double f[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) f[c] = F.f[c] ? F.f[c][node] : 0.0;
    s[0] += w;
#pragma unroll
    for (int c = 0; c < 6; ++c) s[1 + c] += w * f[c];
    s[7] += w * (f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    s[8] += w * (f[3] * f[3] + f[4] * f[4] + f[5] * f[5]);
  }
#pragma unroll
  for (int k = 0; k < AVG_NV; ++k) G[k * npos + u] = s[k];
}

// vis rows [14][n]: pt_e (3), pt_b (3), pt_e_stddev, pt_b_stddev, el_force
// (3), mag_force (3) (push_average.hpp:388-421)
template <bool ALPHA2>
__global__ void __launch_bounds__(AVG_BLOCK, 4)
    average_forces_kernel(DevMesh M, CentreBinsDev CB, const double *__restrict__ pos,
                          long long npos, prt_dep::ShapeParams S, double normalizer,
                          const double *__restrict__ G, long long n,
                          const double *__restrict__ x, const double *__restrict__ q,
                          const double *__restrict__ v, const uint32_t *__restrict__ el,
                          double *__restrict__ forces, double *__restrict__ vis,
                          double *__restrict__ scales, DevStatus *st) {
  __shared__ GatherStage<AVG_NV> stage[AVG_BLOCK / 32];
  const int warp = threadIdx.x >> 5;
  const long long i = blockIdx.x * (long long)AVG_BLOCK + threadIdx.x;
  const bool live = i < n && (!el || el[i] != PRT_INVALID);
  double p[3] = {0, 0, 0};
  if (live) {
#pragma unroll
    for (int d = 0; d < 3; ++d) p[d] = x[d * n + i];
  }
  double acc[AVG_NV];
#pragma unroll
  for (int k = 0; k < AVG_NV; ++k) acc[k] = 0;
  warp_gather_positions<AVG_NV>(
      M, CB, pos, npos, G, S.radius, live, p, stage[warp],
      [&](double, double, double, double r2, const double *g) {
        const double rt = fmax(fma(-r2, S.inv_radius, S.radius), 0.0);
        const double sw = normalizer * (ALPHA2 ? rt * rt : (rt > 0 ? pow(rt, S.alpha) : 0.0));
#pragma unroll
        for (int k = 0; k < AVG_NV; ++k) acc[k] = fma(sw, g[k], acc[k]);
      });
  if (!live) return;
  const double charge = q[i];
  double f[3] = {0, 0, 0}, ef[6] = {0, 0, 0, 0, 0, 0}, sde = 0, sdb = 0;
  const double den = charge * acc[0];  // the reconstructed charge
  double el_f[3] = {0, 0, 0}, mag_f[3] = {0, 0, 0};
  if (den == 0) {
    record_warning(st, PRT_WARN_ZERO_AVERAGE, i);
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) ef[c] = acc[1 + c] / acc[0];
    const double vv[3] = {v[i], v[n + i], v[2 * n + i]};
    double qb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      el_f[d] = charge * ef[d];
      qb[d] = charge * ef[3 + d];
    }
    mag_f[0] = vv[1] * qb[2] - vv[2] * qb[1];
    mag_f[1] = vv[2] * qb[0] - vv[0] * qb[2];
    mag_f[2] = vv[0] * qb[1] - vv[1] * qb[0];
#pragma unroll
    for (int d = 0; d < 3; ++d) f[d] = el_f[d] + mag_f[d];
    const double ve = acc[7] / acc[0] - (ef[0] * ef[0] + ef[1] * ef[1] + ef[2] * ef[2]);
    const double vb = acc[8] / acc[0] - (ef[3] * ef[3] + ef[4] * ef[4] + ef[5] * ef[5]);
    sde = ve < 0 ? 0.0 : sqrt(ve);
    sdb = vb < 0 ? 0.0 : sqrt(vb);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) forces[d * n + i] = f[d];
  if (scales) scales[i] = den == 0 ? 0.0 : charge / den;
  if (vis) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      vis[d * n + i] = ef[d];
      vis[(3 + d) * n + i] = ef[3 + d];
      vis[(8 + d) * n + i] = el_f[d];
      vis[(11 + d) * n + i] = mag_f[d];
    }
    vis[6 * n + i] = sde;
    vis[7 * n + i] = sdb;
  }
}

// RK update and relocation from given forces (the stage of a pusher whose
// forces come from a separate pass).
__global__ void __launch_bounds__(256)
    lsrk_update_kernel(DevMesh M, long long n, double *__restrict__ x, double *__restrict__ p,
                       const double *__restrict__ mass, uint32_t *__restrict__ el,
                       double *__restrict__ kx, double *__restrict__ kp,
                       const double *__restrict__ forces, double a, double b, double dt,
                       double c, DevStatus *st) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned ctr[4] = {0, 0, 0, 0};
  const uint32_t e = i < n ? el[i] : PRT_INVALID;
  if (e != PRT_INVALID) {
    double xx[3] = {x[i], x[n + i], x[2 * n + i]};
    double pp[3] = {p[i], p[n + i], p[2 * n + i]};
    double v[3];
    velocity_exact(pp[0], pp[1], pp[2], mass[i], c, v[0], v[1], v[2]);
    const double f[3] = {forces[i], forces[n + i], forces[2 * n + i]};
    int err = 0;
    const uint32_t ne = update_particle(M, e, f, v, xx, pp, kx, kp, n, i, a, b, dt, ctr, &err);
    if (err) record_error(st, err, i);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x[d * n + i] = xx[d];
      p[d * n + i] = pp[d];
    }
    if (!err) el[i] = ne;
  }
  flush_counters(st, ctr);
}

}  // namespace

extern "C" int prt_average_forces(const prt_mesh *mesh, prt_workspace *ws,
                                  prt_shape_function shape, const double *integral_weights,
                                  int64_t n, const double *positions, const double *charges,
                                  const double *velocities, const uint32_t *elements,
                                  const double *const fields[6], double *forces, double *vis,
                                  double *scales, void *stream) {
  if (!mesh || !ws || n < 0 || !(shape.radius > 0) || !integral_weights || !fields)
    return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  if (!positions || !charges || !velocities || !forces) return PRT_ERR_INVALID_ARGUMENT;
  const PositionSet &PS = mesh->positions;
  const int np = mesh->dev.Np;
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  double *buf = (double *)ws_buffer(ws, PRT_WS_AVERAGE,
                                    sizeof(double) * ((size_t)AVG_NV * PS.count + np), &rc);
  if (!buf) return rc;
  double *G = buf, *iwd = buf + (size_t)AVG_NV * PS.count;
  PRT_CHECK_CUDA(
      cudaMemcpyAsync(iwd, integral_weights, sizeof(double) * np, cudaMemcpyHostToDevice, s));
  Fields6 F;
  for (int k = 0; k < 6; ++k) F.f[k] = fields[k];
  average_prepare_kernel<<<prt_grid_blocks(PS.count, 256), 256, 0, s>>>(
      PS.count, np, PS.run_starts, PS.run_nodes, iwd, mesh->dev.jacobians, F, G);
  PRT_CHECK_CUDA(cudaGetLastError());
  prt_dep::ShapeParams S;
  S.radius = shape.radius;
  S.radius2 = shape.radius * shape.radius;
  S.inv_radius = 1.0 / shape.radius;
  S.alpha = shape.alpha;
  for (int d = 0; d < 3; ++d) S.reach[d] = shape.radius;
  const CentreBinsDev CB = centre_bins_dev(PS);
  const unsigned blocks = (unsigned)((n + AVG_BLOCK - 1) / AVG_BLOCK);
  if (shape.alpha == 2)
    average_forces_kernel<true><<<blocks, AVG_BLOCK, 0, s>>>(
        mesh->dev, CB, PS.pos, PS.count, S, shape.normalizer, G, n, positions, charges,
        velocities, elements, forces, vis, scales, ws->status);
  else
    average_forces_kernel<false><<<blocks, AVG_BLOCK, 0, s>>>(
        mesh->dev, CB, PS.pos, PS.count, S, shape.normalizer, G, n, positions, charges,
        velocities, elements, forces, vis, scales, ws->status);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

extern "C" int prt_lsrk_update(const prt_mesh *mesh, prt_workspace *ws, int64_t n,
                               double *positions, double *momenta, const double *masses,
                               uint32_t *elements, double *kx, double *kp,
                               const double *forces, double rk_a, double rk_b, double dt,
                               double vacuum_c, void *stream) {
  if (!mesh || !ws || n < 0) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  if (!positions || !momenta || !masses || !elements || !kx || !kp || !forces)
    return PRT_ERR_INVALID_ARGUMENT;
  ScopedTimer timer(ws, PRT_TIME_LSRK_STAGE, (cudaStream_t)stream);
  lsrk_update_kernel<<<prt_grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(
      mesh->dev, n, positions, momenta, masses, elements, kx, kp, forces, rk_a, rk_b, dt,
      vacuum_c, ws->status);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}
