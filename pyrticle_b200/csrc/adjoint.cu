// adjoint.cu -- reverse-mode derivatives of the particle step.
//
// The reference has no derivatives; these kernels differentiate the forward
// kernels of this library (prt_lsrk_stage, prt_get_velocities,
// prt_deposit_shape in plain mode) exactly, treating the containing element
// of every stage as fixed (the element id is piecewise constant in x; the
// fields interpolated from continuous nodal data are continuous across
// faces, so the derivative is that of the smooth branch).
//
// Gather and scatter swap roles: the forward deposition gathers particles
// onto node positions, its adjoint gathers node adjoints onto particles
// (one lane per particle, position groups staged per warp); the forward
// interpolation gathers nodal fields onto particles, its adjoint scatters particle
// adjoints onto the nodes (warp-segmented sums, then FP64 atomics, only when
// nodal field gradients are requested). Gradients along a few basis fields
// (field = sum_k theta_k basis_k + fixed) are reduced per block in a fixed
// order instead, which is deterministic.
//
// Stage adjoint, for the stage  kx' = a kx + dt v(p),  kp' = a kp + dt F(x, p),
// x' = x + b kx',  p' = p + b kp'  (F = q E(x) + q v x B(x)):
//   Lx = lkx' + b lx',  Lp = lkp' + b lp'
//   gE = dt q Lp,  gB = dt q (Lp x v)                  (dL/dE, dL/dB at x)
//   lx = lx' + grad_x [gE . E(x) + gB . B(x)]
//   lp = lp' + Jv^T (dt Lx + dt q (B(x) x Lp)),  Jv = (c/s)(I - p p^T / s^2),
//        s = sqrt(m^2 c^2 + |p|^2)
//   lkx = a Lx,  lkp = a Lp.

#include <cmath>

#include "gather.cuh"
#include "push.cuh"

namespace {

struct FieldBasis {
  int count;
  const double *f[PRT_MAX_FIELD_BASIS][6];
};

struct GradFields {
  double *f[6];
};

constexpr int ADJ_BLOCK = 128;
// resident blocks per SM the stage adjoint is compiled for: the kernel is
// latency-bound, and 6 (80 registers at order 3, a few spilled) measured
// fastest on B200 (0.25 ms per 1M-particle stage against 0.27 at 5 and 0.37
// at 3); order 4 keeps 3 (35 monomials in registers)
#ifndef ADJ_MIN_BLOCKS
#define ADJ_MIN_BLOCKS 6
#endif

// Forward stage writing its output state to separate arrays (the recorded
// tape keeps the input). Same arithmetic as lsrk_stage_kernel.
template <int ORDER>
__global__ void __launch_bounds__(256, ORDER >= 4 ? 2 : 3)
    lsrk_stage_record_kernel(DevMesh M, const Lagrange<ORDER> L, Fields6 F, long long n,
                             const double *__restrict__ x_in, const double *__restrict__ p_in,
                             const uint32_t *__restrict__ el_in, double *__restrict__ x_out,
                             double *__restrict__ p_out, uint32_t *__restrict__ el_out,
                             const double *__restrict__ q, const double *__restrict__ mass,
                             double *__restrict__ kx, double *__restrict__ kp, double a,
                             double b, double dt, double c, DevStatus *st) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned ctr[4] = {0, 0, 0, 0};
  if (i < n) {
    const uint32_t e = el_in[i];
    double xx[3] = {x_in[i], x_in[n + i], x_in[2 * n + i]};
    double pp[3] = {p_in[i], p_in[n + i], p_in[2 * n + i]};
    uint32_t ne = e;
    if (e != PRT_INVALID) {
      int err = 0;
      const uint32_t r = stage_particle<ORDER>(M, L, F, e, xx, pp, q[i], mass[i], kx, kp, n,
                                               i, a, b, dt, c, ctr, &err);
      if (err)
        record_error(st, err, i);
      else
        ne = r;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      x_out[d * n + i] = xx[d];
      p_out[d * n + i] = pp[d];
    }
    el_out[i] = ne;
  }
  flush_counters(st, ctr);
}

// Per-element monomial coefficients of a nodal field:
// f(r) = sum_n F_n l_n(r) = sum_j (sum_n F_n W[n][j]) m_j(r).
template <int ORDER>
__global__ void to_monomial_kernel(const Lagrange<ORDER> L, long long E,
                                   const double *__restrict__ f, double *__restrict__ c) {
  constexpr int NP = Lagrange<ORDER>::NP;
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= E) return;
  double fv[NP];
#pragma unroll
  for (int nd = 0; nd < NP; ++nd) fv[nd] = f[e * NP + nd];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    double s = 0;
#pragma unroll
    for (int nd = 0; nd < NP; ++nd) s = fma(L.w[nd * NP + j], fv[nd], s);
    c[e * NP + j] = s;
  }
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// Adjoint of one stage (see the file comment). One thread per particle; dead
// particles (PRT_INVALID) pass their adjoints through unchanged, as the
// forward stage leaves them untouched. F and FB hold per-element monomial
// coefficients of the fields (to_monomial_kernel): the field and its
// gradient at x are then one pass over the monomials. NODAL: also scatter
// dL/dfield onto the nodes (per-warp shared staging of the Lagrange values
// and gE/gB, summed over runs of lanes in one element, then one atomic per
// run and node).
template <int ORDER, bool NODAL>
__global__ void __launch_bounds__(ADJ_BLOCK, ORDER >= 4 ? 3 : ADJ_MIN_BLOCKS)
    lsrk_stage_adjoint_kernel(DevMesh M, const Lagrange<ORDER> L, Fields6 F, FieldBasis FB,
                              GradFields GF, long long n, const double *__restrict__ x,
                              const double *__restrict__ p, const uint32_t *__restrict__ el,
                              const double *__restrict__ q, const double *__restrict__ mass,
                              double *__restrict__ lx, double *__restrict__ lp,
                              double *__restrict__ lkx, double *__restrict__ lkp, double a,
                              double b, double dt, double c,
                              double *__restrict__ theta_partials) {
  constexpr int NP = Lagrange<ORDER>::NP;
  extern __shared__ double sh_nodal[];  // NODAL: per warp [NP + 6][32] + el[32]
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double tb[PRT_MAX_FIELD_BASIS];
#pragma unroll
  for (int k = 0; k < PRT_MAX_FIELD_BASIS; ++k) tb[k] = 0;
  const uint32_t e = i < n ? el[i] : PRT_INVALID;
  double *wl = nullptr, *wg = nullptr;
  uint32_t *wel = nullptr;
  if (NODAL) {
    double *base = sh_nodal + (size_t)warp * ((NP + 6) * 32 + 16);
    wl = base;
    wg = base + NP * 32;
    wel = (uint32_t *)(base + (NP + 6) * 32);
    wel[lane] = e;
  }
  if (e != PRT_INVALID) {
    const double charge = q[i], m = mass[i];
    double LX[3], LP[3], pp[3], v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      LX[d] = fma(b, lx[d * n + i], lkx[d * n + i]);
      LP[d] = fma(b, lp[d * n + i], lkp[d * n + i]);
      pp[d] = p[d * n + i];
    }
    const double s2 = m * m * c * c + pp[0] * pp[0] + pp[1] * pp[1] + pp[2] * pp[2];
    const double s = sqrt(s2);
    velocity_exact(pp[0], pp[1], pp[2], m, c, v[0], v[1], v[2]);
    double gE[3], gB[3];
    {
      double t[3];
      cross3(LP, v, t);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        gE[d] = dt * charge * LP[d];
        gB[d] = dt * charge * t[d];
      }
    }
    // powers of the reference coordinates
    const double *A = M.inv_maps + 12 * (size_t)e;
    double r0, r1, r2;
    apply_map_exact(A, x[i], x[n + i], x[2 * n + i], r0, r1, r2);
    double pw0[ORDER + 1], pw1[ORDER + 1], pw2[ORDER + 1];
    pw0[0] = pw1[0] = pw2[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= ORDER; ++k) {
      pw0[k] = pw0[k - 1] * r0;
      pw1[k] = pw1[k - 1] * r1;
      pw2[k] = pw2[k - 1] * r2;
    }
    // one pass over the monomials (the fields come as per-element monomial
    // coefficients): B(x), grad of h = gE . E + gB . B, basis projections
    double mono[NP];
    double Bx[3] = {0, 0, 0}, gr[3] = {0, 0, 0};
    const size_t nb = (size_t)e * NP;
    {
      int idx = 0;
#pragma unroll
      for (int cc = 0; cc <= ORDER; ++cc)
#pragma unroll
        for (int bb = 0; bb <= ORDER - cc; ++bb)
#pragma unroll
          for (int aa = 0; aa <= ORDER - bb - cc; ++aa) {
            const double mj = pw0[aa] * pw1[bb] * pw2[cc];
            if (NODAL) mono[idx] = mj;
            double h = 0;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const double ce = F.f[d] ? __ldg(F.f[d] + nb + idx) : 0.0;
              const double cb = F.f[3 + d] ? __ldg(F.f[3 + d] + nb + idx) : 0.0;
              Bx[d] = fma(cb, mj, Bx[d]);
              h = fma(gE[d], ce, h);
              h = fma(gB[d], cb, h);
            }
            if (aa > 0) gr[0] = fma(h, aa * pw0[aa - 1] * pw1[bb] * pw2[cc], gr[0]);
            if (bb > 0) gr[1] = fma(h, bb * pw0[aa] * pw1[bb - 1] * pw2[cc], gr[1]);
            if (cc > 0) gr[2] = fma(h, cc * pw0[aa] * pw1[bb] * pw2[cc - 1], gr[2]);
#pragma unroll
            for (int k = 0; k < PRT_MAX_FIELD_BASIS; ++k) {
              if (k >= FB.count) break;
              double hb = 0;
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                if (FB.f[k][d]) hb = fma(gE[d], __ldg(FB.f[k][d] + nb + idx), hb);
                if (FB.f[k][3 + d]) hb = fma(gB[d], __ldg(FB.f[k][3 + d] + nb + idx), hb);
              }
              tb[k] = fma(hb, mj, tb[k]);
            }
            ++idx;
          }
    }
    if (NODAL) {
      // Lagrange values for the nodal scatter
#pragma unroll
      for (int nd = 0; nd < NP; ++nd) {
        double ln = 0;
#pragma unroll
        for (int j = 0; j < NP; ++j) ln = fma(L.w[nd * NP + j], mono[j], ln);
        wl[nd * 32 + lane] = ln;
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        wg[d * 32 + lane] = gE[d];
        wg[(3 + d) * 32 + lane] = gB[d];
      }
    }
    double w[3];
    {
      double t[3];
      cross3(Bx, LP, t);
#pragma unroll
      for (int d = 0; d < 3; ++d) w[d] = dt * (LX[d] + charge * t[d]);
    }
    const double pw_dot = pp[0] * w[0] + pp[1] * w[1] + pp[2] * w[2];
    const double cs = c / s;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      // r = A[0..8] x + A[9..11]: d r_k / d x_d = A[3k + d]
      const double gx = gr[0] * A[d] + gr[1] * A[3 + d] + gr[2] * A[6 + d];
      lx[d * n + i] += gx;
      lp[d * n + i] += cs * (w[d] - pp[d] * pw_dot / s2);
      lkx[d * n + i] = a * LX[d];
      lkp[d * n + i] = a * LP[d];
    }
  } else if (NODAL) {
#pragma unroll
    for (int k = 0; k < 6; ++k) wg[k * 32 + lane] = 0;
  }
  if (NODAL) {
    __syncwarp();
    // outputs (node, component) split over the lanes; each walks the 32
    // staged lanes in order and flushes one sum per run of equal elements
    for (int o = lane; o < NP * 6; o += 32) {
      const int nd = o / 6, k = o % 6;
      if (!GF.f[k]) continue;
      double acc = 0;
      for (int l = 0; l < 32; ++l) {
        const uint32_t el_l = wel[l];
        if (el_l != PRT_INVALID) acc = fma(wl[nd * 32 + l], wg[k * 32 + l], acc);
        if (l == 31 || wel[l + 1] != el_l) {
          if (el_l != PRT_INVALID && acc != 0)
            atomicAdd(GF.f[k] + (size_t)el_l * NP + nd, acc);
          acc = 0;
        }
      }
    }
  }
  if (FB.count > 0) {
    __shared__ double red[PRT_MAX_FIELD_BASIS][ADJ_BLOCK / 32];
#pragma unroll
    for (int k = 0; k < PRT_MAX_FIELD_BASIS; ++k) {
      double t = tb[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) red[k][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < FB.count) {
      double t = 0;
      for (int w2 = 0; w2 < ADJ_BLOCK / 32; ++w2) t += red[threadIdx.x][w2];
      theta_partials[(size_t)blockIdx.x * FB.count + threadIdx.x] = t;
    }
  }
}

// grad_theta[k] += sum over blocks of the partials, in a fixed order.
__global__ void theta_reduce_kernel(long long blocks, int count,
                                    const double *__restrict__ partials,
                                    double *__restrict__ grad_theta) {
  __shared__ double sh[256];
  for (int k = 0; k < count; ++k) {
    double t = 0;
    for (long long bl = threadIdx.x; bl < blocks; bl += blockDim.x) t += partials[bl * count + k];
    sh[threadIdx.x] = t;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) grad_theta[k] += sh[0];
    __syncthreads();
  }
}

// lp += Jv^T lv, Jv = d v / d p = (c/s)(I - p p^T / s^2).
__global__ void velocities_adjoint_kernel(long long n, const double *__restrict__ p,
                                          const double *__restrict__ m, double c,
                                          const double *__restrict__ lv,
                                          double *__restrict__ lp) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double p0 = p[i], p1 = p[n + i], p2 = p[2 * n + i], mm = m[i];
  const double s2 = mm * mm * c * c + p0 * p0 + p1 * p1 + p2 * p2;
  const double cs = c / sqrt(s2);
  const double w0 = lv[i], w1 = lv[n + i], w2 = lv[2 * n + i];
  const double pw = (p0 * w0 + p1 * w1 + p2 * w2) / s2;
  lp[i] += cs * (w0 - p0 * pw);
  lp[n + i] += cs * (w1 - p1 * pw);
  lp[2 * n + i] += cs * (w2 - p2 * pw);
}

// Adjoint of the expansion from positions to nodes: every position sums the
// node adjoints of its nodes (ascending node order): G[0] from dL/drho,
// G[1..3] from dL/dj.
__global__ void contract_kernel(long long npos, long long nn,
                                const uint32_t *__restrict__ run_starts,
                                const uint32_t *__restrict__ run_nodes,
                                const double *__restrict__ grho, const double *__restrict__ gj,
                                double *__restrict__ G) {
  const long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (u >= npos) return;
  double s[4] = {0, 0, 0, 0};
  for (uint32_t k = run_starts[u]; k < run_starts[u + 1]; ++k) {
    const uint32_t node = run_nodes[k];
    if (grho) s[0] += grho[node];
    if (gj) {
      s[1] += gj[node];
      s[2] += gj[nn + node];
      s[3] += gj[2 * nn + node];
    }
  }
#pragma unroll
  for (int d = 0; d < 4; ++d) G[d * npos + u] = s[d];
}

constexpr int DEP_ADJ_BLOCK = 128;

// Adjoint of the plain shape deposition. With weight w = q N and
// S = (a - r^2/a)^alpha:
//   dL/dx_p = w sum_u (G0_u + G_u . v_p) dS/dx_p,
//   dL/dv_p = w sum_u G_u S,   dS/dx_p = alpha (a - r^2/a)^(alpha-1) (2/a) (x_u - x_p),
// gathered per particle (lane) over the positions within the radius
// (warp_gather_positions, gather.cuh).
template <bool ALPHA2>
__global__ void __launch_bounds__(DEP_ADJ_BLOCK, 4)
    deposit_adjoint_kernel(DevMesh M, CentreBinsDev CB, const double *__restrict__ pos,
                           long long npos, prt_dep::ShapeParams S, double normalizer,
                           const double *__restrict__ G, long long n,
                           const double *__restrict__ x, const double *__restrict__ q,
                           const double *__restrict__ v, const uint32_t *__restrict__ el,
                           double *__restrict__ lx, double *__restrict__ lv) {
  __shared__ GatherStage<4> stage[DEP_ADJ_BLOCK / 32];
  const int warp = threadIdx.x >> 5;
  const long long i = blockIdx.x * (long long)DEP_ADJ_BLOCK + threadIdx.x;
  const bool live = i < n && (!el || el[i] != PRT_INVALID);
  double p[3] = {0, 0, 0}, vv[3] = {0, 0, 0};
  if (live) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      p[d] = x[d * n + i];
      if (v) vv[d] = v[d * n + i];
    }
  }
  double ax0 = 0, ax1 = 0, ax2 = 0, as1 = 0, as2 = 0, as3 = 0;
  warp_gather_positions<4>(
      M, CB, pos, npos, G, S.radius, live, p, stage[warp],
      [&](double f0, double f1, double f2, double r2, const double *g) {
        const double rt = fmax(fma(-r2, S.inv_radius, S.radius), 0.0);
        double sv, ds;
        if (ALPHA2) {
          sv = rt * rt;
          ds = rt * (4.0 * S.inv_radius);
        } else {
          const double pm = rt > 0 ? pow(rt, S.alpha - 1.0) : 0.0;
          sv = pm * rt;
          ds = S.alpha * pm * (2.0 * S.inv_radius);
        }
        const double h = fma(g[2], vv[1], fma(g[1], vv[0], fma(g[3], vv[2], g[0])));
        const double hd = h * ds;
        ax0 = fma(hd, f0, ax0);
        ax1 = fma(hd, f1, ax1);
        ax2 = fma(hd, f2, ax2);
        as1 = fma(g[1], sv, as1);
        as2 = fma(g[2], sv, as2);
        as3 = fma(g[3], sv, as3);
      });
  if (live) {
    const double w = q[i] * normalizer;
    lx[i] += w * ax0;
    lx[n + i] += w * ax1;
    lx[2 * n + i] += w * ax2;
    if (lv) {
      lv[i] += w * as1;
      lv[n + i] += w * as2;
      lv[2 * n + i] += w * as3;
    }
  }
}

template <int ORDER>
int launch_record(const prt_pusher *P, prt_workspace *ws, long long n, const double *x_in,
                  const double *p_in, const uint32_t *el_in, double *x_out, double *p_out,
                  uint32_t *el_out, const double *q, const double *m, double *kx, double *kp,
                  Fields6 F, double a, double b, double dt, double c, cudaStream_t s) {
  ScopedTimer timer(ws, PRT_TIME_LSRK_STAGE, s);
  lsrk_stage_record_kernel<ORDER><<<prt_grid_blocks(n, 256), 256, 0, s>>>(
      P->mesh->dev, make_lagrange<ORDER>(P), F, n, x_in, p_in, el_in, x_out, p_out, el_out, q,
      m, kx, kp, a, b, dt, c, ws->status);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

template <int ORDER, bool NODAL>
int launch_adjoint(const prt_pusher *P, prt_workspace *ws, long long n, const double *x,
                   const double *p, const uint32_t *el, const double *q, const double *m,
                   double *lx, double *lp, double *lkx, double *lkp, Fields6 F,
                   const FieldBasis &FB, const GradFields &GF, double a, double b, double dt,
                   double c, double *grad_theta, cudaStream_t s) {
  constexpr int NP = Lagrange<ORDER>::NP;
  const long long blocks = prt_grid_blocks(n, ADJ_BLOCK);
  double *partials = nullptr;
  int rc = PRT_OK;
  if (FB.count > 0) {
    partials = (double *)ws_buffer(ws, PRT_WS_ADJ_PARTIALS,
                                   sizeof(double) * (size_t)blocks * FB.count, &rc);
    if (!partials) return rc;
  }
  const size_t shmem = NODAL ? sizeof(double) * (ADJ_BLOCK / 32) * ((NP + 6) * 32 + 16) : 0;
  auto kern = lsrk_stage_adjoint_kernel<ORDER, NODAL>;
  if (shmem > 48 * 1024)
    PRT_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)shmem));
  {
    ScopedTimer timer(ws, PRT_TIME_STAGE_ADJOINT, s);
    kern<<<blocks, ADJ_BLOCK, shmem, s>>>(P->mesh->dev, make_lagrange<ORDER>(P), F, FB, GF, n,
                                          x, p, el, q, m, lx, lp, lkx, lkp, a, b, dt, c,
                                          partials);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  if (FB.count > 0) {
    theta_reduce_kernel<<<1, 256, 0, s>>>(blocks, FB.count, partials, grad_theta);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  return PRT_OK;
}

template <int ORDER>
int dispatch_adjoint(bool nodal, const prt_pusher *P, prt_workspace *ws, long long n,
                     const double *x, const double *p, const uint32_t *el, const double *q,
                     const double *m, double *lx, double *lp, double *lkx, double *lkp,
                     Fields6 F, const FieldBasis &FB, const GradFields &GF, double a, double b,
                     double dt, double c, double *grad_theta, cudaStream_t s) {
  if (nodal)
    return launch_adjoint<ORDER, true>(P, ws, n, x, p, el, q, m, lx, lp, lkx, lkp, F, FB, GF,
                                       a, b, dt, c, grad_theta, s);
  return launch_adjoint<ORDER, false>(P, ws, n, x, p, el, q, m, lx, lp, lkx, lkp, F, FB, GF, a,
                                      b, dt, c, grad_theta, s);
}

}  // namespace

extern "C" int prt_lsrk_stage_record(const prt_pusher *P, prt_workspace *ws, int64_t n,
                                     const double *x_in, const double *p_in,
                                     const uint32_t *el_in, double *x_out, double *p_out,
                                     uint32_t *el_out, const double *q, const double *m,
                                     double *kx, double *kp, const double *const fields[6],
                                     double a, double b, double dt, double c, void *stream) {
  if (!P || !ws || n < 0 || !fields) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  if (!x_in || !p_in || !el_in || !x_out || !p_out || !el_out || !q || !m || !kx || !kp)
    return PRT_ERR_INVALID_ARGUMENT;
  if (x_in == x_out || p_in == p_out || el_in == el_out) return PRT_ERR_INVALID_ARGUMENT;
  Fields6 F;
  for (int k = 0; k < 6; ++k) F.f[k] = fields[k];
  cudaStream_t s = (cudaStream_t)stream;
  switch (P->order) {
    case 1: return launch_record<1>(P, ws, n, x_in, p_in, el_in, x_out, p_out, el_out, q, m, kx, kp, F, a, b, dt, c, s);
    case 2: return launch_record<2>(P, ws, n, x_in, p_in, el_in, x_out, p_out, el_out, q, m, kx, kp, F, a, b, dt, c, s);
    case 3: return launch_record<3>(P, ws, n, x_in, p_in, el_in, x_out, p_out, el_out, q, m, kx, kp, F, a, b, dt, c, s);
    case 4: return launch_record<4>(P, ws, n, x_in, p_in, el_in, x_out, p_out, el_out, q, m, kx, kp, F, a, b, dt, c, s);
  }
  return PRT_ERR_INVALID_ARGUMENT;
}

extern "C" int prt_lsrk_stage_adjoint(const prt_pusher *P, prt_workspace *ws, int64_t n,
                                      const double *x, const double *p, const uint32_t *el,
                                      const double *q, const double *m, double *lam_x,
                                      double *lam_p, double *lam_kx, double *lam_kp,
                                      const double *const field_coefficients[6], double a,
                                      double b, double dt, double c,
                                      double *const grad_fields[6], int32_t nbasis,
                                      const double *const *basis, double *grad_theta,
                                      void *stream) {
  if (!P || !ws || n < 0 || !field_coefficients) return PRT_ERR_INVALID_ARGUMENT;
  if (nbasis < 0 || nbasis > PRT_MAX_FIELD_BASIS || (nbasis > 0 && (!basis || !grad_theta)))
    return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  if (!x || !p || !el || !q || !m || !lam_x || !lam_p || !lam_kx || !lam_kp)
    return PRT_ERR_INVALID_ARGUMENT;
  Fields6 F;
  for (int k = 0; k < 6; ++k) F.f[k] = field_coefficients[k];
  FieldBasis FB;
  FB.count = nbasis;
  for (int k = 0; k < PRT_MAX_FIELD_BASIS; ++k)
    for (int d = 0; d < 6; ++d) FB.f[k][d] = k < nbasis ? basis[6 * k + d] : nullptr;
  GradFields GF;
  bool nodal = false;
  for (int d = 0; d < 6; ++d) {
    GF.f[d] = grad_fields ? grad_fields[d] : nullptr;
    nodal = nodal || GF.f[d];
  }
  cudaStream_t s = (cudaStream_t)stream;
  switch (P->order) {
    case 1: return dispatch_adjoint<1>(nodal, P, ws, n, x, p, el, q, m, lam_x, lam_p, lam_kx, lam_kp, F, FB, GF, a, b, dt, c, grad_theta, s);
    case 2: return dispatch_adjoint<2>(nodal, P, ws, n, x, p, el, q, m, lam_x, lam_p, lam_kx, lam_kp, F, FB, GF, a, b, dt, c, grad_theta, s);
    case 3: return dispatch_adjoint<3>(nodal, P, ws, n, x, p, el, q, m, lam_x, lam_p, lam_kx, lam_kp, F, FB, GF, a, b, dt, c, grad_theta, s);
    case 4: return dispatch_adjoint<4>(nodal, P, ws, n, x, p, el, q, m, lam_x, lam_p, lam_kx, lam_kp, F, FB, GF, a, b, dt, c, grad_theta, s);
  }
  return PRT_ERR_INVALID_ARGUMENT;
}

template <int ORDER>
static int launch_to_monomial(const prt_pusher *P, int32_t count, const double *const *fields,
                              double *const *coefficients, cudaStream_t s) {
  const long long E = P->mesh->dev.E;
  const Lagrange<ORDER> L = make_lagrange<ORDER>(P);
  for (int k = 0; k < count; ++k) {
    if (!fields[k] || !coefficients[k]) continue;
    to_monomial_kernel<ORDER><<<prt_grid_blocks(E, 128), 128, 0, s>>>(L, E, fields[k],
                                                                    coefficients[k]);
    PRT_CHECK_CUDA(cudaGetLastError());
  }
  return PRT_OK;
}

extern "C" int prt_fields_to_monomial(const prt_pusher *P, int32_t count,
                                      const double *const *fields, double *const *coefficients,
                                      void *stream) {
  if (!P || count < 0 || (count > 0 && (!fields || !coefficients)))
    return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  switch (P->order) {
    case 1: return launch_to_monomial<1>(P, count, fields, coefficients, s);
    case 2: return launch_to_monomial<2>(P, count, fields, coefficients, s);
    case 3: return launch_to_monomial<3>(P, count, fields, coefficients, s);
    case 4: return launch_to_monomial<4>(P, count, fields, coefficients, s);
  }
  return PRT_ERR_INVALID_ARGUMENT;
}

extern "C" int prt_velocities_adjoint(int64_t n, const double *p, const double *m, double c,
                                      const double *lam_v, double *lam_p, void *stream) {
  if (n < 0) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  if (!p || !m || !lam_v || !lam_p) return PRT_ERR_INVALID_ARGUMENT;
  velocities_adjoint_kernel<<<prt_grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(
      n, p, m, c, lam_v, lam_p);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

extern "C" int prt_deposit_shape_adjoint(const prt_mesh *mesh, prt_workspace *ws,
                                         prt_shape_function shape, int64_t n, const double *x,
                                         const double *q, const double *v, const uint32_t *el,
                                         const double *grad_rho, const double *grad_j,
                                         double *lam_x, double *lam_v, void *stream) {
  if (!mesh || !ws || n < 0 || n >= (1ll << 31) || !(shape.radius > 0))
    return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0 || (!grad_rho && !grad_j)) return PRT_OK;
  if (!x || !q || !lam_x || (grad_j && !v)) return PRT_ERR_INVALID_ARGUMENT;
  const PositionSet &PS = mesh->positions;
  const long long nn = mesh->dev.E * (long long)mesh->dev.Np;
  cudaStream_t s = (cudaStream_t)stream;
  ScopedTimer timer(ws, PRT_TIME_DEPOSIT_ADJOINT, s);
  int rc;
  double *G = (double *)ws_buffer(ws, PRT_WS_ADJ_POSITIONS, sizeof(double) * 4 * PS.count, &rc);
  if (!G) return rc;
  contract_kernel<<<prt_grid_blocks(PS.count, 256), 256, 0, s>>>(
      PS.count, nn, PS.run_starts, PS.run_nodes, grad_rho, grad_j, G);
  PRT_CHECK_CUDA(cudaGetLastError());
  prt_dep::ShapeParams S;
  S.radius = shape.radius;
  S.radius2 = shape.radius * shape.radius;
  S.inv_radius = 1.0 / shape.radius;
  S.alpha = shape.alpha;
  for (int d = 0; d < 3; ++d) S.reach[d] = shape.radius;
  const CentreBinsDev CB = centre_bins_dev(PS);
  const double *vv = grad_j ? v : nullptr;
  double *lvv = grad_j ? lam_v : nullptr;
  const unsigned blocks = (unsigned)((n + DEP_ADJ_BLOCK - 1) / DEP_ADJ_BLOCK);
  if (shape.alpha == 2)
    deposit_adjoint_kernel<true><<<blocks, DEP_ADJ_BLOCK, 0, s>>>(
        mesh->dev, CB, PS.pos, PS.count, S, shape.normalizer, G, n, x, q, vv, el, lam_x, lvv);
  else
    deposit_adjoint_kernel<false><<<blocks, DEP_ADJ_BLOCK, 0, s>>>(
        mesh->dev, CB, PS.pos, PS.count, S, shape.normalizer, G, n, x, q, vv, el, lam_x, lvv);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}
