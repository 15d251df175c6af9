// diagnostics.cu -- beam diagnostics as one fused reduction over the device
// particle store.
//
// The reference computes each quantity in its own serial loop over the
// particles (diagnostics.hpp:38-180) for the log quantities of
// pyrticle/log.py:107-325: particle momentum, kinetic energies, total charge,
// RMS beam size and emittance, RMS energy spread, particle current. Here one
// pass reads every live particle once and accumulates all the sums those
// quantities are built from (prt_beam_moments); the host finishes each
// quantity with the reference's formula. The block sums and the final sum
// run in a fixed order: the result is deterministic for a given launch.

#include <cmath>

#include "push.cuh"

namespace {

constexpr int DG_BLOCK = 256;
constexpr int DG_GRID = 592;  // 4 blocks per SM of a 148-SM B200 (grid-stride)

// kinetic energy (gamma - 1) m c^2 = p^2 c^2 / (E + m c^2), E = c sqrt(m^2 c^2 + p^2):
// the reference's (p/v - m) c^2 (diagnostics.hpp:43-57) in a form without
// the 0/0 of a particle at rest
__device__ __forceinline__ double kinetic_energy(double p0, double p1, double p2, double m,
                                                 double c) {
  const double p2sum = p0 * p0 + p1 * p1 + p2 * p2;
  const double e = c * sqrt(m * m * c * c + p2sum);
  return p2sum * c * c / (e + m * c * c);
}

__global__ void kinetic_energies_kernel(long long n, const double *__restrict__ p,
                                        const double *__restrict__ m,
                                        const uint32_t *__restrict__ el, double c,
                                        double *__restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = (el && el[i] == PRT_INVALID)
               ? 0.0
               : kinetic_energy(p[i], p[n + i], p[2 * n + i], m[i], c);
}

__global__ void __launch_bounds__(DG_BLOCK)
    beam_moments_kernel(long long n, const double *__restrict__ x, const double *__restrict__ p,
                        const double *__restrict__ q, const double *__restrict__ m,
                        const uint32_t *__restrict__ el, double c, int beam_axis,
                        double ke_shift, double *__restrict__ partials) {
  double acc[PRT_BEAM_MOMENTS];
#pragma unroll
  for (int k = 0; k < PRT_BEAM_MOMENTS; ++k) acc[k] = 0;
  for (long long i = blockIdx.x * (long long)DG_BLOCK + threadIdx.x; i < n;
       i += (long long)gridDim.x * DG_BLOCK) {
    if (el && el[i] == PRT_INVALID) continue;
    const double xx[3] = {x[i], x[n + i], x[2 * n + i]};
    const double pp[3] = {p[i], p[n + i], p[2 * n + i]};
    const double qq = q[i], mm = m[i];
    const double ke = kinetic_energy(pp[0], pp[1], pp[2], mm, c);
    double v[3];
    velocity_exact(pp[0], pp[1], pp[2], mm, c, v[0], v[1], v[2]);
    const double pb = pp[beam_axis];
    acc[PRT_BM_COUNT] += 1;
    acc[PRT_BM_CHARGE] += qq;
    acc[PRT_BM_KE] += ke;
    acc[PRT_BM_KE2] += (ke - ke_shift) * (ke - ke_shift);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double xp = pb != 0 ? pp[d] / pb : 0.0;  // x' = p_d / p_beam
      acc[PRT_BM_P + d] += pp[d];
      acc[PRT_BM_X + d] += xx[d];
      acc[PRT_BM_X2 + d] += xx[d] * xx[d];
      acc[PRT_BM_XP + d] += xp;
      acc[PRT_BM_XP2 + d] += xp * xp;
      acc[PRT_BM_XXP + d] += xx[d] * xp;
      acc[PRT_BM_QV + d] += qq * v[d];
    }
  }
  __shared__ double sh[DG_BLOCK];
  for (int k = 0; k < PRT_BEAM_MOMENTS; ++k) {
    sh[threadIdx.x] = acc[k];
    __syncthreads();
    for (int o = DG_BLOCK / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) partials[(size_t)blockIdx.x * PRT_BEAM_MOMENTS + k] = sh[0];
    __syncthreads();
  }
}

// the block sums in block order (one thread per moment)
__global__ void beam_moments_final_kernel(int blocks, const double *__restrict__ partials,
                                          double *__restrict__ out) {
  const int k = threadIdx.x;
  if (k >= PRT_BEAM_MOMENTS) return;
  double s = 0;
  for (int b = 0; b < blocks; ++b) s += partials[(size_t)b * PRT_BEAM_MOMENTS + k];
  out[k] = s;
}

}  // namespace

extern "C" int prt_kinetic_energies(int64_t n, const double *momenta, const double *masses,
                                    const uint32_t *elements, double vacuum_c, double *out,
                                    void *stream) {
  if (n < 0) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  if (!momenta || !masses || !out) return PRT_ERR_INVALID_ARGUMENT;
  kinetic_energies_kernel<<<prt_grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(
      n, momenta, masses, elements, vacuum_c, out);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

extern "C" int prt_beam_moments(prt_workspace *ws, int64_t n, const double *positions,
                                const double *momenta, const double *charges,
                                const double *masses, const uint32_t *elements,
                                double vacuum_c, int32_t beam_axis, double ke_shift,
                                double out[PRT_BEAM_MOMENTS], void *stream) {
  if (!ws || n < 0 || !out || beam_axis < 0 || beam_axis > 2) return PRT_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < PRT_BEAM_MOMENTS; ++k) out[k] = 0;
  if (n == 0) return PRT_OK;
  if (!positions || !momenta || !charges || !masses) return PRT_ERR_INVALID_ARGUMENT;
  int rc;
  double *buf = (double *)ws_buffer(ws, PRT_WS_DIAGNOSTICS,
                                    sizeof(double) * PRT_BEAM_MOMENTS * (DG_GRID + 1), &rc);
  if (!buf) return rc;
  const long long need = (n + DG_BLOCK - 1) / DG_BLOCK;
  const int blocks = (int)(need < DG_GRID ? need : DG_GRID);
  cudaStream_t s = (cudaStream_t)stream;
  beam_moments_kernel<<<blocks, DG_BLOCK, 0, s>>>(n, positions, momenta, charges, masses,
                                                   elements, vacuum_c, beam_axis, ke_shift,
                                                   buf + PRT_BEAM_MOMENTS);
  PRT_CHECK_CUDA(cudaGetLastError());
  beam_moments_final_kernel<<<1, 32, 0, s>>>(blocks, buf + PRT_BEAM_MOMENTS, buf);
  PRT_CHECK_CUDA(cudaGetLastError());
  PRT_CHECK_CUDA(cudaMemcpyAsync(out, buf, sizeof(double) * PRT_BEAM_MOMENTS,
                                 cudaMemcpyDeviceToHost, s));
  PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  return PRT_OK;
}
