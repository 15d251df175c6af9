// push.cuh -- per-particle arithmetic of the monomial pusher, shared by the
// forward stage kernels and their adjoints: relativistic velocity, Lagrange
// interpolation of nodal fields, Lorentz force and the fused low-storage RK
// stage update.
#pragma once

#include "common.cuh"
#include "handles.cuh"

// get_velocities arithmetic (particle_state.hpp:98-125), rounded as written.
__device__ __forceinline__ void velocity_exact(double p0, double p1, double p2, double m,
                                               double c, double &v0, double &v1,
                                               double &v2) {
  double pa = __dmul_rn(p0, p0);
  pa = __dadd_rn(pa, __dmul_rn(p1, p1));
  pa = __dadd_rn(pa, __dmul_rn(p2, p2));
  pa = __dsqrt_rn(pa);
  if (pa == 0) {
    v0 = v1 = v2 = 0;
    return;
  }
  double den = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(m, m), c), c), __dmul_rn(pa, pa));
  double vv = __ddiv_rn(__dmul_rn(c, pa), __dsqrt_rn(den));
  double s = __ddiv_rn(vv, pa);
  v0 = __dmul_rn(s, p0);
  v1 = __dmul_rn(s, p1);
  v2 = __dmul_rn(s, p2);
}

template <int ORDER>
struct Lagrange {
  static constexpr int NP = (ORDER + 1) * (ORDER + 2) * (ORDER + 3) / 6;
  // w[i*NP + j]: Lagrange value i = sum_j w[i][j] * monomial_j (canonical
  // monomial order: exponents (a, b, c), a fastest, a + b + c <= ORDER).
  double w[NP * NP];
};

struct Fields6 {
  const double *f[6];
};

// Interpolates the six field components at x inside element e: Lagrange
// values c = V^{-T} m(r) (push_monomial.hpp:155-210), then <c, F_k[e]>
// (push_monomial.hpp:99-111).
template <int ORDER>
__device__ __forceinline__ void interpolate_fields(const DevMesh &M,
                                                   const Lagrange<ORDER> &L,
                                                   const Fields6 &F, uint32_t e,
                                                   double x0, double x1, double x2,
                                                   double ef[6]) {
  constexpr int NP = Lagrange<ORDER>::NP;
  double r0, r1, r2;
  apply_map_exact(M.inv_maps + 12 * (size_t)e, x0, x1, x2, r0, r1, r2);
  double pw0[ORDER + 1], pw1[ORDER + 1], pw2[ORDER + 1];
  pw0[0] = pw1[0] = pw2[0] = 1.0;
#pragma unroll
  for (int k = 1; k <= ORDER; ++k) {
    pw0[k] = pw0[k - 1] * r0;
    pw1[k] = pw1[k - 1] * r1;
    pw2[k] = pw2[k - 1] * r2;
  }
  double mono[NP];
  {
    int idx = 0;
#pragma unroll
    for (int c = 0; c <= ORDER; ++c)
#pragma unroll
      for (int b = 0; b <= ORDER - c; ++b)
#pragma unroll
        for (int a = 0; a <= ORDER - b - c; ++a) mono[idx++] = pw0[a] * pw1[b] * pw2[c];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) ef[k] = 0;
  const size_t base = (size_t)e * NP;
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    double ci = 0;
#pragma unroll
    for (int j = 0; j < NP; ++j) ci = fma(L.w[i * NP + j], mono[j], ci);
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (F.f[k]) ef[k] = fma(ci, __ldg(F.f[k] + base + i), ef[k]);
  }
}

template <int ORDER>
static Lagrange<ORDER> make_lagrange(const prt_pusher *P) {
  Lagrange<ORDER> L;
  for (int i = 0; i < Lagrange<ORDER>::NP * Lagrange<ORDER>::NP; ++i) L.w[i] = P->w[i];
  return L;
}

// RK update and relocation from a force f at (x, p): k = a k + dt (v(p), f),
// (x, p) += b k (residuals kx, kp [3][n] at index i, read and written before
// the relocation), then the new containing element (PRT_INVALID if the
// particle left the mesh; *err on a locate error).
__device__ __forceinline__ uint32_t update_particle(const DevMesh &M, uint32_t e,
                                                    const double f[3], const double v[3],
                                                    double xx[3], double pp[3],
                                                    double *__restrict__ kx,
                                                    double *__restrict__ kp, long long n,
                                                    long long i, double a, double b,
                                                    double dt, unsigned ctr[4], int *err) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double kxd = __dadd_rn(__dmul_rn(a, kx[d * n + i]), __dmul_rn(dt, v[d]));
    const double kpd = __dadd_rn(__dmul_rn(a, kp[d * n + i]), __dmul_rn(dt, f[d]));
    kx[d * n + i] = kxd;
    kp[d * n + i] = kpd;
    xx[d] = __dadd_rn(xx[d], __dmul_rn(b, kxd));
    pp[d] = __dadd_rn(pp[d], __dmul_rn(b, kpd));
  }
  bool wrapped;
  return relocate(M, xx[0], xx[1], xx[2], pp[0], pp[1], pp[2], e, ctr, err, &wrapped);
}

// Lorentz force F = q E + v x (q B) in the reference's operation order
// (push_monomial.hpp:219-325).
__device__ __forceinline__ void lorentz_force(double charge, const double ef[6],
                                              const double v[3], double f[3]) {
  double elf[3], qb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    elf[d] = __dmul_rn(charge, ef[d]);
    qb[d] = __dmul_rn(charge, ef[3 + d]);
  }
  f[0] = __dadd_rn(elf[0], __dsub_rn(__dmul_rn(v[1], qb[2]), __dmul_rn(v[2], qb[1])));
  f[1] = __dadd_rn(elf[1], __dsub_rn(__dmul_rn(v[2], qb[0]), __dmul_rn(v[0], qb[2])));
  f[2] = __dadd_rn(elf[2], __dsub_rn(__dmul_rn(v[0], qb[1]), __dmul_rn(v[1], qb[0])));
}

// The stage after the interpolation: Lorentz force from the fields ef at x,
// RK update, relocation (shared by the FP64 stage and the mixed-precision
// stage, whose fields come from the tensor cores).
__device__ __forceinline__ uint32_t stage_from_fields(const DevMesh &M, uint32_t e,
                                                      const double ef[6], double xx[3],
                                                      double pp[3], double charge, double mass,
                                                      double *__restrict__ kx,
                                                      double *__restrict__ kp, long long n,
                                                      long long i, double a, double b,
                                                      double dt, double c, unsigned ctr[4],
                                                      int *err) {
  double v[3], f[3];
  velocity_exact(pp[0], pp[1], pp[2], mass, c, v[0], v[1], v[2]);
  lorentz_force(charge, ef, v, f);
  return update_particle(M, e, f, v, xx, pp, kx, kp, n, i, a, b, dt, ctr, err);
}

// One low-storage RK stage for one live particle in element e:
//   v = v(p), F = q E(x) + v x (q B(x)), k = a k + dt (v, F), (x, p) += b k,
// then relocation. Updates xx, pp in place and the residuals kx, kp [3][n]
// at index i (read and written before the relocation, which keeps them out
// of its live registers). Returns the new element (PRT_INVALID if the
// particle left the mesh); *err is set on a locate error.
template <int ORDER>
__device__ __forceinline__ uint32_t stage_particle(const DevMesh &M, const Lagrange<ORDER> &L,
                                                   const Fields6 &F, uint32_t e, double xx[3],
                                                   double pp[3], double charge, double mass,
                                                   double *__restrict__ kx,
                                                   double *__restrict__ kp, long long n,
                                                   long long i, double a,
                                                   double b, double dt, double c,
                                                   unsigned ctr[4], int *err) {
  double ef[6];
  interpolate_fields<ORDER>(M, L, F, e, xx[0], xx[1], xx[2], ef);
  return stage_from_fields(M, e, ef, xx, pp, charge, mass, kx, kp, n, i, a, b, dt, c, ctr,
                           err);
}
