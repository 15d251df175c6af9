// common.cuh -- device-side mesh view, status word and exact-arithmetic
// helpers shared by the libprt kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/prt.h"

#define PRT_INVALID PRT_INVALID_ELEMENT

// Launch-status check: returns PRT_ERR_CUDA from the enclosing C-ABI call.
#define PRT_CHECK_CUDA(expr)                         \
  do {                                               \
    cudaError_t prt_e_ = (expr);                     \
    if (prt_e_ != cudaSuccess) {                     \
      prt_note_cuda_error(prt_e_, #expr, __LINE__);  \
      return PRT_ERR_CUDA;                           \
    }                                                \
  } while (0)

void prt_note_cuda_error(cudaError_t e, const char *what, int line);

// Device-resident status word of a workspace: first error (code, particle),
// first warning, and the four find-path counters.
struct DevStatus {
  int error;
  int warning;
  long long error_index;
  long long warning_index;
  unsigned long long counters[4];  // same, neighbor, vertex, global
};

enum { CTR_SAME = 0, CTR_NEIGHBOR = 1, CTR_VERTEX = 2, CTR_GLOBAL = 3 };

// Device copy of mesh_data (meshdata.hpp:53-124), passed to kernels by value.
struct DevMesh {
  long long E, V;
  int Np;
  const double *__restrict__ inv_maps;     // [E][12]
  const double *__restrict__ jacobians;    // [E]
  const double *__restrict__ normals;      // [E][4][3]
  const double *__restrict__ plane_rhs;    // [E][4]
  const uint32_t *__restrict__ neighbors;  // [E][4]
  const uint32_t *__restrict__ axes;       // [E][4]
  const uint32_t *__restrict__ el_verts;   // [E][4]
  const double *__restrict__ verts;        // [V][3]
  const uint32_t *__restrict__ vadj_starts;
  const uint32_t *__restrict__ vadj;
  double pmin[3], pmax[3];
  const double *__restrict__ nodes;        // [E*Np][3]
  double bin_origin[3], bin_inv[3];
  int bin_dims[3];
  const uint32_t *__restrict__ bin_starts;
  const uint32_t *__restrict__ bin_elements;
};

// Records the first device error (lowest particle index wins among equal
// codes raised in one launch) without trapping.
__device__ __forceinline__ void record_error(DevStatus *st, int code, long long idx) {
  if (atomicCAS(&st->error, 0, code) == 0) {
    atomicExch((unsigned long long *)&st->error_index, (unsigned long long)idx);
  } else if (st->error == code) {
    atomicMin(&st->error_index, idx);
  }
}

__device__ __forceinline__ void record_warning(DevStatus *st, int code, long long idx) {
  if (atomicCAS(&st->warning, 0, code) == 0) {
    atomicExch((unsigned long long *)&st->warning_index, (unsigned long long)idx);
  } else if (st->warning == code) {
    atomicMin(&st->warning_index, idx);
  }
}

// ---- exact restatements (round-to-nearest, no contraction) ---------------

// hedge affine_map::operator(): y_i = ((A_i0 x0 + A_i1 x1) + A_i2 x2) + b_i
__device__ __forceinline__ void apply_map_exact(const double *__restrict__ m, double x0,
                                                double x1, double x2, double &y0,
                                                double &y1, double &y2) {
  double t;
  t = __dmul_rn(m[0], x0);
  t = __dadd_rn(t, __dmul_rn(m[1], x1));
  t = __dadd_rn(t, __dmul_rn(m[2], x2));
  y0 = __dadd_rn(t, m[9]);
  t = __dmul_rn(m[3], x0);
  t = __dadd_rn(t, __dmul_rn(m[4], x1));
  t = __dadd_rn(t, __dmul_rn(m[5], x2));
  y1 = __dadd_rn(t, m[10]);
  t = __dmul_rn(m[6], x0);
  t = __dadd_rn(t, __dmul_rn(m[7], x1));
  t = __dadd_rn(t, __dmul_rn(m[8], x2));
  y2 = __dadd_rn(t, m[11]);
}

// is_in_unit_simplex (meshdata.hpp:38-48), tolerance 1e-10.
__device__ __forceinline__ bool in_unit_simplex(double r0, double r1, double r2) {
  const double lo = -1.0 - 1e-10;
  if (r0 < lo) return false;
  if (r1 < lo) return false;
  if (r2 < lo) return false;
  double s = __dadd_rn(__dadd_rn(r0, r1), r2);
  return s <= -1.0 + 1e-10;
}

__device__ __forceinline__ bool in_element(const DevMesh &M, uint32_t e, double x0,
                                           double x1, double x2) {
  double r0, r1, r2;
  apply_map_exact(M.inv_maps + 12 * (size_t)e, x0, x1, x2, r0, r1, r2);
  return in_unit_simplex(r0, r1, r2);
}

__device__ __forceinline__ double inner3_exact(const double *__restrict__ a, double b0,
                                               double b1, double b2) {
  double t = __dmul_rn(a[0], b0);
  t = __dadd_rn(t, __dmul_rn(a[1], b1));
  return __dadd_rn(t, __dmul_rn(a[2], b2));
}

__device__ __forceinline__ double dist_exact(const double *__restrict__ a, double b0,
                                             double b1, double b2) {
  double d0 = __dsub_rn(a[0], b0), d1 = __dsub_rn(a[1], b1), d2 = __dsub_rn(a[2], b2);
  double t = __dmul_rn(d0, d0);
  t = __dadd_rn(t, __dmul_rn(d1, d1));
  t = __dadd_rn(t, __dmul_rn(d2, d2));
  return __dsqrt_rn(t);
}

// Global search (meshdata.hpp:208-215) through the element bins: the lowest
// id among the bin's elements that contain the point.
__device__ __forceinline__ uint32_t find_global(const DevMesh &M, double x0, double x1,
                                                double x2) {
  const double xs[3] = {x0, x1, x2};
  int b[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double u = (xs[d] - M.bin_origin[d]) * M.bin_inv[d];
    int bi;
    if (!(u >= 0.0))
      bi = 0;
    else if (u >= (double)M.bin_dims[d])
      bi = M.bin_dims[d] - 1;
    else
      bi = min((int)u, M.bin_dims[d] - 1);
    b[d] = bi;
  }
  size_t bid = b[0] + (size_t)M.bin_dims[0] * (b[1] + (size_t)M.bin_dims[1] * b[2]);
  const uint32_t s = M.bin_starts[bid], t = M.bin_starts[bid + 1];
  for (uint32_t i = s; i < t; ++i) {
    uint32_t e = M.bin_elements[i];
    if (in_element(M, e, x0, x1, x2)) return e;
  }
  return PRT_INVALID;
}

// find_new_containing_element (particle_state.hpp:130-261), same decision
// sequence and arithmetic. ctr[] counts locally; *err receives
// PRT_ERR_NO_BEST_NORMAL when no face normal has a positive product with p.
__device__ __forceinline__ uint32_t find_new_containing(const DevMesh &M, double x0,
                                                        double x1, double x2,
                                                        double p0, double p1,
                                                        double p2, uint32_t prev,
                                                        unsigned ctr[4], int *err) {
  if (prev != PRT_INVALID) {
    if (in_element(M, prev, x0, x1, x2)) {
      ++ctr[CTR_SAME];
      return prev;
    }
    int best = -1;
    double max_ip = 0;
    const double *nrm = M.normals + 12 * (size_t)prev;
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      double ip = inner3_exact(nrm + 3 * f, p0, p1, p2);
      if (ip > max_ip) {
        best = f;
        max_ip = ip;
      }
    }
    if (best < 0) {
      *err = PRT_ERR_NO_BEST_NORMAL;
      return PRT_INVALID;
    }
    uint32_t nb = M.neighbors[4 * (size_t)prev + best];
    if (nb != PRT_INVALID && in_element(M, nb, x0, x1, x2)) {
      ++ctr[CTR_NEIGHBOR];
      return nb;
    }
    uint32_t cv = PRT_INVALID;
    double min_dist = __longlong_as_double(0x7ff0000000000000ll);  // +inf
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      uint32_t vi = M.el_verts[4 * (size_t)prev + v];
      double d = dist_exact(M.verts + 3 * (size_t)vi, x0, x1, x2);
      if (d < min_dist) {
        cv = vi;
        min_dist = d;
      }
    }
    if (cv != PRT_INVALID) {
      const uint32_t s = M.vadj_starts[cv], t = M.vadj_starts[cv + 1];
      for (uint32_t i = s; i < t; ++i) {
        uint32_t e = M.vadj[i];
        if (in_element(M, e, x0, x1, x2)) {
          ++ctr[CTR_VERTEX];
          return e;
        }
      }
    }
  }
  ++ctr[CTR_GLOBAL];
  return find_global(M, x0, x1, x2);
}

// update of one particle's element (particle_state.hpp:266-357): locate,
// else periodic wrap (positions written back) and locate again, else mark
// dead (PRT_INVALID). A successful wrap costs the extra find_same the
// reference's loop spends re-visiting the particle.
__device__ __forceinline__ uint32_t relocate(const DevMesh &M, double &x0, double &x1,
                                             double &x2, double p0, double p1,
                                             double p2, uint32_t prev, unsigned ctr[4],
                                             int *err, bool *wrapped) {
  *wrapped = false;
  uint32_t ne = find_new_containing(M, x0, x1, x2, p0, p1, p2, prev, ctr, err);
  if (ne != PRT_INVALID || *err) return ne;
  double pt[3] = {x0, x1, x2};
  bool trip = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double mn = M.pmin[a], mx = M.pmax[a];
    if (mn != mx) {
      if (pt[a] < mn) {
        pt[a] = __dadd_rn(pt[a], __dsub_rn(mx, mn));
        trip = true;
      } else if (pt[a] > mx) {
        pt[a] = __dsub_rn(pt[a], __dsub_rn(mx, mn));
        trip = true;
      }
    }
  }
  if (!trip) return PRT_INVALID;
  x0 = pt[0];
  x1 = pt[1];
  x2 = pt[2];
  *wrapped = true;
  ne = find_new_containing(M, x0, x1, x2, p0, p1, p2, prev, ctr, err);
  if (ne != PRT_INVALID) ++ctr[CTR_SAME];
  return ne;
}

// Warp-reduce the four counters and add them to the status word.
__device__ __forceinline__ void flush_counters(DevStatus *st, unsigned ctr[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    unsigned v = ctr[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&st->counters[k], (unsigned long long)v);
  }
}

inline int prt_grid_blocks(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  return (int)(b < 1 ? 1 : b);
}
