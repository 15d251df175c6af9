// core.cu -- mesh and workspace handles, kinematics, element location, the
// monomial pusher with the fused low-storage RK stage, and the element sort.
//
// Kernels here are particle-parallel (one thread per particle, SoA particle
// arrays) and HBM-bound: per particle and stage they move the state
// (x, p, q, m, element, two residuals: 216 bytes) once.

#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "handles.cuh"
#include "push.cuh"

// ------------------------------------------------------------------ errors

static thread_local char g_last_error[512];

void prt_note_cuda_error(cudaError_t e, const char *what, int line) {
  snprintf(g_last_error, sizeof(g_last_error), "CUDA error %d (%s) at core line %d: %s",
           (int)e, cudaGetErrorString(e), line, what);
}

extern "C" const char *prt_last_error_message(void) { return g_last_error; }

extern "C" const char *prt_version(void) { return "libprt 0.1 (sm_100a)"; }

// ------------------------------------------------------------------ memory

template <class T>
static int upload(T **dst, const T *src, size_t count) {
  *dst = nullptr;
  if (count == 0) return PRT_OK;
  if (!src) return PRT_ERR_INVALID_ARGUMENT;
  PRT_CHECK_CUDA(cudaMalloc((void **)dst, count * sizeof(T)));
  PRT_CHECK_CUDA(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
  return PRT_OK;
}

void *ws_buffer(prt_workspace *ws, int slot, size_t bytes, int *rc) {
  *rc = PRT_OK;
  if (slot < 0 || slot >= PRT_WS_SLOTS) {
    *rc = PRT_ERR_INVALID_ARGUMENT;
    return nullptr;
  }
  if (bytes == 0) bytes = 16;
  if (ws->cap[slot] < bytes) {
    if (ws->buf[slot]) {
      // earlier launches may still read the old buffer
      cudaDeviceSynchronize();
      cudaError_t e = cudaFree(ws->buf[slot]);
      if (e != cudaSuccess) {
        prt_note_cuda_error(e, "cudaFree(workspace)", __LINE__);
        *rc = PRT_ERR_CUDA;
        return nullptr;
      }
      ws->buf[slot] = nullptr;
      ws->cap[slot] = 0;
    }
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&ws->buf[slot], want);
    if (e != cudaSuccess) {
      prt_note_cuda_error(e, "cudaMalloc(workspace)", __LINE__);
      *rc = e == cudaErrorMemoryAllocation ? PRT_ERR_OUT_OF_MEMORY : PRT_ERR_CUDA;
      ws->buf[slot] = nullptr;
      return nullptr;
    }
    ws->cap[slot] = want;
  }
  return ws->buf[slot];
}

extern "C" int prt_mesh_create(const prt_mesh_desc *d, prt_mesh **out) {
  if (!d || !out || d->element_count <= 0 || d->vertex_count <= 0 ||
      d->nodes_per_element <= 0)
    return PRT_ERR_INVALID_ARGUMENT;
  prt_mesh *m = new prt_mesh();
  const size_t E = d->element_count, V = d->vertex_count, Np = d->nodes_per_element;
  const size_t nb = (size_t)d->bin_dims[0] * d->bin_dims[1] * d->bin_dims[2];
  if (nb == 0 || !d->bin_starts) {
    delete m;
    return PRT_ERR_INVALID_ARGUMENT;
  }
  DevMesh &D = m->dev;
  std::memset(&D, 0, sizeof(D));
  D.E = E;
  D.V = V;
  D.Np = (int)Np;
  int rc = PRT_OK;
  // upload `cnt` elements of `src` and store the device pointer in `field`
#define UP(field, src, cnt, T)             \
  do {                                     \
    T *p_ = nullptr;                       \
    if (rc == PRT_OK) rc = upload<T>(&p_, src, cnt); \
    field = p_;                            \
  } while (0)
  UP(D.inv_maps, d->inverse_maps, 12 * E, double);
  UP(D.jacobians, d->jacobians, E, double);
  UP(D.normals, d->face_normals, 12 * E, double);
  UP(D.plane_rhs, d->face_plane_rhs, 4 * E, double);
  UP(D.neighbors, d->face_neighbors, 4 * E, uint32_t);
  UP(D.axes, d->face_periodicity_axes, 4 * E, uint32_t);
  UP(D.el_verts, d->element_vertices, 4 * E, uint32_t);
  UP(D.verts, d->vertices, 3 * V, double);
  UP(D.vadj_starts, d->vertex_adj_starts, V + 1, uint32_t);
  size_t nadj = (rc == PRT_OK && d->vertex_adj_starts) ? d->vertex_adj_starts[V] : 0;
  UP(D.vadj, d->vertex_adj_elements, nadj, uint32_t);
  UP(D.nodes, d->nodes, 3 * E * Np, double);
  UP(D.bin_starts, d->bin_starts, nb + 1, uint32_t);
  size_t nbe = rc == PRT_OK ? d->bin_starts[nb] : 0;
  UP(D.bin_elements, d->bin_elements, nbe, uint32_t);
  UP(m->face_centroids, d->face_centroids, 12 * E, double);
  UP(m->face_radii, d->face_radii, 4 * E, double);
#undef UP
  for (int a = 0; a < 3; ++a) {
    D.pmin[a] = d->periodicity_min[a];
    D.pmax[a] = d->periodicity_max[a];
    D.bin_origin[a] = d->bin_origin[a];
    D.bin_inv[a] = d->bin_inv_width[a];
    D.bin_dims[a] = d->bin_dims[a];
  }
  if (rc == PRT_OK) rc = prt_mesh_build_positions(m, d);
  if (rc != PRT_OK) {
    prt_mesh_destroy(m);
    return rc;
  }
  *out = m;
  return PRT_OK;
}

extern "C" int prt_mesh_destroy(prt_mesh *m) {
  if (!m) return PRT_OK;
  const PositionSet &P = m->positions;
  const void *ptrs[] = {m->dev.inv_maps, m->dev.jacobians, m->dev.normals,
                        m->dev.plane_rhs, m->dev.neighbors, m->dev.axes,
                        m->dev.el_verts, m->dev.verts, m->dev.vadj_starts,
                        m->dev.vadj, m->dev.nodes, m->dev.bin_starts,
                        m->dev.bin_elements, m->face_centroids, m->face_radii,
                        P.pos, P.node_to_pos, P.run_starts, P.run_nodes,
                        P.group_starts, P.group_spheres,
                        P.centre_bins.starts, P.centre_bins.spheres, P.centre_bins.ranges,
                        P.wide_starts, P.wide_spheres};
  for (const void *p : ptrs)
    if (p) cudaFree((void *)p);
  delete m;
  return PRT_OK;
}

extern "C" int prt_workspace_create(prt_workspace **out) {
  if (!out) return PRT_ERR_INVALID_ARGUMENT;
  prt_workspace *ws = new prt_workspace();
  std::memset(ws->buf, 0, sizeof(ws->buf));
  std::memset(ws->cap, 0, sizeof(ws->cap));
  cudaError_t e = cudaMalloc(&ws->status, sizeof(DevStatus));
  if (e == cudaSuccess) e = cudaMemset(ws->status, 0, sizeof(DevStatus));
  if (e != cudaSuccess) {
    prt_note_cuda_error(e, "workspace status", __LINE__);
    delete ws;
    return PRT_ERR_CUDA;
  }
  *out = ws;
  return PRT_OK;
}

// ------------------------------------------------------------------ timing

static void fold_timer(KernelTimer &T) {
  for (int i = 0; i < T.used; ++i) {
    cudaEventSynchronize(T.stop[i]);
    float ms = 0;
    if (cudaEventElapsedTime(&ms, T.start[i], T.stop[i]) == cudaSuccess) {
      T.total_ms += ms;
      T.launches += 1;
    }
  }
  T.used = 0;
}

ScopedTimer::ScopedTimer(prt_workspace *w, int c, cudaStream_t st) : ws(w), cat(c), s(st) {
  if (!ws || !ws->timing || c < 0 || c >= PRT_TIME_CATEGORIES) return;
  // launches captured into a CUDA graph are not timed (the ring's
  // synchronising fold is not allowed while capturing)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return;
  KernelTimer &T = ws->timers[c];
  if (!T.created) {
    for (int i = 0; i < KernelTimer::RING; ++i) {
      cudaEventCreate(&T.start[i]);
      cudaEventCreate(&T.stop[i]);
    }
    T.created = true;
  }
  if (T.used >= KernelTimer::RING) fold_timer(T);
  slot = T.used++;
  cudaEventRecord(T.start[slot], s);
}

ScopedTimer::~ScopedTimer() {
  if (slot >= 0) cudaEventRecord(ws->timers[cat].stop[slot], s);
}

extern "C" int prt_workspace_timing(prt_workspace *ws, int32_t enable) {
  if (!ws) return PRT_ERR_INVALID_ARGUMENT;
  ws->timing = enable != 0;
  return PRT_OK;
}

extern "C" int prt_workspace_timing_read(prt_workspace *ws, int32_t cat, double *total_ms,
                                         int64_t *launches, int32_t reset) {
  if (!ws || cat < 0 || cat >= PRT_TIME_CATEGORIES) return PRT_ERR_INVALID_ARGUMENT;
  KernelTimer &T = ws->timers[cat];
  fold_timer(T);
  if (total_ms) *total_ms = T.total_ms;
  if (launches) *launches = T.launches;
  if (reset) {
    T.total_ms = 0;
    T.launches = 0;
  }
  return PRT_OK;
}

extern "C" int prt_workspace_destroy(prt_workspace *ws) {
  if (!ws) return PRT_OK;
  for (int c = 0; c < PRT_TIME_CATEGORIES; ++c)
    if (ws->timers[c].created)
      for (int i = 0; i < KernelTimer::RING; ++i) {
        cudaEventDestroy(ws->timers[c].start[i]);
        cudaEventDestroy(ws->timers[c].stop[i]);
      }
  for (int i = 0; i < PRT_WS_SLOTS; ++i)
    if (ws->buf[i]) cudaFree(ws->buf[i]);
  if (ws->status) cudaFree(ws->status);
  delete ws;
  return PRT_OK;
}

extern "C" int prt_workspace_status(prt_workspace *ws, void *stream, int32_t *error,
                                    int64_t *error_index, int32_t *warning,
                                    int64_t *warning_index, int32_t clear) {
  if (!ws) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  DevStatus h;
  PRT_CHECK_CUDA(cudaMemcpyAsync(&h, ws->status, sizeof(h), cudaMemcpyDeviceToHost, s));
  PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  if (error) *error = h.error;
  if (error_index) *error_index = h.error_index;
  if (warning) *warning = h.warning;
  if (warning_index) *warning_index = h.warning_index;
  if (clear) {
    PRT_CHECK_CUDA(cudaMemsetAsync(ws->status, 0, offsetof(DevStatus, counters), s));
    PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  }
  return PRT_OK;
}

extern "C" int prt_workspace_counters(prt_workspace *ws, void *stream,
                                      prt_find_counters *out, int32_t reset) {
  if (!ws || !out) return PRT_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  DevStatus h;
  PRT_CHECK_CUDA(cudaMemcpyAsync(&h, ws->status, sizeof(h), cudaMemcpyDeviceToHost, s));
  PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  out->find_same = h.counters[0];
  out->find_by_neighbor = h.counters[1];
  out->find_by_vertex = h.counters[2];
  out->find_global = h.counters[3];
  if (reset) {
    PRT_CHECK_CUDA(cudaMemsetAsync((char *)ws->status + offsetof(DevStatus, counters), 0,
                                   sizeof(h.counters), s));
    PRT_CHECK_CUDA(cudaStreamSynchronize(s));
  }
  return PRT_OK;
}

// -------------------------------------------------------------- kinematics

__global__ void velocities_kernel(long long n, const double *__restrict__ p,
                                  const double *__restrict__ m, double c,
                                  double *__restrict__ v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v0, v1, v2;
  velocity_exact(p[i], p[n + i], p[2 * n + i], m[i], c, v0, v1, v2);
  v[i] = v0;
  v[n + i] = v1;
  v[2 * n + i] = v2;
}

extern "C" int prt_get_velocities(int64_t n, const double *p, const double *m, double c,
                                  double *v, void *stream) {
  if (n < 0 || (n > 0 && (!p || !m || !v))) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  velocities_kernel<<<prt_grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(n, p, m, c, v);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

__global__ void find_global_kernel(DevMesh M, long long n, const double *__restrict__ x,
                                   uint32_t *__restrict__ el) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  el[i] = find_global(M, x[i], x[n + i], x[2 * n + i]);
}

extern "C" int prt_find_containing_elements(const prt_mesh *mesh, int64_t n,
                                            const double *x, uint32_t *el,
                                            void *stream) {
  if (!mesh || n < 0 || (n > 0 && (!x || !el))) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  find_global_kernel<<<prt_grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(mesh->dev, n,
                                                                                 x, el);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

__global__ void update_elements_kernel(DevMesh M, long long n, double *__restrict__ x,
                                       const double *__restrict__ p,
                                       uint32_t *__restrict__ el, DevStatus *st) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned ctr[4] = {0, 0, 0, 0};
  uint32_t prev = i < n ? el[i] : PRT_INVALID;
  if (prev != PRT_INVALID) {
    double x0 = x[i], x1 = x[n + i], x2 = x[2 * n + i];
    int err = 0;
    bool wrapped;
    uint32_t ne = relocate(M, x0, x1, x2, p[i], p[n + i], p[2 * n + i], prev, ctr, &err,
                           &wrapped);
    if (err) {
      record_error(st, err, i);
    } else {
      if (wrapped) {
        x[i] = x0;
        x[n + i] = x1;
        x[2 * n + i] = x2;
      }
      el[i] = ne;
    }
  }
  flush_counters(st, ctr);
}

extern "C" int prt_update_containing_elements(const prt_mesh *mesh, prt_workspace *ws,
                                              int64_t n, double *x, const double *p,
                                              uint32_t *el, void *stream) {
  if (!mesh || !ws || n < 0 || (n > 0 && (!x || !p || !el)))
    return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  update_elements_kernel<<<prt_grid_blocks(n, 256), 256, 0, (cudaStream_t)stream>>>(
      mesh->dev, n, x, p, el, ws->status);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

// ------------------------------------------------------------------ pusher

template <int ORDER>
__global__ void __launch_bounds__(256)
    forces_kernel(DevMesh M, const Lagrange<ORDER> L, Fields6 F, long long n,
                  const double *__restrict__ x, const uint32_t *__restrict__ el,
                  const double *__restrict__ q, const double *__restrict__ v,
                  double *__restrict__ out, double *__restrict__ vis) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t e = el[i];
  double ef[6] = {0, 0, 0, 0, 0, 0};
  if (e != PRT_INVALID)
    interpolate_fields<ORDER>(M, L, F, e, x[i], x[n + i], x[2 * n + i], ef);
  const double charge = q[i];
  double elf[3], qb[3], mag[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    elf[d] = __dmul_rn(charge, ef[d]);
    qb[d] = __dmul_rn(charge, ef[3 + d]);
  }
  const double v0 = v[i], v1 = v[n + i], v2 = v[2 * n + i];
  mag[0] = __dsub_rn(__dmul_rn(v1, qb[2]), __dmul_rn(v2, qb[1]));
  mag[1] = __dsub_rn(__dmul_rn(v2, qb[0]), __dmul_rn(v0, qb[2]));
  mag[2] = __dsub_rn(__dmul_rn(v0, qb[1]), __dmul_rn(v1, qb[0]));
#pragma unroll
  for (int d = 0; d < 3; ++d) out[d * n + i] = __dadd_rn(elf[d], mag[d]);
  if (vis) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      vis[(0 * 3 + d) * n + i] = ef[d];
      vis[(1 * 3 + d) * n + i] = ef[3 + d];
      vis[(2 * 3 + d) * n + i] = elf[d];
      vis[(3 * 3 + d) * n + i] = mag[d];
    }
  }
}

#ifndef PRT_STAGE_MIN_BLOCKS
#define PRT_STAGE_MIN_BLOCKS 3
#endif

// One fused stage: velocity, interpolation, Lorentz force, 2N-storage RK
// update, relocation. Dead particles (PRT_INVALID) are not touched.
// resident 256-thread CTAs per SM the stage kernel is compiled for: the
// kernel is latency-bound, so occupancy matters more than registers, up to
// order 3; order 4 (35 monomials in registers) keeps the larger budget
template <int ORDER>
__global__ void __launch_bounds__(256, ORDER >= 4 ? 2 : PRT_STAGE_MIN_BLOCKS)
    lsrk_stage_kernel(DevMesh M, const Lagrange<ORDER> L, Fields6 F, long long n,
                      double *__restrict__ x, double *__restrict__ p,
                      const double *__restrict__ q, const double *__restrict__ mass,
                      uint32_t *__restrict__ el, double *__restrict__ kx,
                      double *__restrict__ kp, double a, double b, double dt,
                      double c, DevStatus *st) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  unsigned ctr[4] = {0, 0, 0, 0};
  const uint32_t e = i < n ? el[i] : PRT_INVALID;
  if (e != PRT_INVALID) {
    double xx[3] = {x[i], x[n + i], x[2 * n + i]};
    double pp[3] = {p[i], p[n + i], p[2 * n + i]};
    int err = 0;
    const uint32_t ne = stage_particle<ORDER>(M, L, F, e, xx, pp, q[i], mass[i], kx, kp, n, i,
                                              a, b, dt, c, ctr, &err);
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

// Host-side inverse of the monomial Vandermonde, by Gaussian elimination
// with partial pivoting (n <= 35).
static bool invert(int n, std::vector<double> a, std::vector<double> &inv) {
  inv.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1;
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(a[(size_t)r * n + col]) > std::fabs(a[(size_t)piv * n + col])) piv = r;
    if (a[(size_t)piv * n + col] == 0) return false;
    if (piv != col)
      for (int k = 0; k < n; ++k) {
        std::swap(a[(size_t)piv * n + k], a[(size_t)col * n + k]);
        std::swap(inv[(size_t)piv * n + k], inv[(size_t)col * n + k]);
      }
    double d = a[(size_t)col * n + col];
    for (int k = 0; k < n; ++k) {
      a[(size_t)col * n + k] /= d;
      inv[(size_t)col * n + k] /= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      double f = a[(size_t)r * n + col];
      if (f == 0) continue;
      for (int k = 0; k < n; ++k) {
        a[(size_t)r * n + k] -= f * a[(size_t)col * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)col * n + k];
      }
    }
  }
  return true;
}

extern "C" int prt_monomial_pusher_create(const prt_mesh *mesh, int32_t np,
                                          const uint32_t *exps, const double *vdm,
                                          prt_pusher **out) {
  if (!mesh || !exps || !vdm || !out || np != mesh->dev.Np) return PRT_ERR_INVALID_ARGUMENT;
  int order = -1;
  for (int o = 0; o <= 4; ++o)
    if ((o + 1) * (o + 2) * (o + 3) / 6 == np) order = o;
  if (order < 1) return PRT_ERR_INVALID_ARGUMENT;
  // canonical position of each exponent tuple; the set must be all of P_order
  std::vector<int> canon(np, -1);
  {
    int idx = 0;
    std::vector<int> seen(np, 0);
    for (int c = 0; c <= order; ++c)
      for (int b = 0; b <= order - c; ++b)
        for (int a = 0; a <= order - b - c; ++a) {
          int found = -1;
          for (int k = 0; k < np; ++k)
            if ((int)exps[3 * k] == a && (int)exps[3 * k + 1] == b &&
                (int)exps[3 * k + 2] == c)
              found = k;
          if (found < 0 || seen[found]) return PRT_ERR_INVALID_ARGUMENT;
          seen[found] = 1;
          canon[found] = idx++;
        }
  }
  std::vector<double> V(vdm, vdm + (size_t)np * np), Vinv;
  if (!invert(np, V, Vinv)) return PRT_ERR_INVALID_ARGUMENT;
  // Lagrange value i = sum_k Vinv[k][i] monomial_k; reorder k canonically.
  prt_pusher *P = new prt_pusher();
  P->mesh = mesh;
  P->order = order;
  P->np = np;
  P->w.assign((size_t)np * np, 0.0);
  for (int i = 0; i < np; ++i)
    for (int k = 0; k < np; ++k) P->w[(size_t)i * np + canon[k]] = Vinv[(size_t)k * np + i];
  int rc = prt_pusher_prepare_mixed(P);
  if (rc) {
    delete P;
    return rc;
  }
  *out = P;
  return PRT_OK;
}

extern "C" int prt_monomial_pusher_destroy(prt_pusher *p) {
  if (p && p->w_split) cudaFree(p->w_split);
  delete p;
  return PRT_OK;
}

template <int ORDER>
static int launch_forces(const prt_pusher *P, long long n, const double *x,
                         const uint32_t *el, const double *q, const double *v,
                         Fields6 F, double *out, double *vis, cudaStream_t s) {
  forces_kernel<ORDER><<<prt_grid_blocks(n, 256), 256, 0, s>>>(
      P->mesh->dev, make_lagrange<ORDER>(P), F, n, x, el, q, v, out, vis);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

extern "C" int prt_forces(const prt_pusher *P, int64_t n, const double *x,
                          const uint32_t *el, const double *q, const double *v,
                          const double *const fields[6], double *out, double *vis,
                          void *stream) {
  if (!P || n < 0 || (n > 0 && (!x || !el || !q || !v || !out)) || !fields)
    return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  Fields6 F;
  for (int k = 0; k < 6; ++k) F.f[k] = fields[k];
  cudaStream_t s = (cudaStream_t)stream;
  switch (P->order) {
    case 1: return launch_forces<1>(P, n, x, el, q, v, F, out, vis, s);
    case 2: return launch_forces<2>(P, n, x, el, q, v, F, out, vis, s);
    case 3: return launch_forces<3>(P, n, x, el, q, v, F, out, vis, s);
    case 4: return launch_forces<4>(P, n, x, el, q, v, F, out, vis, s);
  }
  return PRT_ERR_INVALID_ARGUMENT;
}

template <int ORDER>
static int launch_stage(const prt_pusher *P, prt_workspace *ws, long long n, double *x,
                        double *p, const double *q, const double *m, uint32_t *el,
                        double *kx, double *kp, Fields6 F, double a, double b,
                        double dt, double c, cudaStream_t s) {
  ScopedTimer timer(ws, PRT_TIME_LSRK_STAGE, s);
  lsrk_stage_kernel<ORDER><<<prt_grid_blocks(n, 256), 256, 0, s>>>(
      P->mesh->dev, make_lagrange<ORDER>(P), F, n, x, p, q, m, el, kx, kp, a, b, dt, c,
      ws->status);
  PRT_CHECK_CUDA(cudaGetLastError());
  return PRT_OK;
}

extern "C" int prt_lsrk_stage(const prt_pusher *P, prt_workspace *ws, int64_t n,
                              double *x, double *p, const double *q, const double *m,
                              uint32_t *el, double *kx, double *kp,
                              const double *const fields[6], double a, double b,
                              double dt, double c, int32_t precision, void *stream) {
  if (!P || !ws || n < 0 || !fields) return PRT_ERR_INVALID_ARGUMENT;
  if (precision != PRT_PRECISION_FP64 && precision != PRT_PRECISION_MIXED)
    return PRT_ERR_INVALID_ARGUMENT;
  if (precision == PRT_PRECISION_MIXED && !P->w_split) return PRT_ERR_INVALID_ARGUMENT;
  if (n > 0 && (!x || !p || !q || !m || !el || !kx || !kp)) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  Fields6 F;
  for (int k = 0; k < 6; ++k) F.f[k] = fields[k];
  cudaStream_t s = (cudaStream_t)stream;
  if (precision == PRT_PRECISION_MIXED)
    return launch_stage_mixed(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
  switch (P->order) {
    case 1: return launch_stage<1>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
    case 2: return launch_stage<2>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
    case 3: return launch_stage<3>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
    case 4: return launch_stage<4>(P, ws, n, x, p, q, m, el, kx, kp, F, a, b, dt, c, s);
  }
  return PRT_ERR_INVALID_ARGUMENT;
}

// -------------------------------------------------------------------- sort

__global__ void iota_kernel(long long n, uint32_t *__restrict__ v) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) v[i] = (uint32_t)i;
}

template <class T, int C>
__global__ void permute_kernel(long long n, const uint32_t *__restrict__ perm,
                              const T *__restrict__ src, T *__restrict__ dst) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t j = perm[i];
#pragma unroll
  for (int c = 0; c < C; ++c) dst[c * n + i] = src[c * n + j];
}

template <class T, int C>
static int permute(prt_workspace *ws, long long n, const uint32_t *perm, T *arr,
                   cudaStream_t s) {
  if (!arr) return PRT_OK;
  int rc;
  T *tmp = (T *)ws_buffer(ws, PRT_WS_SORT_TMP, sizeof(T) * C * (size_t)n, &rc);
  if (!tmp) return rc;
  permute_kernel<T, C><<<prt_grid_blocks(n, 256), 256, 0, s>>>(n, perm, arr, tmp);
  PRT_CHECK_CUDA(cudaGetLastError());
  PRT_CHECK_CUDA(
      cudaMemcpyAsync(arr, tmp, sizeof(T) * C * (size_t)n, cudaMemcpyDeviceToDevice, s));
  return PRT_OK;
}

extern "C" int prt_sort_by_element(prt_workspace *ws, int64_t n, uint32_t *el, double *x,
                                   double *p, double *q, double *m, double *kx,
                                   double *kp, int64_t *ids, void *stream) {
  if (!ws || n < 0 || (n > 0 && !el) || n >= (1ll << 31)) return PRT_ERR_INVALID_ARGUMENT;
  if (n == 0) return PRT_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int rc;
  ScopedTimer timer(ws, PRT_TIME_SORT, s);
  uint32_t *keys_out = (uint32_t *)ws_buffer(ws, PRT_WS_SORT_KEYS, 4 * (size_t)n, &rc);
  if (!keys_out) return rc;
  uint32_t *vals = (uint32_t *)ws_buffer(ws, PRT_WS_SORT_VALS, 8 * (size_t)n, &rc);
  if (!vals) return rc;
  uint32_t *vals_out = vals + n;
  size_t temp_bytes = 0;
  PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, el, keys_out, vals,
                                                 vals_out, (int)n, 0, 32, s));
  void *temp = ws_buffer(ws, PRT_WS_CUB, temp_bytes, &rc);
  if (!temp) return rc;
  iota_kernel<<<prt_grid_blocks(n, 256), 256, 0, s>>>(n, vals);
  PRT_CHECK_CUDA(cudaGetLastError());
  PRT_CHECK_CUDA(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, el, keys_out, vals,
                                                 vals_out, (int)n, 0, 32, s));
  PRT_CHECK_CUDA(cudaMemcpyAsync(el, keys_out, 4 * (size_t)n, cudaMemcpyDeviceToDevice, s));
  if ((rc = permute<double, 3>(ws, n, vals_out, x, s))) return rc;
  if ((rc = permute<double, 3>(ws, n, vals_out, p, s))) return rc;
  if ((rc = permute<double, 1>(ws, n, vals_out, q, s))) return rc;
  if ((rc = permute<double, 1>(ws, n, vals_out, m, s))) return rc;
  if ((rc = permute<double, 3>(ws, n, vals_out, kx, s))) return rc;
  if ((rc = permute<double, 3>(ws, n, vals_out, kp, s))) return rc;
  if ((rc = permute<int64_t, 1>(ws, n, vals_out, ids, s))) return rc;
  return PRT_OK;
}
