// oracle.cpp -- CPU restatement of pyrticle's particle-side algorithms.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity oracle: tests/, the
// smoke check and the CPU-baseline leg of bench.py call it as the checker.
// The product path (libprt.so) never links, loads or calls it.
//
// The reference (inducer/pyrticle) cannot be built here: it needs Python 2,
// Boost.Python/uBLAS, boost-bindings, PyUblas and hedge. So this is a
// restatement, serial, in the reference's own loop and decision order, with
// ublas's summation order (t = 0; t += a_i b_i) and no FMA contraction
// (build with -ffp-contract=off). Layout follows the reference: positions and
// momenta are [n][3], fields are [Nn] per component, j is [Nn][3].
//
// Each function cites the reference source it restates.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <unordered_set>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/prt.h"

namespace {

typedef prt_mesh_desc Mesh;
const uint32_t INVALID = PRT_INVALID_ELEMENT;

// hedge affine_map::operator(): prod(matrix, x) + vector, ublas row order.
inline void apply_map(const double *m, const double *x, double *y) {
  for (int i = 0; i < 3; ++i) {
    double t = 0;
    t += m[3 * i + 0] * x[0];
    t += m[3 * i + 1] * x[1];
    t += m[3 * i + 2] * x[2];
    y[i] = t + m[9 + i];
  }
}

// meshdata.hpp:38-48
inline bool is_in_unit_simplex(const double *r, double tolerance = 1e-10) {
  for (int i = 0; i < 3; ++i)
    if (r[i] < -1 - tolerance) return false;
  double s = 0;
  s = s + r[0];
  s = s + r[1];
  s = s + r[2];
  return s <= -(3 - 2) + tolerance;
}

inline bool in_element(const Mesh &m, uint32_t en, const double *pt) {
  double r[3];
  apply_map(m.inverse_maps + 12 * (size_t)en, pt, r);
  return is_in_unit_simplex(r);
}

inline double inner3(const double *a, const double *b) {
  double t = 0;
  t += a[0] * b[0];
  t += a[1] * b[1];
  t += a[2] * b[2];
  return t;
}

inline double norm2_diff(const double *a, const double *b) {
  double t = 0;
  for (int i = 0; i < 3; ++i) {
    double d = a[i] - b[i];
    t += d * d;
  }
  return std::sqrt(t);
}

// meshdata.hpp:208-215: the first element (in element order) containing pt.
uint32_t find_containing_element(const Mesh &m, const double *pt) {
  for (int64_t e = 0; e < m.element_count; ++e)
    if (in_element(m, (uint32_t)e, pt)) return (uint32_t)e;
  return INVALID;
}

struct NoBestNormal : std::runtime_error {
  NoBestNormal() : std::runtime_error("no best normal found--weird") {}
};

// particle_state.hpp:130-261
uint32_t find_new_containing_element(const Mesh &m, const double *pt,
                                     const double *mom, uint32_t prev,
                                     prt_find_counters &ctr, bool linear_global) {
  if (prev != INVALID) {
    if (in_element(m, prev, pt)) {
      ++ctr.find_same;
      return prev;
    }
    {
      int closest_normal_idx = -1;
      double max_ip = 0;
      for (int f = 0; f < 4; ++f) {
        double ip = inner3(m.face_normals + 12 * (size_t)prev + 3 * f, mom);
        if (ip > max_ip) {
          closest_normal_idx = f;
          max_ip = ip;
        }
      }
      if (closest_normal_idx == -1) throw NoBestNormal();
      uint32_t possible = m.face_neighbors[4 * (size_t)prev + closest_normal_idx];
      if (possible != INVALID && in_element(m, possible, pt)) {
        ++ctr.find_by_neighbor;
        return possible;
      }
    }
    {
      uint32_t closest_vertex = INVALID;
      double min_dist = std::numeric_limits<double>::infinity();
      for (int v = 0; v < 4; ++v) {
        uint32_t vi = m.element_vertices[4 * (size_t)prev + v];
        double dist = norm2_diff(m.vertices + 3 * (size_t)vi, pt);
        if (dist < min_dist) {
          closest_vertex = vi;
          min_dist = dist;
        }
      }
      for (uint32_t i = m.vertex_adj_starts[closest_vertex];
           i < m.vertex_adj_starts[closest_vertex + 1]; ++i) {
        uint32_t possible = m.vertex_adj_elements[i];
        if (in_element(m, possible, pt)) {
          ++ctr.find_by_vertex;
          return possible;
        }
      }
    }
  }
  ++ctr.find_global;
  if (linear_global) return find_containing_element(m, pt);
  // Same answer through the element bins: lowest id among containing
  // candidates (every element that can contain pt is listed in its bin).
  int b[3];
  for (int d = 0; d < 3; ++d) {
    double u = (pt[d] - m.bin_origin[d]) * m.bin_inv_width[d];
    int bi;
    if (!(u >= 0))
      bi = 0;
    else if (u >= (double)m.bin_dims[d])
      bi = m.bin_dims[d] - 1;
    else
      bi = std::min((int)u, m.bin_dims[d] - 1);
    b[d] = bi;
  }
  size_t bid = b[0] + (size_t)m.bin_dims[0] * (b[1] + (size_t)m.bin_dims[1] * b[2]);
  for (uint32_t i = m.bin_starts[bid]; i < m.bin_starts[bid + 1]; ++i)
    if (in_element(m, m.bin_elements[i], pt)) return m.bin_elements[i];
  return INVALID;
}

// A particle store with the swap-with-last removal of particle_state.hpp:361-407,
// carrying the LSRK residuals along (the NumberShiftableVectors of
// tools.py:106-178 shift with the particles) and a stable id.
struct Store {
  int64_t n;
  double *x, *p, *q, *m;
  uint32_t *el;
  double *kx, *kp;
  int64_t *ids;
  void move(int64_t from, int64_t to) {
    el[to] = el[from];
    for (int i = 0; i < 3; ++i) {
      x[3 * to + i] = x[3 * from + i];
      p[3 * to + i] = p[3 * from + i];
      if (kx) kx[3 * to + i] = kx[3 * from + i];
      if (kp) kp[3 * to + i] = kp[3 * from + i];
    }
    q[to] = q[from];
    m[to] = m[from];
    if (ids) ids[to] = ids[from];
  }
  void kill(int64_t pn) {
    --n;
    if (n) move(n, pn);
  }
};

// particle_state.hpp:301-357 (boundary_hit); returns true when the particle
// was re-found after a periodic wrap, false when the listener must kill it.
bool boundary_hit(const Mesh &m, Store &s, int64_t pn, prt_find_counters &ctr,
                  bool linear_global) {
  double pt[3] = {s.x[3 * pn], s.x[3 * pn + 1], s.x[3 * pn + 2]};
  bool trip = false;
  for (int axis = 0; axis < 3; ++axis) {
    double mn = m.periodicity_min[axis], mx = m.periodicity_max[axis];
    if (mn != mx) {
      double xi = pt[axis];
      if (xi < mn) {
        pt[axis] += (mx - mn);
        trip = true;
      } else if (xi > mx) {
        pt[axis] -= (mx - mn);
        trip = true;
      }
    }
  }
  if (trip) {
    for (int i = 0; i < 3; ++i) s.x[3 * pn + i] = pt[i];
    uint32_t ce = find_new_containing_element(m, s.x + 3 * pn, s.p + 3 * pn,
                                              s.el[pn], ctr, linear_global);
    if (ce != INVALID) {
      s.el[pn] = ce;
      return true;
    }
  }
  return false;
}

// particle_state.hpp:266-295 with the kill listener of cloud.py:581-585.
void update_containing_elements(const Mesh &m, Store &s, prt_find_counters &ctr,
                                bool linear_global) {
  for (int64_t pn = 0; pn < s.n;) {
    uint32_t prev = s.el[pn];
    uint32_t ne = find_new_containing_element(m, s.x + 3 * pn, s.p + 3 * pn, prev,
                                              ctr, linear_global);
    if (ne == INVALID) {
      if (!boundary_hit(m, s, pn, ctr, linear_global)) s.kill(pn);
    } else {
      s.el[pn] = ne;
      ++pn;
    }
  }
}

// particle_state.hpp:98-125
void get_velocities(int64_t n, const double *p, const double *mass, double c,
                    double *v) {
  for (int64_t pn = 0; pn < n; ++pn) {
    const double *pp = p + 3 * pn;
    double pabs = 0;
    pabs += pp[0] * pp[0];
    pabs += pp[1] * pp[1];
    pabs += pp[2] * pp[2];
    pabs = std::sqrt(pabs);
    if (pabs == 0) {
      v[3 * pn] = v[3 * pn + 1] = v[3 * pn + 2] = 0;
    } else {
      const double mm = mass[pn];
      double vv = c * pabs / std::sqrt(mm * mm * c * c + pabs * pabs);
      for (int i = 0; i < 3; ++i) v[3 * pn + i] = vv / pabs * pp[i];
    }
  }
}

// ---------------------------------------------------------------- pusher

// LU with partial pivoting, column by column (the published dgetf2 algorithm,
// called by lu() in wrap_tools.cpp:126-145); a is column-major n x n.
int lu_factor(int n, double *a, int *piv) {
  for (int j = 0; j < n; ++j) {
    int p = j;
    double best = std::fabs(a[j + n * j]);
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(a[i + n * j]) > best) {
        best = std::fabs(a[i + n * j]);
        p = i;
      }
    piv[j] = p;
    if (a[p + n * j] == 0) return j + 1;
    if (p != j)
      for (int k = 0; k < n; ++k) std::swap(a[j + n * k], a[p + n * k]);
    double r = 1.0 / a[j + n * j];
    for (int i = j + 1; i < n; ++i) a[i + n * j] *= r;
    for (int k = j + 1; k < n; ++k) {
      double t = a[j + n * k];
      for (int i = j + 1; i < n; ++i) a[i + n * k] -= a[i + n * j] * t;
    }
  }
  return 0;
}

// getrs('N') (push_monomial.hpp:188-206): row swaps, unit-lower solve, upper solve.
void lu_solve(int n, const double *lu, const int *piv, double *b) {
  for (int j = 0; j < n; ++j)
    if (piv[j] != j) std::swap(b[j], b[piv[j]]);
  for (int j = 0; j < n; ++j) {
    double t = b[j];
    if (t != 0)
      for (int i = j + 1; i < n; ++i) b[i] -= t * lu[i + n * j];
  }
  for (int j = n - 1; j >= 0; --j) {
    if (b[j] != 0) {
      b[j] /= lu[j + n * j];
      double t = b[j];
      for (int i = 0; i < j; ++i) b[i] -= t * lu[i + n * j];
    }
  }
}

struct Pusher {
  int np;
  std::vector<uint32_t> exps;   // [np][3]
  std::vector<double> lu;       // column-major LU of V^T
  std::vector<int> piv;
};

inline double ipow(double x, unsigned e) {
  // pow(v[i], exp) with integer exponent (push_monomial.hpp:66)
  return std::pow(x, (double)e);
}

// push_monomial.hpp:155-325 for a range of particles; fields[k] may be NULL.
void forces(const Pusher &P, const Mesh &m, int64_t n, const double *x,
            const uint32_t *el, const double *q, const double *v,
            const double *const fields[6], double *out, double *vis) {
  const int np = P.np;
  static thread_local std::vector<double> coeff;
  coeff.resize(np);
  for (int64_t pn = 0; pn < n; ++pn) {
    uint32_t en = el[pn];
    double unit_pt[3];
    apply_map(m.inverse_maps + 12 * (size_t)en, x + 3 * pn, unit_pt);
    for (int i = 0; i < np; ++i) {
      double r = 1;
      for (int d = 0; d < 3; ++d) r *= ipow(unit_pt[d], P.exps[3 * i + d]);
      coeff[i] = r;
    }
    lu_solve(np, P.lu.data(), P.piv.data(), coeff.data());
    double eb[6];
    for (int k = 0; k < 6; ++k) {
      if (!fields[k]) {
        eb[k] = 0;
        continue;
      }
      const double *f = fields[k] + (size_t)en * np;
      double t = 0;
      for (int i = 0; i < np; ++i) t += coeff[i] * f[i];
      eb[k] = t;
    }
    const double charge = q[pn];
    double el_force[3], qb[3], mag[3];
    for (int i = 0; i < 3; ++i) {
      el_force[i] = charge * eb[i];
      qb[i] = charge * eb[3 + i];
    }
    const double *vv = v + 3 * pn;
    mag[0] = vv[1] * qb[2] - vv[2] * qb[1];
    mag[1] = vv[2] * qb[0] - vv[0] * qb[2];
    mag[2] = vv[0] * qb[1] - vv[1] * qb[0];
    for (int i = 0; i < 3; ++i) out[3 * pn + i] = el_force[i] + mag[i];
    if (vis) {
      for (int i = 0; i < 3; ++i) {
        vis[0 * 3 * n + 3 * pn + i] = eb[i];
        vis[1 * 3 * n + 3 * pn + i] = eb[3 + i];
        vis[2 * 3 * n + 3 * pn + i] = el_force[i];
        vis[3 * 3 * n + 3 * pn + i] = mag[i];
      }
    }
  }
}

// ------------------------------------------------------------ deposition

struct Shape {
  double radius, radius_squared, alpha, normalizer;
  bool alpha_is_2;
  // tools.hpp:514-535
  double operator()(const double *r) const {
    double r_squared = 0;
    r_squared += r[0] * r[0];
    r_squared += r[1] * r[1];
    r_squared += r[2] * r[2];
    if (r_squared > radius_squared) return 0;
    double radius_term = radius - r_squared / radius;
    if (alpha_is_2) return normalizer * radius_term * radius_term;
    return normalizer * std::pow(radius_term, alpha);
  }
};

Shape make_shape(const prt_shape_function &s) {
  Shape sh;
  sh.radius = s.radius;
  sh.radius_squared = s.radius * s.radius;
  sh.alpha = s.alpha;
  sh.normalizer = s.normalizer;
  sh.alpha_is_2 = s.alpha == 2;
  return sh;
}

// Deposition target: rho [Nn] and/or j [Nn][3] (dep_target.hpp:54-148).
struct Target {
  double *rho;
  double *j;
  const double *vel;  // [n][3]
  double sf[3];
  void begin_particle(int64_t pn) {
    if (j)
      for (int a = 0; a < 3; ++a) sf[a] = vel[3 * pn + a];
  }
  void add(size_t start, const double *contrib, int len) {
    if (rho)
      for (int i = 0; i < len; ++i) rho[start + i] += contrib[i];
    if (j)
      for (int i = 0; i < len; ++i) {
        double r = contrib[i];
        for (int a = 0; a < 3; ++a) j[(start + i) * 3 + a] += sf[a] * r;
      }
  }
};

struct DepStats {
  // Welford accumulators (tools.hpp:340-417)
  struct W {
    unsigned count = 0;
    double mean = 0, m2 = 0, mn = 0, mx = 0;
    void add(double x) {
      if (count == 0 || x < mn) mn = x;
      if (count == 0 || x > mx) mx = x;
      ++count;
      double delta = x - mean;
      mean += delta / double(count);
      m2 += delta * (x - mean);
    }
  } norm, centroid, el_per_particle;
};

// face_based_element_finder::recurse (element_finder.hpp:239-293). The
// visitor receives (center, element).
template <class Visitor>
void walk(const Mesh &m, const double *pos, double radius,
          std::unordered_set<uint32_t> &el_set, uint32_t en, Visitor &vis) {
  vis(pos, en);
  el_set.insert(en);
  for (int f = 0; f < 4; ++f) {
    const size_t fi = 4 * (size_t)en + f;
    uint32_t nb = m.face_neighbors[fi];
    if (nb == INVALID) continue;
    if (el_set.find(nb) != el_set.end()) continue;
    const double *normal = m.face_normals + 3 * fi;
    double plane_dist = std::fabs(inner3(pos, normal) - m.face_plane_rhs[fi]);
    if (plane_dist > radius) continue;
    if (norm2_diff(m.face_centroids + 3 * fi, pos) > radius + m.face_radii[fi])
      continue;
    uint32_t per_axis = m.face_periodicity_axes[fi];
    if (per_axis == PRT_INVALID_AXIS)
      walk(m, pos, radius, el_set, nb, vis);
    else {
      double pos2[3] = {pos[0], pos[1], pos[2]};
      double mn = m.periodicity_min[per_axis], mx = m.periodicity_max[per_axis];
      if (pos[per_axis] - radius < mn) {
        pos2[per_axis] += (mx - mn);
        walk(m, pos2, radius, el_set, nb, vis);
      }
      if (pos[per_axis] + radius > mx) {
        pos2[per_axis] -= (mx - mn);
        walk(m, pos2, radius, el_set, nb, vis);
      }
    }
  }
}

// shape_function_depositor (dep_shape.hpp:67-149)
void deposit_plain(const Mesh &m, const Shape &sf, int64_t n, const double *x,
                   const double *q, const uint32_t *el, Target &tgt) {
  const int np = m.nodes_per_element;
  std::vector<double> el_rho(np);
  for (int64_t pn = 0; pn < n; ++pn) {
    const double charge = q[pn];
    tgt.begin_particle(pn);
    auto add_shape_on_element = [&](const double *center, uint32_t en) {
      size_t start = (size_t)en * np;
      for (int i = 0; i < np; ++i) {
        const double *node = m.nodes + 3 * (start + i);
        double d[3] = {node[0] - center[0], node[1] - center[1], node[2] - center[2]};
        el_rho[i] = charge * sf(d);
      }
      tgt.add(start, el_rho.data(), np);
    };
    std::unordered_set<uint32_t> el_set;
    walk(m, x + 3 * pn, sf.radius, el_set, el[pn], add_shape_on_element);
  }
}

// normalized_shape_function_depositor (dep_normshape.hpp:53-246)
int64_t deposit_normalized(const Mesh &m, const Shape &sf, const double *iw,
                           int64_t n, const double *x, const double *q,
                           const uint32_t *el, Target &tgt, DepStats &st) {
  const int np = m.nodes_per_element;
  std::vector<double> interp;
  std::vector<uint32_t> els;
  std::vector<double> scaled(np);
  int64_t zero_mass = -1;
  for (int64_t pn = 0; pn < n; ++pn) {
    interp.clear();
    els.clear();
    double integral = 0;
    auto add_shape_on_element = [&](const double *center, uint32_t en) {
      size_t start = (size_t)en * np;
      {
        const uint32_t *vv = m.element_vertices + 4 * (size_t)en;
        double c[3];
        for (int d = 0; d < 3; ++d) {
          c[d] = m.vertices[3 * vv[0] + d];
          for (int k = 1; k < 4; ++k) c[d] += m.vertices[3 * vv[k] + d];
          c[d] /= 4;
        }
        st.centroid.add(norm2_diff(c, center));
      }
      double el_integral = 0;
      for (int i = 0; i < np; ++i) {
        const double *node = m.nodes + 3 * (start + i);
        double d[3] = {node[0] - center[0], node[1] - center[1], node[2] - center[2]};
        double s = sf(d);
        interp.push_back(s);
        el_integral += s * iw[i];
      }
      integral += el_integral * m.jacobians[en];
      els.push_back(en);
    };
    std::unordered_set<uint32_t> el_set;
    walk(m, x + 3 * pn, sf.radius, el_set, el[pn], add_shape_on_element);
    st.el_per_particle.add((double)els.size());
    if (integral == 0) {
      if (zero_mass < 0) zero_mass = pn;
      continue;
    }
    const double scale = q[pn] / integral;
    st.norm.add(scale);
    tgt.begin_particle(pn);
    for (size_t k = 0; k < els.size(); ++k) {
      for (int i = 0; i < np; ++i) scaled[i] = scale * interp[k * np + i];
      tgt.add((size_t)els[k] * np, scaled.data(), np);
    }
  }
  return zero_mass;
}

// ------------------------------------------------------------ grid

struct Brick {
  double origin[3], h[3], oph[3];
  int dims[3];
  int64_t strides[3];
  int64_t start;
  // jiggly_brick (grid.hpp:345-449): three point origins, chosen per point
  // by (i + j + k) % 3
  bool jiggly;
  double po[3][3];
};

// `po`: the brick's three point origins ([3][3]) for a jiggly brick, or NULL
Brick make_brick(const prt_brick &b, const double *po = nullptr) {
  Brick r;
  for (int d = 0; d < 3; ++d) {
    r.origin[d] = b.origin[d];
    r.h[d] = b.stepwidths[d];
    r.dims[d] = b.dims[d];
    r.oph[d] = r.origin[d] + r.h[d] / 2;
  }
  r.strides[0] = 1;
  r.strides[1] = r.dims[0];
  r.strides[2] = (int64_t)r.dims[0] * r.dims[1];
  r.start = b.start_index;
  r.jiggly = po != nullptr;
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) r.po[i][d] = po ? po[3 * i + d] : 0.0;
  return r;
}

// jiggly_brick::point (grid.hpp:386-396): point_origins[(i+j+k) % 3] + idx h.
// The reference's jiggly iterator (grid.hpp:398-440) instead advances along x
// by the offset of the origin AFTER the next one (it bumps the origin index
// before choosing the offset), so its points along a row depend on where the
// row starts; this restatement, like the device path, uses point(idx).
void jiggly_point(const Brick &b, int i, int j, int k, double pt[3]) {
  const int oi = (i + j + k) % 3;
  const int idx[3] = {i, j, k};
  for (int d = 0; d < 3; ++d) pt[d] = b.po[oi][d] + idx[d] * b.h[d];
}

// grid_depositor::deposit_particle_on_one_brick (dep_grid.hpp:220-264) with
// the brick_iterator of grid.hpp:44-135 (incremental point along x).
template <class Add>
bool deposit_on_brick(const Brick &brk, const Shape &sf, const double *center,
                      const double *plo, const double *phi, double charge,
                      bool *complete, Add add) {
  double ilo[3], ihi[3];
  for (int d = 0; d < 3; ++d) {
    double blo = brk.origin[d], bhi = brk.origin[d] + brk.dims[d] * brk.h[d];
    ilo[d] = std::max(blo, plo[d]);
    ihi[d] = std::min(bhi, phi[d]);
  }
  if (complete) {
    bool eq = true;
    for (int d = 0; d < 3; ++d) eq = eq && ilo[d] == plo[d] && ihi[d] == phi[d];
    *complete = eq;
  }
  for (int d = 0; d < 3; ++d)
    if (ilo[d] >= ihi[d]) return false;
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = (int)std::floor((ilo[d] - brk.origin[d]) / brk.h[d]);
    hi[d] = (int)std::ceil((ihi[d] - brk.origin[d]) / brk.h[d]);
  }
  for (int d = 0; d < 3; ++d)
    if (lo[d] >= hi[d]) return true;
  for (int k = lo[2]; k < hi[2]; ++k)
    for (int j = lo[1]; j < hi[1]; ++j) {
      double pt[3] = {brk.oph[0] + lo[0] * brk.h[0], brk.oph[1] + j * brk.h[1],
                      brk.oph[2] + k * brk.h[2]};
      int64_t idx = brk.start + lo[0] + brk.strides[1] * j + brk.strides[2] * k;
      for (int i = lo[0]; i < hi[0]; ++i) {
        if (brk.jiggly) jiggly_point(brk, i, j, k, pt);
        double d[3] = {center[0] - pt[0], center[1] - pt[1], center[2] - pt[2]};
        add(idx, charge * sf(d));
        pt[0] += brk.h[0];
        idx += 1;
      }
    }
  return true;
}

// deposit_densities_on_grid_target + deposit_periodic_copies +
// deposit_single_particle_with/without_cache (dep_grid_base.hpp:210-382) for
// one particle at x: the particle box [x - a, x + a], then recursively its
// periodic copies, one per set of axes crossed (at most one image per axis:
// the lower end first). on_brick(brick, center, box_lo, box_hi, complete*)
// deposits on one brick and returns whether the box met it. `cache` (or
// NULL: every brick, no cache) is this particle's brick cache.
template <class OnBrick>
void deposit_periodic_copies(const prt_mesh_desc &m, const std::vector<Brick> &B,
                             double radius, const double *x, uint32_t *cache,
                             OnBrick &&on_brick) {
  std::vector<unsigned> pset;
  struct Frame {
    double c[3], lo[3], hi[3];
    unsigned abf;
  };
  auto go = [&](auto &&self, const Frame &f) -> void {
    if (f.abf == 0 && cache) {
      uint32_t &bn = *cache;
      bool complete;
      const bool hit_cached = on_brick(B[bn], f.c, f.lo, f.hi, &complete);
      if (!complete)
        for (size_t bi = 0; bi < B.size(); ++bi) {
          if (bi == bn) continue;
          if (on_brick(B[bi], f.c, f.lo, f.hi, nullptr) && !hit_cached) bn = (uint32_t)bi;
        }
    } else {
      for (const Brick &b : B) on_brick(b, f.c, f.lo, f.hi, nullptr);
    }
    pset.push_back(f.abf);
    for (int axis = 0; axis < 3; ++axis) {
      const double mn = m.periodicity_min[axis], mx = m.periodicity_max[axis];
      if (mn == mx) continue;
      const unsigned abf2 = f.abf | (1u << axis);
      if (std::find(pset.begin(), pset.end(), abf2) != pset.end()) continue;
      double off;
      if (f.lo[axis] < mn)
        off = mx - mn;
      else if (f.hi[axis] > mx)
        off = -(mx - mn);
      else
        continue;
      Frame g = f;
      g.c[axis] += off;
      g.lo[axis] += off;
      g.hi[axis] += off;
      g.abf = abf2;
      self(self, g);
    }
  };
  Frame f0;
  for (int d = 0; d < 3; ++d) {
    f0.c[d] = x[d];
    f0.lo[d] = x[d] - radius;
    f0.hi[d] = x[d] + radius;
  }
  f0.abf = 0;
  go(go, f0);
}

}  // namespace

// =================================================================== C ABI

extern "C" {

int orc_get_velocities(int64_t n, const double *p, const double *m, double c,
                       double *v) {
  get_velocities(n, p, m, c, v);
  return 0;
}

int orc_find_containing_elements(const prt_mesh_desc *m, int64_t n,
                                 const double *x, uint32_t *el, int linear) {
  prt_find_counters c = {0, 0, 0, 0};
  for (int64_t i = 0; i < n; ++i)
    el[i] = linear ? find_containing_element(*m, x + 3 * i)
                   : find_new_containing_element(*m, x + 3 * i, x + 3 * i,
                                                 INVALID, c, false);
  return 0;
}

// update_containing_elements with kills. On return *n is the surviving count;
// arrays are compacted by swap-with-last (ids/kx/kp follow when non-NULL).
int orc_update_containing_elements(const prt_mesh_desc *m, int64_t *n, double *x,
                                   double *p, double *q, double *mass,
                                   uint32_t *el, double *kx, double *kp,
                                   int64_t *ids, prt_find_counters *ctr,
                                   int linear_global) {
  Store s{*n, x, p, q, mass, el, kx, kp, ids};
  try {
    update_containing_elements(*m, s, *ctr, linear_global != 0);
  } catch (NoBestNormal &) {
    *n = s.n;
    return PRT_ERR_NO_BEST_NORMAL;
  }
  *n = s.n;
  return 0;
}

void *orc_pusher_create(int np, const uint32_t *exps, const double *vdm) {
  Pusher *P = new Pusher;
  P->np = np;
  P->exps.assign(exps, exps + 3 * np);
  // lu(V^T) with V^T stored column-major: (V^T)[i][k] = V[k][i] -> a[i + n k] = V[k][i]
  P->lu.resize((size_t)np * np);
  for (int i = 0; i < np; ++i)
    for (int k = 0; k < np; ++k) P->lu[i + (size_t)np * k] = vdm[(size_t)k * np + i];
  P->piv.resize(np);
  if (lu_factor(np, P->lu.data(), P->piv.data()) != 0) {
    delete P;
    return nullptr;
  }
  return P;
}

void orc_pusher_destroy(void *P) { delete (Pusher *)P; }

int orc_forces(void *P, const prt_mesh_desc *m, int64_t n, const double *x,
               const uint32_t *el, const double *q, const double *v,
               const double *ex, const double *ey, const double *ez,
               const double *bx, const double *by, const double *bz, double *out,
               double *vis) {
  const double *f[6] = {ex, ey, ez, bx, by, bz};
  forces(*(Pusher *)P, *m, n, x, el, q, v, f, out, vis);
  return 0;
}

// One LSRK step (5 stages of hedge's LSRK4 driven through PicMethod, see
// cloud.py:159-311 and 554-603): per stage v = velocities, F = forces,
// k = a k + dt f, (x, p) += b k, relocate with kills. kx, kp persist across
// calls (the stepper's residual). Returns 0 or a prt_status.
int orc_lsrk_steps(void *P, const prt_mesh_desc *m, int64_t *n, double *x,
                   double *p, double *q, double *mass, uint32_t *el, double *kx,
                   double *kp, int64_t *ids, const double *const *fields,
                   int nstages, const double *ca, const double *cb, double dt,
                   double c, int steps, prt_find_counters *ctr, int linear_global) {
  Pusher &pu = *(Pusher *)P;
  std::vector<double> v, F;
  for (int step = 0; step < steps; ++step)
    for (int s = 0; s < nstages; ++s) {
      int64_t cnt = *n;
      v.resize(3 * cnt);
      F.resize(3 * cnt);
      get_velocities(cnt, p, mass, c, v.data());
      forces(pu, *m, cnt, x, el, q, v.data(), fields, F.data(), nullptr);
      const double a = ca[s], b = cb[s];
      for (int64_t i = 0; i < 3 * cnt; ++i) {
        double t1 = a * kx[i];
        double t2 = dt * v[i];
        kx[i] = t1 + t2;
        t1 = a * kp[i];
        t2 = dt * F[i];
        kp[i] = t1 + t2;
      }
      for (int64_t i = 0; i < 3 * cnt; ++i) {
        x[i] = x[i] + b * kx[i];
        p[i] = p[i] + b * kp[i];
      }
      int rc = orc_update_containing_elements(m, n, x, p, q, mass, el, kx, kp, ids,
                                              ctr, linear_global);
      if (rc) return rc;
    }
  return 0;
}

// deposit_rho / deposit_j / deposit_densities for the shape depositors
// (dep_target.hpp:203-273). rho [Nn] / j [Nn][3] are zeroed first. For the
// normalised mode `stats` receives (count, mean, m2, min, max) x 3:
// normalization, centroid distance, elements per particle. Returns the first
// particle with zero mass, or -1.
int64_t orc_deposit_shape(const prt_mesh_desc *m, int mode, prt_shape_function shape,
                          const double *iw, int64_t n, const double *x,
                          const double *q, const double *v, const uint32_t *el,
                          double *rho, double *j, double *stats) {
  const size_t nn = (size_t)m->element_count * m->nodes_per_element;
  if (rho) std::memset(rho, 0, nn * sizeof(double));
  if (j) std::memset(j, 0, 3 * nn * sizeof(double));
  Target tgt{rho, j, v, {0, 0, 0}};
  Shape sf = make_shape(shape);
  if (mode == PRT_DEPOSIT_PLAIN) {
    deposit_plain(*m, sf, n, x, q, el, tgt);
    return -1;
  }
  DepStats st;
  int64_t zm = deposit_normalized(*m, sf, iw, n, x, q, el, tgt, st);
  if (stats) {
    const DepStats::W *w[3] = {&st.norm, &st.centroid, &st.el_per_particle};
    for (int k = 0; k < 3; ++k) {
      stats[5 * k + 0] = w[k]->count;
      stats[5 * k + 1] = w[k]->mean;
      stats[5 * k + 2] = w[k]->m2;
      stats[5 * k + 3] = w[k]->mn;
      stats[5 * k + 4] = w[k]->mx;
    }
  }
  return zm;
}

// Visits the elements of one particle's walk; out[k] = element, returns count.
int orc_walk_elements(const prt_mesh_desc *m, const double *pos, uint32_t start,
                      double radius, uint32_t *out, int cap) {
  std::unordered_set<uint32_t> el_set;
  int cnt = 0;
  auto vis = [&](const double *, uint32_t en) {
    if (cnt < cap) out[cnt] = en;
    ++cnt;
  };
  walk(*m, pos, radius, el_set, start, vis);
  return cnt;
}

// deposit_grid_rho / _j / _densities (dep_grid.hpp:441-501) through
// deposit_densities_on_grid_target (dep_grid_base.hpp:175-382) with the
// per-particle brick cache and periodic copies. weights: PRT_GRID_SHAPE or
// PRT_GRID_TRILINEAR. grid_rho [G], grid_j [G][3] are zeroed first.
int orc_deposit_grid(const prt_mesh_desc *m, int nbricks, const prt_brick *bricks,
                     const double *point_origins, int weights, prt_shape_function shape,
                     int64_t n, const double *x, const double *q, const double *v,
                     int64_t gnc, double *grid_rho, double *grid_j,
                     uint32_t *brick_cache) {
  if (grid_rho) std::memset(grid_rho, 0, gnc * sizeof(double));
  if (grid_j) std::memset(grid_j, 0, 3 * gnc * sizeof(double));
  std::vector<Brick> B;
  for (int i = 0; i < nbricks; ++i)
    B.push_back(make_brick(bricks[i], point_origins ? point_origins + 9 * i : nullptr));
  Shape sf = make_shape(shape);
  for (int64_t pn = 0; pn < n; ++pn) {
    const double *c0 = x + 3 * pn;
    double sfac[3] = {0, 0, 0};
    if (grid_j)
      for (int a = 0; a < 3; ++a) sfac[a] = v[3 * pn + a];
    auto add = [&](int64_t idx, double val) {
      if (grid_rho) grid_rho[idx] += val;
      if (grid_j)
        for (int a = 0; a < 3; ++a) grid_j[3 * idx + a] += sfac[a] * val;
    };
    if (weights == PRT_GRID_TRILINEAR) {
      // trilinear charge assignment onto the cell-centred points of the brick
      // containing the particle (no reference counterpart), clamped at the
      // brick edge so the weights always sum to one; value = q w / dV.
      for (const Brick &b : B) {
        bool inside = true;
        for (int d = 0; d < 3; ++d)
          inside = inside && c0[d] >= b.origin[d] &&
                   c0[d] < b.origin[d] + b.dims[d] * b.h[d];
        if (!inside) continue;
        int i0[3];
        double f[3];
        for (int d = 0; d < 3; ++d) {
          double u = (c0[d] - b.origin[d]) / b.h[d] - 0.5;
          double fl = std::floor(u);
          i0[d] = (int)fl;
          f[d] = u - fl;
        }
        const double dv = b.h[0] * b.h[1] * b.h[2];
        const double qv = q[pn] / dv;
        for (int dz = 0; dz < 2; ++dz)
          for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx) {
              int ii[3] = {i0[0] + dx, i0[1] + dy, i0[2] + dz};
              for (int d = 0; d < 3; ++d) ii[d] = std::min(std::max(ii[d], 0), b.dims[d] - 1);
              double w = (dx ? f[0] : 1 - f[0]) * (dy ? f[1] : 1 - f[1]) *
                         (dz ? f[2] : 1 - f[2]);
              int64_t idx = b.start + ii[0] + b.strides[1] * ii[1] + b.strides[2] * ii[2];
              add(idx, qv * w);
            }
        break;
      }
      continue;
    }
    auto on_brick = [&](const Brick &b, const double *center, const double *plo,
                        const double *phi, bool *complete) {
      return deposit_on_brick(b, sf, center, plo, phi, q[pn], complete, add);
    };
    deposit_periodic_copies(*m, B, sf.radius, c0, brick_cache ? brick_cache + pn : nullptr,
                            on_brick);
  }
  return 0;
}

// grid_find_depositor (dep_grid_find.hpp:33-184; node lists from
// grid_find.py:55-104): every particle (and each of its periodic copies,
// with the brick cache, dep_grid_base.hpp:175-382) walks the cells of
// index_range(brick box & particle box) of each brick and adds
// q S(center - node) to every mesh node in the cell's node list.
// cell_starts [G+1] / cell_nodes: the node numbers per global grid index.
// nodes [Nn][3]; rho [Nn] and j [Nn][3] are zeroed first.
int orc_deposit_grid_find(const prt_mesh_desc *m, int nbricks, const prt_brick *bricks,
                          const uint32_t *cell_starts, const uint32_t *cell_nodes,
                          const double *nodes, int64_t nn, prt_shape_function shape,
                          int64_t n, const double *x, const double *q, const double *v,
                          double *rho, double *j, uint32_t *brick_cache) {
  if (rho) std::memset(rho, 0, nn * sizeof(double));
  if (j) std::memset(j, 0, 3 * nn * sizeof(double));
  std::vector<Brick> B;
  for (int i = 0; i < nbricks; ++i) B.push_back(make_brick(bricks[i]));
  Shape sf = make_shape(shape);
  for (int64_t pn = 0; pn < n; ++pn) {
    double sfac[3] = {0, 0, 0};
    if (j)
      for (int a = 0; a < 3; ++a) sfac[a] = v[3 * pn + a];
    // deposit_particle_on_one_brick (dep_grid_find.hpp:73-112)
    auto on_brick = [&](const Brick &brk, const double *center, const double *plo,
                        const double *phi, bool *complete) {
      double ilo[3], ihi[3];
      for (int d = 0; d < 3; ++d) {
        ilo[d] = std::max(brk.origin[d], plo[d]);
        ihi[d] = std::min(brk.origin[d] + brk.dims[d] * brk.h[d], phi[d]);
      }
      if (complete) {
        bool eq = true;
        for (int d = 0; d < 3; ++d) eq = eq && ilo[d] == plo[d] && ihi[d] == phi[d];
        *complete = eq;
      }
      for (int d = 0; d < 3; ++d)
        if (ilo[d] >= ihi[d]) return false;
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d) {
        // brick::index_range (grid.hpp:323-331); the clamp only guards the
        // arrays against a quotient that rounds past the brick's last cell
        lo[d] = std::max(0, (int)std::floor((ilo[d] - brk.origin[d]) / brk.h[d]));
        hi[d] = std::min(brk.dims[d], (int)std::ceil((ihi[d] - brk.origin[d]) / brk.h[d]));
      }
      for (int k = lo[2]; k < hi[2]; ++k)
        for (int jj = lo[1]; jj < hi[1]; ++jj)
          for (int i = lo[0]; i < hi[0]; ++i) {
            const int64_t g = brk.start + i + brk.strides[1] * jj + brk.strides[2] * k;
            for (uint32_t t = cell_starts[g]; t < cell_starts[g + 1]; ++t) {
              const uint32_t node = cell_nodes[t];
              const double d[3] = {center[0] - nodes[3 * (size_t)node],
                                   center[1] - nodes[3 * (size_t)node + 1],
                                   center[2] - nodes[3 * (size_t)node + 2]};
              const double val = q[pn] * sf(d);
              if (rho) rho[node] += val;
              if (j)
                for (int a = 0; a < 3; ++a) j[3 * (size_t)node + a] += sfac[a] * val;
            }
          }
      return true;
    };
    deposit_periodic_copies(*m, B, sf.radius, x + 3 * pn,
                            brick_cache ? brick_cache + pn : nullptr, on_brick);
  }
  return 0;
}

// remap_grid_to_mesh (dep_grid.hpp:270-358): gemv('N', alpha=1, beta=1) in
// reference-BLAS column order, then the average-group pass.
int orc_remap_grid_to_mesh(const prt_grid_desc *g, const double *from, double *to,
                           int64_t offset, int64_t increment) {
  const int np = g->nodes_per_element;
  std::vector<double> gv;
  for (int64_t e = 0; e < g->eog_count; ++e) {
    uint64_t s = g->eog_starts[e], t = g->eog_starts[e + 1];
    int cnt = (int)(t - s);
    gv.resize(cnt);
    bool had_nonzero = false;
    for (int i = 0; i < cnt; ++i) {
      double w = g->eog_weights[s + i] * from[offset + (int64_t)g->eog_grid_nodes[s + i] * increment];
      gv[i] = w;
      if (w) had_nonzero = true;
    }
    if (!had_nonzero) continue;
    const double *M = g->eog_matrices + g->eog_matrix_starts[e];
    double *y = to + (int64_t)g->eog_elements[e] * np * increment + offset;
    for (int k = 0; k < cnt; ++k) {
      double temp = gv[k];
      if (temp != 0)
        for (int i = 0; i < np; ++i) y[i * increment] += temp * M[i + (size_t)np * k];
    }
  }
  for (int64_t a = 0; a < g->avg_group_count; ++a) {
    uint32_t s = g->avg_group_starts[a], t = g->avg_group_starts[a + 1];
    if (s == t) continue;
    double avg = 0;
    for (uint32_t i = s; i < t; ++i) avg += to[offset + (int64_t)g->avg_group_nodes[i] * increment];
    avg /= (t - s);
    for (uint32_t i = s; i < t; ++i) to[offset + (int64_t)g->avg_group_nodes[i] * increment] = avg;
  }
  return 0;
}

// ---------------------------------------------------- multi-core baseline
//
// The same algorithms, particle-parallel over `threads` host threads, for
// timing the CPU baseline: locate and push are independent per particle;
// kills are marked (element = INVALID) instead of compacted; deposition
// accumulates per-thread partial sums of rho/j over contiguous node ranges.

int orc_pic_steps_parallel(void *P, const prt_mesh_desc *m, int64_t n, double *x,
                           double *p, const double *q, const double *mass,
                           uint32_t *el, double *kx, double *kp,
                           const double *const *fields, int nstages,
                           const double *ca, const double *cb, double dt, double c,
                           int steps, prt_shape_function shape, double *rho,
                           double *j, int threads) {
  Pusher &pu = *(Pusher *)P;
  Shape sf = make_shape(shape);
  const int np = m->nodes_per_element;
  const size_t nn = (size_t)m->element_count * np;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  int err = 0;
  for (int step = 0; step < steps; ++step) {
    for (int s = 0; s < nstages; ++s) {
      const double a = ca[s], b = cb[s];
#pragma omp parallel for schedule(static, 4096)
      for (int64_t i = 0; i < n; ++i) {
        if (el[i] == INVALID) continue;
        double v[3], F[3];
        get_velocities(1, p + 3 * i, mass + i, c, v);
        forces(pu, *m, 1, x + 3 * i, el + i, q + i, v, fields, F, nullptr);
        for (int d = 0; d < 3; ++d) {
          kx[3 * i + d] = a * kx[3 * i + d] + dt * v[d];
          kp[3 * i + d] = a * kp[3 * i + d] + dt * F[d];
          x[3 * i + d] = x[3 * i + d] + b * kx[3 * i + d];
          p[3 * i + d] = p[3 * i + d] + b * kp[3 * i + d];
        }
        prt_find_counters ctr = {0, 0, 0, 0};
        try {
          uint32_t ne = find_new_containing_element(*m, x + 3 * i, p + 3 * i, el[i],
                                                    ctr, false);
          if (ne == INVALID) {
            double qq = q[i], mm = mass[i];
            Store st{1, x + 3 * i, p + 3 * i, &qq, &mm, el + i, nullptr, nullptr, nullptr};
            if (!boundary_hit(*m, st, 0, ctr, false)) el[i] = INVALID;
          } else {
            el[i] = ne;
          }
        } catch (NoBestNormal &) {
#pragma omp atomic write
          err = PRT_ERR_NO_BEST_NORMAL;
        }
      }
      if (err) return err;
    }
    // deposit rho and j. Phase 1: walk every particle (parallel over
    // particles) and record (element, particle, centre) pairs. Phase 2: each
    // thread owns a contiguous element range and accumulates its pairs in
    // (element, particle) order, so no two threads write the same node.
    struct Pair {
      uint32_t en;
      uint32_t pn;
      double c[3];
    };
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    std::vector<std::vector<Pair>> tl(nt);
    std::vector<double> vel(3 * (size_t)n);
#pragma omp parallel
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
#pragma omp for schedule(dynamic, 64)
      for (int64_t pn = 0; pn < n; ++pn) {
        if (el[pn] == INVALID) continue;
        get_velocities(1, p + 3 * pn, mass + pn, c, vel.data() + 3 * pn);
        auto rec = [&](const double *center, uint32_t en) {
          tl[tid].push_back(Pair{en, (uint32_t)pn, {center[0], center[1], center[2]}});
        };
        std::unordered_set<uint32_t> el_set;
        walk(*m, x + 3 * pn, sf.radius, el_set, el[pn], rec);
      }
    }
    std::memset(rho, 0, nn * sizeof(double));
    std::memset(j, 0, 3 * nn * sizeof(double));
#pragma omp parallel
    {
      int tid = 0, ntt = 1;
#ifdef _OPENMP
      tid = omp_get_thread_num();
      ntt = omp_get_num_threads();
#endif
      const int64_t e0 = m->element_count * tid / ntt;
      const int64_t e1 = m->element_count * (tid + 1) / ntt;
      std::vector<Pair> mine;
      for (auto &v : tl)
        for (auto &pr : v)
          if ((int64_t)pr.en >= e0 && (int64_t)pr.en < e1) mine.push_back(pr);
      std::sort(mine.begin(), mine.end(), [](const Pair &a, const Pair &b) {
        return a.en != b.en ? a.en < b.en : a.pn < b.pn;
      });
      for (const Pair &pr : mine) {
        const double charge = q[pr.pn];
        const double *vv = vel.data() + 3 * (size_t)pr.pn;
        size_t start = (size_t)pr.en * np;
        for (int i = 0; i < np; ++i) {
          const double *node = m->nodes + 3 * (start + i);
          double d[3] = {node[0] - pr.c[0], node[1] - pr.c[1], node[2] - pr.c[2]};
          double r = charge * sf(d);
          rho[start + i] += r;
          for (int ax = 0; ax < 3; ++ax) j[(start + i) * 3 + ax] += vv[ax] * r;
        }
      }
    }
  }
  return 0;
}

int orc_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
