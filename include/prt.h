/*
 * prt.h -- C ABI of libprt.so, the B200 particle side of a pyrticle PIC step.
 *
 * The reference exposes this path through one Boost.Python module,
 * pyrticle._internal (src/wrapper/wrap_main.cpp:43-57). Each entry point below
 * names the reference interface it replaces. Conventions:
 *
 *   - every function returns int: PRT_OK (0) or a negative prt_status;
 *   - particle vectors are device pointers in SoA layout: a 3-vector array is
 *     [3][n] (component c of particle i at c*n + i); scalars are [n];
 *   - node vectors are device pointers: rho [Nn], j [3][Nn] (the [vdim, Nn]
 *     C-order layout PicMethod.deposit_j returns, pyrticle/cloud.py:535-538);
 *   - element e owns nodes [e*Np, (e+1)*Np) (push_monomial.hpp:104-110);
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *   - errors found on the device (the reference throws or warns there) are
 *     recorded in the workspace status word and read by prt_workspace_status.
 *
 * No function here allocates device memory per call except the ones that
 * take a prt_workspace, which grows its own scratch on demand.
 */
#ifndef PRT_H_INCLUDED
#define PRT_H_INCLUDED

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRT_INVALID_ELEMENT 0xffffffffu /* hedge::INVALID_ELEMENT */
#define PRT_INVALID_AXIS 0xffffffffu    /* mesh_data::INVALID_AXIS, meshdata.hpp:68 */

enum prt_status {
  PRT_OK = 0,
  PRT_ERR_INVALID_ARGUMENT = -1,
  PRT_ERR_CUDA = -2,
  PRT_ERR_OUT_OF_MEMORY = -3,
  /* "no best normal found--weird" (particle_state.hpp:176-189) */
  PRT_ERR_NO_BEST_NORMAL = -4,
  /* a particle handed to a kernel has no containing element */
  PRT_ERR_NOT_LOCATED = -5,
  /* scratch larger than a fixed-capacity entry point supports */
  PRT_ERR_CAPACITY = -6,
  /* a kernel's bounded wait on its own tensor-core work ran out */
  PRT_ERR_TIMEOUT = -7
};

/* Warnings recorded in the status word (the reference WARNs, tools.hpp:467-508). */
enum prt_warning {
  PRT_WARN_NONE = 0,
  /* "deposited particle mass is zero" (dep_normshape.hpp:179-185) */
  PRT_WARN_ZERO_MASS = 1,
  /* "average pusher: particle %d had zero reconstructed charge"
   * (push_average.hpp:161-166) */
  PRT_WARN_ZERO_AVERAGE = 2
};

/* ---------------------------------------------------------------- mesh --- */

/* Host-side description of mesh_data (meshdata.hpp:53-124), as filled by
 * MeshData.fill_from_hedge (pyrticle/meshdata.py:37-133). All pointers are
 * HOST pointers; prt_mesh_create copies them to the device. */
typedef struct prt_mesh_desc {
  int64_t element_count;            /* E */
  int64_t vertex_count;             /* V */
  int32_t nodes_per_element;        /* Np */
  int32_t reserved0;
  const double *vertices;           /* [V][3] */
  const uint32_t *element_vertices; /* [E][4] */
  const double *inverse_maps;       /* [E][12]: row-major A (3x3), then b (3) */
  const double *jacobians;          /* [E] |det| of the unit->element map */
  const double *face_normals;       /* [E][4][3] outward unit normals */
  const double *face_plane_rhs;     /* [E][4] n . x on the face */
  const double *face_centroids;     /* [E][4][3] */
  const double *face_radii;         /* [E][4] bounding-circle radius */
  const uint32_t *face_neighbors;   /* [E][4] or PRT_INVALID_ELEMENT */
  const uint32_t *face_periodicity_axes; /* [E][4] or PRT_INVALID_AXIS */
  const uint32_t *vertex_adj_starts;     /* [V+1] */
  const uint32_t *vertex_adj_elements;   /* ascending element id per vertex */
  double periodicity_min[3];        /* min == max: axis not periodic */
  double periodicity_max[3];
  const double *nodes;              /* [E*Np][3] node coordinates */
  /* element bins for the global search (meshdata.hpp:208-215): bin b lists,
   * ascending, every element whose bounding box overlaps it */
  double bin_origin[3];
  double bin_inv_width[3];
  int32_t bin_dims[3];
  int32_t reserved1;
  const uint32_t *bin_starts;       /* [bins+1] */
  const uint32_t *bin_elements;
} prt_mesh_desc;

typedef struct prt_mesh prt_mesh;

/* Replaces MeshData(dim) + fill_from_hedge (wrap_meshdata.cpp:50-114). */
int prt_mesh_create(const prt_mesh_desc *desc, prt_mesh **out);
int prt_mesh_destroy(prt_mesh *mesh);

/* ----------------------------------------------------------- workspace --- */

typedef struct prt_workspace prt_workspace;

int prt_workspace_create(prt_workspace **out);
int prt_workspace_destroy(prt_workspace *ws);
/* Synchronises `stream`, returns the first recorded device error (or PRT_OK)
 * with the particle index that raised it, and the first warning; clears both
 * when `clear` is nonzero. */
int prt_workspace_status(prt_workspace *ws, void *stream, int32_t *error,
                         int64_t *error_index, int32_t *warning,
                         int64_t *warning_index, int32_t clear);

/* Find-path event counters (particle_state.hpp:86-92, cloud.py:366-377). */
typedef struct prt_find_counters {
  uint64_t find_same;
  uint64_t find_by_neighbor;
  uint64_t find_by_vertex;
  uint64_t find_global;
} prt_find_counters;

/* Copies the workspace's device counters to *out (synchronising `stream`)
 * and zeroes them when `reset` is nonzero. */
int prt_workspace_counters(prt_workspace *ws, void *stream,
                           prt_find_counters *out, int32_t reset);

/* Kernel timing (measurement hook; no reference counterpart). When enabled,
 * the library brackets its main kernels with CUDA events on the launch
 * stream; prt_workspace_timing_read sums the elapsed times per category
 * (synchronising) and optionally resets them. */
enum prt_timing_category {
  PRT_TIME_DEPOSIT_GATHER = 0, /* node-centric deposition kernel */
  PRT_TIME_DEPOSIT_STAGE = 1,  /* particle binning, sort and packing */
  PRT_TIME_LSRK_STAGE = 2,     /* fused RK stage kernel */
  PRT_TIME_SORT = 3,           /* prt_sort_by_element */
  PRT_TIME_STAGE_ADJOINT = 4,  /* prt_lsrk_stage_adjoint kernel */
  PRT_TIME_DEPOSIT_ADJOINT = 5,/* prt_deposit_shape_adjoint */
  PRT_TIME_DEPOSIT_NORMALIZE = 6,/* normalising integrals of the tensor-core deposition */
  PRT_TIME_CATEGORIES = 7
};
int prt_workspace_timing(prt_workspace *ws, int32_t enable);
int prt_workspace_timing_read(prt_workspace *ws, int32_t category,
                              double *total_ms, int64_t *launches,
                              int32_t reset);

/* ---------------------------------------------------------- kinematics --- */

/* Replaces get_velocities(ps, c) (particle_state.hpp:98-125,
 * wrap_pic.cpp:71): v = c p / sqrt(m^2 c^2 + |p|^2), zero for p = 0. */
int prt_get_velocities(int64_t n, const double *momenta, const double *masses,
                       double vacuum_c, double *velocities, void *stream);

/* Replaces MeshData.find_containing_element(pt) (meshdata.hpp:208-215) used by
 * PicMethod.add_particles (cloud.py:470): the lowest-id element whose inverse
 * map passes is_in_unit_simplex, or PRT_INVALID_ELEMENT. */
int prt_find_containing_elements(const prt_mesh *mesh, int64_t n,
                                 const double *positions, uint32_t *elements,
                                 void *stream);

/* Replaces update_containing_elements(mesh, ps, bhit_listener, counters)
 * (particle_state.hpp:266-357, wrap_pic.cpp:73). A particle that is found
 * nowhere, even after the periodic wrap, gets PRT_INVALID_ELEMENT: the
 * caller removes it (the reference kills it through the boundary-hit
 * listener, cloud.py:581-585). Particles that already carry
 * PRT_INVALID_ELEMENT are skipped. Counters accumulate in `ws`. */
int prt_update_containing_elements(const prt_mesh *mesh, prt_workspace *ws,
                                   int64_t n, double *positions,
                                   const double *momenta, uint32_t *elements,
                                   void *stream);

/* ------------------------------------------------------ monomial pusher --- */

typedef struct prt_pusher prt_pusher;

/* Replaces MonomialPusher3d3v(mesh) + LocalMonomialDiscretization set-up
 * (pusher.py:86-114, push_monomial.hpp:45-80): `exponents` [Np][3] are the
 * monomial exponents, `vandermonde` [Np][Np] row-major is V[i][k] =
 * monomial_k(unit_node_i). */
int prt_monomial_pusher_create(const prt_mesh *mesh, int32_t np,
                               const uint32_t *exponents,
                               const double *vandermonde, prt_pusher **out);
int prt_monomial_pusher_destroy(prt_pusher *pusher);

/* Replaces MonomialPusher3d3v.forces(ex, ey, ez, bx, by, bz, ps, velocities,
 * vis_listener) (push_monomial.hpp:219-325, wrap_pusher.cpp:160-165):
 * forces[3][n] = q E(x) + v x (q B(x)). fields[k] is a device [Nn] array or
 * NULL for a zero component. vis, if not NULL, receives [4][3][n]: pt_e, pt_b,
 * el_force, mag_force (the verbose_vis vectors, push_monomial.hpp:307-322).
 * Particles with element PRT_INVALID_ELEMENT get zero force. */
int prt_forces(const prt_pusher *pusher, int64_t n, const double *positions,
               const uint32_t *elements, const double *charges,
               const double *velocities, const double *const fields[6],
               double *forces, double *vis, void *stream);

/* One low-storage Runge-Kutta stage of the particle ODE, fused:
 *   f = (v(p), F(x, p)),  k = a k + dt f,  (x, p) += b k,  relocate.
 * This is PicMethod.advance_state (cloud.py:554-603) driven by the 2N-storage
 * RK update through TimesteppablePicState.__add__ (cloud.py:172-186), with the
 * force of prt_forces and the relocation of prt_update_containing_elements.
 * kx, kp are the [3][n] residuals; dead particles (PRT_INVALID_ELEMENT) are
 * left untouched. `precision` 0 = FP64 plain form. */
int prt_lsrk_stage(const prt_pusher *pusher, prt_workspace *ws, int64_t n,
                   double *positions, double *momenta, const double *charges,
                   const double *masses, uint32_t *elements, double *kx,
                   double *kp, const double *const fields[6], double rk_a,
                   double rk_b, double dt, double vacuum_c, int32_t precision,
                   void *stream);

/* ----------------------------------------------------------- deposition --- */

/* polynomial_shape_function(radius, dimensions, alpha) (tools.hpp:514-556,
 * tools.cpp:43-58): S(r) = normalizer * (radius - r^2/radius)^alpha inside
 * the radius, 0 outside. */
typedef struct prt_shape_function {
  double radius;
  double alpha;
  double normalizer;
} prt_shape_function;

/* Arithmetic of a call (`precision` arguments). */
enum prt_precision {
  PRT_PRECISION_FP64 = 0,  /* plain form: FP64 throughout */
  /* chosen form. Stage: Lagrange values on the tensor cores (split BF16,
   * FP32 accumulation), force, update and locate in FP64. Deposition (shape
   * exponent 2): the weight max(1 - r^2/a^2, 0)^2 from a split-FP16
   * tensor-core product with FP32 accumulation, rounded to a 23-bit integer,
   * and summed exactly on the integer tensor cores against charges scaled to
   * integers below 2^46 (currents below 2^22), combined into FP64 per node;
   * the normalising integral per particle is summed exactly from the same
   * integer weights, so deposited charge matches the particles' charge to
   * FP64 rounding. Other exponents: as PRT_PRECISION_MIXED_SIMT. */
  PRT_PRECISION_MIXED = 1,
  /* deposition weights and per-batch sums in FP32 on the CUDA cores,
   * combined into FP64 per node (deposition only) */
  PRT_PRECISION_MIXED_SIMT = 2
};

enum prt_deposit_mode {
  PRT_DEPOSIT_PLAIN = 0,      /* ShapeFunctionDepositor (dep_shape.hpp) */
  PRT_DEPOSIT_NORMALIZED = 1  /* NormalizedShapeFunctionDepositor (dep_normshape.hpp) */
};

/* Per-call statistics of the normalising depositor (dep_normshape.hpp:42-47):
 * count / sum / sum of squares / min / max of the applied scale q / integral
 * and of the number of elements each particle reaches. */
typedef struct prt_deposit_stats {
  double norm_count, norm_sum, norm_sum_sq, norm_min, norm_max;
  double el_count, el_sum, el_sum_sq, el_min, el_max;
  /* (particle, position) pairs within the radius, over distinct node
   * positions (what the device evaluates: coincident DG nodes share one) */
  double pair_count;
  /* (particle, node) pairs within the radius, over all DG nodes */
  double node_pair_count;
  /* (particle, position) pairs the kernel evaluated (after culling) */
  double evaluated_pairs;
} prt_deposit_stats;

/* Replaces deposit_rho / deposit_j / deposit_densities(dep, ds, ps,
 * node_count, [velocities,] slice) for InterpolatingDepositor3d3v and
 * NormalizingInterpolatingDepositor3d3v (dep_target.hpp:203-273,
 * wrap_depositor.cpp:44-50):
 *   rho[n]    = sum_p w_p S(x_n - x_p),  j[c][n] = sum_p w_p v_p[c] S(x_n - x_p)
 * with w_p = q_p (plain) or q_p / (sum_e |J_e| sum_i w_i S(x_i - x_p))
 * (normalised, `integral_weights` [Np] = M 1, a HOST array). rho or j may
 * be NULL. The sum is deterministic: no floating-point atomics, fixed order.
 * Coincident DG nodes (shared faces, edges, vertices) are evaluated once and
 * receive the same values. For the normalising mode the statistics count, per
 * particle, the node positions within the radius (the reference counts the
 * elements its walk visits, dep_normshape.hpp:176-177).
 * Particles with element PRT_INVALID_ELEMENT are skipped. When `stats` is
 * not NULL the call also counts the (particle, node) pairs inside the
 * radius, and synchronises `stream`. */
int prt_deposit_shape(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                      prt_shape_function shape, const double *integral_weights,
                      int64_t n, const double *positions, const double *charges,
                      const double *velocities, const uint32_t *elements,
                      double *rho, double *j, int32_t precision,
                      prt_deposit_stats *stats, void *stream);

/* Scratch capacity of prt_deposit_shape_noalloc, in bytes, per device. */
#define PRT_NOALLOC_SCRATCH_BYTES (64u << 20)

/* No counterpart in the reference: the plain-form deposition of
 * prt_deposit_shape (mode PRT_DEPOSIT_PLAIN, FP64; the same sums in another
 * order, so the results agree to rounding, about 1e-15 relative, not
 * bitwise) for callers that must not
 * allocate device memory while they run -- code with a fixed, pre-reserved
 * memory budget, real-time loops where an allocation would stall or
 * synchronise the device, or hosts that forbid it. It calls no cudaMalloc,
 * cudaFree or allocating library routine and takes no workspace: all scratch
 * comes from one file-scope device array of PRT_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit. Inputs and outputs are the
 * caller's, as for prt_deposit_shape; rho or j may be NULL.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) and caches it; make that first call before any
 *    stream capture. The cache lives as long as the process: after a
 *    cudaDeviceReset the address is stale, so do not call this entry point
 *    on a device that was reset.
 *  - With rho and j both NULL the call does nothing.
 *  - A call whose scratch (about 84 bytes per particle + 32 bytes per
 *    distinct node position + bins + radix-sort storage) exceeds the
 *    capacity returns PRT_ERR_CAPACITY before touching any pointer.
 *  - All calls share the one array and each leaves its contents behind (no
 *    region needs clearing: every one is written before it is read); calls
 *    that overlap on the GPU (other streams, other host threads) race, so
 *    serialise them. */
int prt_deposit_shape_noalloc(const prt_mesh *mesh, prt_shape_function shape,
                              int64_t n, const double *positions,
                              const double *charges, const double *velocities,
                              const uint32_t *elements, double *rho, double *j,
                              void *stream);

/* Sharded form of the chosen-form deposition (PRT_PRECISION_MIXED, shape
 * exponent 2) for one process per GPU. No reference counterpart: the
 * reference is a single process; its deposition is a sum over particles
 * (dep_target.hpp:203-273), which these three steps split by particle. Every
 * rank holds the mesh and deposits its own particles:
 *  1. prt_deposit_shape_charges: bins the rank's particles and, in the
 *     normalising mode, integrates each one's shape over all node positions
 *     (the mesh is replicated, so this needs no exchange); writes the maxima
 *     of |c|, |c vx|, |c vy|, |c vz| over the rank's particles to
 *     `local_max` (device, [4]); c = q (plain) or q / integral;
 *  -- the caller all-reduces the four maxima with MAX --
 *  2. prt_deposit_shape_sums: the deposition pass with the digits scaled by
 *     the global maxima, writing per distinct node position the 16 digit
 *     sums (device [16][npos], npos from prt_mesh_position_count); every
 *     value is an integer below 2^45 held in an FP64;
 *  -- the caller all-reduces the sums with SUM: integers below 2^53 add
 *     exactly in any order --
 *  3. prt_deposit_shape_combine: rho [Nn] and j [3][Nn] (either may be NULL)
 *     from the summed digit sums and the global maxima.
 * rho and j are then bitwise the same for any number of ranks and any split
 * of the particles, and equal to prt_deposit_shape's with every particle on
 * one GPU. Steps 1 and 2 share workspace state: call them with the same
 * workspace, mesh, shape and n, with no other deposition in between.
 * `stats` (step 1, may be NULL) as prt_deposit_shape's, for the rank's
 * particles; it synchronises `stream`. */
int prt_mesh_position_count(const prt_mesh *mesh, int64_t *count);
int prt_deposit_shape_charges(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                              prt_shape_function shape, const double *integral_weights,
                              int64_t n, const double *positions, const double *charges,
                              const double *velocities, const uint32_t *elements,
                              double *local_max, prt_deposit_stats *stats, void *stream);
int prt_deposit_shape_sums(const prt_mesh *mesh, prt_workspace *ws, prt_shape_function shape,
                           int64_t n, const double *global_max, double *sums, void *stream);
int prt_deposit_shape_combine(const prt_mesh *mesh, prt_workspace *ws,
                              prt_shape_function shape, const double *global_max,
                              const double *sums, double *rho, double *j, void *stream);

/* ------------------------------------------------------------ grid dep --- */

/* One brick (grid.hpp:159-340): cell-centred points origin + (idx + 1/2) h,
 * global index start_index + idx . strides with x fastest. */
typedef struct prt_brick {
  double origin[3];
  double stepwidths[3];
  int32_t dims[3];
  int32_t reserved;
  int64_t start_index;
} prt_brick;

enum prt_grid_weights {
  PRT_GRID_SHAPE = 0,     /* q S(x - pt) at brick points (dep_grid.hpp:220-264) */
  PRT_GRID_TRILINEAR = 1  /* q * trilinear weights on the 8 surrounding points */
};

typedef struct prt_grid prt_grid;

/* Replaces RegularGridDepositor3d3v(mesh) with .bricks and .elements_on_grid
 * filled (wrap_depositor.cpp:66-102, grid.py:71-117): per element-on-grid,
 * its element number, grid node list, weight factors and the Np x |G|
 * column-major interpolation matrix. Average groups (dep_grid.hpp:108-117) are
 * given as CSR; avg_group_count = 0 disables continuity enforcement. */
typedef struct prt_grid_desc {
  int32_t brick_count;
  int32_t nodes_per_element;
  const prt_brick *bricks;
  int64_t eog_count;
  const uint32_t *eog_elements;     /* [eog_count] */
  const uint64_t *eog_starts;       /* [eog_count+1] offsets into nodes/weights */
  const uint32_t *eog_grid_nodes;   /* [total] */
  const double *eog_weights;        /* [total] */
  const uint64_t *eog_matrix_starts;/* [eog_count+1] offsets into matrices */
  const double *eog_matrices;       /* column-major Np x |G_e| each */
  int64_t avg_group_count;
  const uint32_t *avg_group_starts; /* [avg_group_count+1] */
  const uint32_t *avg_group_nodes;
  /* Jiggly bricks (JigglyBrick, grid.hpp:345-449): NULL for regular
   * cell-centred points, else [brick_count][3][3], per brick its three point
   * origins; point idx of brick b is point_origins[b][(i + j + k) % 3] +
   * idx * stepwidths. Every offset must stay within half a cell. Shape
   * weights only (PRT_GRID_TRILINEAR is rejected). */
  const double *point_origins;
} prt_grid_desc;

int prt_grid_create(const prt_mesh *mesh, const prt_grid_desc *desc,
                    prt_grid **out);
int prt_grid_destroy(prt_grid *grid);

/* Replaces deposit_grid_rho / deposit_grid_j / deposit_grid_densities
 * (dep_grid.hpp:441-501) including periodic copies (dep_grid_base.hpp:285-347).
 * grid_rho [G] and grid_j [3][G] (either may be NULL). Deterministic. */
int prt_deposit_grid(const prt_grid *grid, prt_workspace *ws, int32_t weights,
                     prt_shape_function shape, int64_t n,
                     const double *positions, const double *charges,
                     const double *velocities, const uint32_t *elements,
                     double *grid_rho, double *grid_j, void *stream);

/* Replaces remap_grid_to_mesh(from, to, offset, increment)
 * (dep_grid.hpp:270-358): for every element-on-grid,
 * to[(start + i)*increment + offset] += sum_k I[i,k] w_k from[offset + g_k*increment]
 * followed by the average-group continuity pass. `to` is accumulated into. */
int prt_remap_grid_to_mesh(const prt_grid *grid, const double *from,
                           double *to, int64_t offset, int64_t increment,
                           void *stream);

/* The shape-weight grid deposition of the chosen (mixed) form, on the tensor
 * cores: the sums of prt_deposit_grid(PRT_GRID_SHAPE) (dep_grid.hpp:220-264)
 * within ~1e-7 relative, from split-FP16 score MMAs, 23-bit integer weights
 * and exact int8 MMA sums (the tensor-core form of prt_deposit_shape). Needs
 * alpha = 2 and bricks numbered contiguously; the grid's points are uploaded
 * on the first call (24 B per point). Same outputs as prt_deposit_grid. */
int prt_deposit_grid_mixed(const prt_grid *grid, prt_workspace *ws,
                           prt_shape_function shape, int64_t n, const double *x,
                           const double *q, const double *v, const uint32_t *el,
                           double *grid_rho, double *grid_j, void *stream);

/* The remap of 1-4 components at once: from [components][grid nodes] to
 * [components][DG nodes] (added into `to`, like prt_remap_grid_to_mesh per
 * component), each element's matrix read once for all components. Same
 * values as `components` calls of prt_remap_grid_to_mesh. No reference
 * counterpart (the reference remaps one component per call). */
int prt_remap_grid_to_mesh_components(const prt_grid *grid, const double *from,
                                      double *to, int32_t components,
                                      void *stream);

/* ------------------------------------------------- adjoint (reverse mode) ---
 * No reference counterpart: the reference computes no derivatives. These
 * differentiate prt_lsrk_stage, prt_get_velocities and prt_deposit_shape
 * (plain mode) exactly, with every stage's containing element held fixed.
 * The caller records the stage inputs (prt_lsrk_stage_record) and runs the
 * adjoints in reverse order; checkpointing is the caller's choice. */

#define PRT_MAX_FIELD_BASIS 4

/* prt_lsrk_stage writing the updated state to separate arrays: reads
 * (x_in, p_in, el_in), writes (x_out, p_out, el_out) (dead particles are
 * copied), updates kx, kp in place. Outputs must not alias the inputs. The
 * arithmetic is prt_lsrk_stage's, so a recorded run is bitwise identical to
 * an in-place one. */
int prt_lsrk_stage_record(const prt_pusher *pusher, prt_workspace *ws, int64_t n,
                          const double *x_in, const double *p_in,
                          const uint32_t *el_in, double *x_out, double *p_out,
                          uint32_t *el_out, const double *charges,
                          const double *masses, double *kx, double *kp,
                          const double *const fields[6], double rk_a, double rk_b,
                          double dt, double vacuum_c, void *stream);

/* Per-element monomial coefficients of nodal fields: for each of `count`
 * device [Nn] arrays fields[k] (NULL entries skipped), coefficients[k]
 * [E][Np] with f(r) = sum_j c_j monomial_j(r) on each element (canonical
 * monomial order). The stage adjoint takes its fields in this form. */
int prt_fields_to_monomial(const prt_pusher *pusher, int32_t count,
                           const double *const *fields, double *const *coefficients,
                           void *stream);

/* Adjoint of one prt_lsrk_stage. positions, momenta, elements: the stage's
 * INPUT state. field_coefficients[6] and the basis: monomial coefficients
 * (prt_fields_to_monomial) of the stage's fields and of the basis fields.
 * lam_x, lam_p, lam_kx, lam_kp [3][n]: on entry the adjoints of
 * the stage's outputs, on exit those of its inputs. grad_fields: NULL, or six
 * device [Nn] arrays (entries may be NULL) that accumulate dL/d(nodal field)
 * (FP64 atomics: the last bits depend on the summation order). nbasis <=
 * PRT_MAX_FIELD_BASIS basis fields, basis[6*k + c] component c of field k
 * (NULL = zero): grad_theta[k] (device) accumulates sum over particles of
 * dL/dE . E_k + dL/dB . B_k in a fixed order (deterministic). */
int prt_lsrk_stage_adjoint(const prt_pusher *pusher, prt_workspace *ws, int64_t n,
                           const double *positions, const double *momenta,
                           const uint32_t *elements, const double *charges,
                           const double *masses, double *lam_x, double *lam_p,
                           double *lam_kx, double *lam_kp,
                           const double *const field_coefficients[6], double rk_a,
                           double rk_b, double dt, double vacuum_c,
                           double *const grad_fields[6],
                           int32_t nbasis, const double *const *basis,
                           double *grad_theta, void *stream);

/* Adjoint of prt_get_velocities: lam_p += (dv/dp)^T lam_v. */
int prt_velocities_adjoint(int64_t n, const double *momenta, const double *masses,
                           double vacuum_c, const double *lam_v, double *lam_p,
                           void *stream);

/* Adjoint of prt_deposit_shape in PRT_DEPOSIT_PLAIN mode: given dL/drho [Nn]
 * and dL/dj [3][Nn] (either may be NULL), accumulates dL/dx into lam_x [3][n]
 * and dL/dv into lam_v [3][n] (may be NULL). One lane per particle gathers
 * the node adjoints within its radius, deterministically; fastest with the
 * particles sorted by element (a warp's 32 particles share candidates). */
int prt_deposit_shape_adjoint(const prt_mesh *mesh, prt_workspace *ws,
                              prt_shape_function shape, int64_t n,
                              const double *positions, const double *charges,
                              const double *velocities, const uint32_t *elements,
                              const double *grad_rho, const double *grad_j,
                              double *lam_x, double *lam_v, void *stream);

/* ---------------------------------------------------- averaging pusher --- */

/* Replaces AveragingPusher3d3v(mesh, mass_matrix).forces(ex, ey, ez, bx, by,
 * bz, ps, pusher_state, depositor, depositor_state, velocities, vis_listener)
 * (push_average.hpp:330-420, wrap_pusher.cpp): forces[3][n] = q <E> +
 * v x (q <B>), <F> the average of the nodal field over the nodes within the
 * shape radius weighted by |J_e| w_i S(x_i - x_p) (integral_weights: HOST
 * [Np], w = M 1). Zero force and PRT_WARN_ZERO_AVERAGE for a particle with
 * no weight. vis (NULL or [14][n]): pt_e (3), pt_b (3), pt_e_stddev,
 * pt_b_stddev, el_force (3), mag_force (3). scales (NULL or [n]): the
 * normalisation q / (reconstructed charge) of each particle (the pusher
 * state's statistics). */
int prt_average_forces(const prt_mesh *mesh, prt_workspace *ws, prt_shape_function shape,
                       const double *integral_weights, int64_t n, const double *positions,
                       const double *charges, const double *velocities,
                       const uint32_t *elements, const double *const fields[6],
                       double *forces, double *vis, double *scales, void *stream);

/* One low-storage RK stage from given forces (a pusher whose forces come
 * from a separate pass): k = a k + dt (v(p), F), (x, p) += b k, relocation,
 * as prt_lsrk_stage after its force. */
int prt_lsrk_update(const prt_mesh *mesh, prt_workspace *ws, int64_t n, double *positions,
                    double *momenta, const double *masses, uint32_t *elements, double *kx,
                    double *kp, const double *forces, double rk_a, double rk_b, double dt,
                    double vacuum_c, void *stream);

/* --------------------------------------------------------- diagnostics --- */

/* Replaces kinetic_energies(ps, c) (diagnostics.hpp:38-58): per particle
 * (gamma - 1) m c^2, written as p^2 c^2 / (E + m c^2) (the reference's
 * (p/v - m) c^2 without its 0/0 at p = 0); 0 for removed particles
 * (elements may be NULL: all live). */
int prt_kinetic_energies(int64_t n, const double *momenta, const double *masses,
                         const uint32_t *elements, double vacuum_c, double *out,
                         void *stream);

/* Sums over the live particles in one fused pass, from which the reference's
 * beam diagnostics follow (diagnostics.hpp:61-180; pyrticle/log.py:107-325):
 * total_charge = Q, particle_momentum = P, kinetic energy = KE,
 * rms_beam_size(d) = sqrt(X2[d] / N), rms_beam_emittance(d, b) from X, X2,
 * XP, XP2, XXP with x' = p_d / p_b (0 where p_b = 0), rms_energy_spread =
 * sqrt(KE2 / N - (KE / N - ke_shift)^2), particle_current = QV / length.
 * KE2 sums (KE - ke_shift)^2: with ke_shift near the mean (a first call's
 * KE / N) the spread loses no digits to cancellation (the reference's
 * sqrt(<KE^2> - <KE>^2), tools.hpp:303-322, loses ~12 for a gamma = 2 beam
 * with 1e-3 momentum spread). `out` is a HOST array; the call synchronises
 * `stream`. Deterministic (fixed-order sums). */
enum prt_beam_moment {
  PRT_BM_COUNT = 0, PRT_BM_CHARGE = 1, PRT_BM_P = 2, PRT_BM_KE = 5, PRT_BM_KE2 = 6,
  PRT_BM_X = 7, PRT_BM_X2 = 10, PRT_BM_XP = 13, PRT_BM_XP2 = 16, PRT_BM_XXP = 19,
  PRT_BM_QV = 22, PRT_BEAM_MOMENTS = 25
};
int prt_beam_moments(prt_workspace *ws, int64_t n, const double *positions,
                     const double *momenta, const double *charges, const double *masses,
                     const uint32_t *elements, double vacuum_c, int32_t beam_axis,
                     double ke_shift, double out[PRT_BEAM_MOMENTS], void *stream);

/* ---------------------------------------------------------------- misc --- */

/* Sorts the particle store by containing element (stable), permuting every
 * given [n] / [3][n] array in place through `ws` scratch. Arrays may be NULL. */
int prt_sort_by_element(prt_workspace *ws, int64_t n, uint32_t *elements,
                        double *positions, double *momenta, double *charges,
                        double *masses, double *kx, double *kp, int64_t *ids,
                        void *stream);

/* Library version string. */
const char *prt_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PRT_H_INCLUDED */
