// handles.cuh -- layouts of the opaque C-ABI handles (library-internal).
#pragma once

#include <vector>

#include "common.cuh"

// Workspace scratch slots (grow-only device buffers).
enum {
  PRT_WS_SORT_KEYS = 0,
  PRT_WS_SORT_VALS,
  PRT_WS_SORT_TMP,
  PRT_WS_CUB,
  PRT_WS_DEP_KEYS,
  PRT_WS_DEP_VALS,
  PRT_WS_DEP_PARTICLES,
  PRT_WS_DEP_BINSTARTS,
  PRT_WS_DEP_SCALE,
  PRT_WS_DEP_STATS,
  PRT_WS_DEP_COUNT,
  PRT_WS_DEP_VALUES,
  PRT_WS_ADJ_POSITIONS,
  PRT_WS_ADJ_PARTIALS,
  PRT_WS_DIAGNOSTICS,
  PRT_WS_AVERAGE,
  PRT_WS_GROUP_ORDER,
  PRT_WS_TC_TILES,    // tensor-core deposition: position-tile operands (per radius)
  PRT_WS_TC_WDIG,     // tensor-core deposition: position weight digits
  PRT_WS_TC_PART,     // tensor-core deposition: per-particle sums, values and digits
  PRT_WS_TC_MISC,     // tensor-core deposition: scales, counters, tile order
  PRT_WS_TC_TILESET,  // tensor-core deposition: tile starts and boxes (per radius)
  PRT_WS_SLOTS
};

// Distinct node positions (coincident DG nodes merged), in Morton order:
// the targets of the mesh deposition.
struct PositionSet {
  long long count = 0;
  const double *pos = nullptr;            // [count][3]
  const uint32_t *node_to_pos = nullptr;  // [Nn]
  const uint32_t *run_starts = nullptr;   // [count + 1] into run_nodes
  const uint32_t *run_nodes = nullptr;    // [Nn] node ids grouped by position, ascending
  // warp groups: runs of <= 32 consecutive positions that never straddle a
  // Morton cell of about 24 positions, with their bounding spheres
  long long groups = 0;
  const uint32_t *group_starts = nullptr; // [groups + 1]
  const double *group_spheres = nullptr;  // [groups][4]: centre xyz, radius
  // wide warp groups for the deposition (two positions per lane): runs of
  // <= 64 positions that never straddle a Morton cell of about twice the
  // group target
  long long wide_groups = 0;
  const uint32_t *wide_starts = nullptr;  // [wide_groups + 1]
  const double *wide_spheres = nullptr;   // [wide_groups][4]
  // the groups binned by the bin of their sphere centre (each group in
  // exactly one bin; uniform bins of about a group radius), in bin order:
  // spheres and position ranges, with CSR bin starts
  struct {
    double origin[3], inv_w[3];
    int dims[3];
    double max_radius = 0;
    const uint32_t *starts = nullptr;   // [nbins + 1]
    const double *spheres = nullptr;    // [groups][4], bin order
    const uint32_t *ranges = nullptr;   // [groups][2]: first position, count
  } centre_bins;
};

struct prt_mesh {
  DevMesh dev;
  const double *face_centroids = nullptr;  // [E][4][3]
  const double *face_radii = nullptr;      // [E][4]
  double box_lo[3], box_hi[3];             // node bounding box of the mesh
  PositionSet positions;
  unsigned long long uid = 0;              // unique per created mesh (workspace caches)
  // host copy of the positions [count][3]: the tensor-core deposition cuts
  // its tiles from them per shape radius
  std::vector<double> pos_host;
};

// CUDA-event timing of the main kernels (prt_workspace_timing).
struct KernelTimer {
  static constexpr int RING = 256;
  cudaEvent_t start[RING], stop[RING];
  int used = 0;          // recorded pairs not yet read
  bool created = false;
  double total_ms = 0;
  long long launches = 0;
};

struct prt_workspace {
  void *buf[PRT_WS_SLOTS];
  size_t cap[PRT_WS_SLOTS];
  // PRT_WS_TC_TILES holds the tile operands of the mesh with this uid and
  // this shape radius
  unsigned long long tc_mesh_uid = 0;
  double tc_radius = 0;
  long long tc_tiles = 0;   // tiles of that mesh and radius (PRT_WS_TC_TILESET)
  double tc_bin_width = 0;  // particle bin width for those tiles
  long long tc_n = -1;      // particles of the last tensor-core charges step
  DevStatus *status = nullptr;
  bool timing = false;
  KernelTimer timers[PRT_TIME_CATEGORIES];
};

// Brackets a launch with events when timing is enabled.
struct ScopedTimer {
  prt_workspace *ws;
  int cat;
  cudaStream_t s;
  int slot = -1;
  ScopedTimer(prt_workspace *w, int c, cudaStream_t st);
  ~ScopedTimer();
};

struct prt_pusher {
  const prt_mesh *mesh;
  int order;
  int np;
  std::vector<double> w;  // [np][np], canonical monomial order
  // the mixed-precision stage's tensor-core operand: W rounded to FP32 and
  // split into three BF16 terms, in the MMA's shared-memory layout (device)
  void *w_split = nullptr;
};

// Builds prt_pusher::w_split (orders 1-3; a no-op for order 4).
int prt_pusher_prepare_mixed(prt_pusher *P);
// The mixed-precision stage (prt_lsrk_stage with PRT_PRECISION_MIXED).
struct Fields6;
int launch_stage_mixed(const prt_pusher *P, prt_workspace *ws, long long n, double *x,
                       double *p, const double *q, const double *m, uint32_t *el, double *kx,
                       double *kp, const Fields6 &F, double a, double b, double dt, double c,
                       cudaStream_t s);

constexpr int PRT_WARP_NODES = 32;
// target positions per Morton cell when cutting warp groups
constexpr double PRT_GROUP_TARGET = 24.0;
// Morton bits dropped from the group cells for the wide groups (1: cells of
// two sibling cells, about twice the positions)
#ifndef PRT_WIDE_CELL_BITS
#define PRT_WIDE_CELL_BITS 1
#endif

void *ws_buffer(prt_workspace *ws, int slot, size_t bytes, int *rc);
int prt_mesh_build_positions(prt_mesh *m, const prt_mesh_desc *d);

// Shared pieces of the shape deposition (deposit.cu) used by the
// tensor-core form (deposit_tc.cu).
// W[u] = sum over the nodes at position u of w_i |J_e| (device; iw a HOST [Np]).
int prt_dep_position_weights(const prt_mesh *mesh, prt_workspace *ws, const double *iw,
                             double *W, cudaStream_t s);
// The normalising depositor's statistics from per-particle scales and hit
// counts (hits < 0: removed particle); synchronises s.
int prt_dep_norm_stats(prt_workspace *ws, long long n, const double *scale,
                       const double *hits, prt_deposit_stats *stats, cudaStream_t s);
// rho/j of every node from the values of its position (vals [4][npos]).
int prt_dep_expand(const prt_mesh *mesh, const double *vals, double *rho, double *j,
                   cudaStream_t s);
// The chosen-form shape deposition on the tensor cores (alpha = 2).
int prt_deposit_shape_tc(const prt_mesh *mesh, prt_workspace *ws, int32_t mode,
                         prt_shape_function shape, const double *iw, long long n,
                         const double *x, const double *q, const double *v,
                         const uint32_t *el, double *rho, double *j,
                         prt_deposit_stats *stats, cudaStream_t s);

// A unique id per mesh or grid (the workspace caches key on it).
unsigned long long prt_next_target_uid();

// The points a tensor-core deposition sums onto: a mesh's distinct node
// positions or a grid's brick points.
struct TcTarget {
  const prt_mesh *mesh = nullptr;  // periodicity
  unsigned long long uid = 0;
  long long npos = 0;
  const double *pos = nullptr;       // device [npos][3]
  const double *pos_host = nullptr;  // host [npos][3]
  double lo[3], hi[3];               // box the particle bins cover
};
// The plain shape deposition (alpha = 2) onto a target's points on the tensor
// cores: rho [npos] and j [3][npos] (either may be NULL).
int prt_deposit_points_tc(const TcTarget &T, prt_workspace *ws, prt_shape_function shape,
                          long long n, const double *x, const double *q, const double *v,
                          const uint32_t *el, double *rho, double *j, cudaStream_t s);
