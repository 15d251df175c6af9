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
  PRT_WS_SLOTS
};

// Uniform bins over the mesh box listing the deposition tiles that overlap
// each bin (used by the particle-centric normalising pass).
struct TileBinsHost {
  double origin[3], inv_w[3];
  int dims[3];
  const uint32_t *starts = nullptr;
  const uint32_t *tiles = nullptr;
};

struct prt_mesh {
  DevMesh dev;
  const double *face_centroids = nullptr;  // [E][4][3]
  const double *face_radii = nullptr;      // [E][4]
  // deposition tiles: consecutive elements grouped so that a tile holds at
  // most PRT_TILE_NODES nodes; per tile the node bounding box
  int tile_elements = 0;                   // elements per tile
  long long tile_count = 0;
  const double *tile_boxes = nullptr;      // [tiles][6]: lo xyz, hi xyz
  const double *el_spheres = nullptr;      // [E][4]: node centroid xyz, radius
  double box_lo[3], box_hi[3];             // node bounding box of the mesh
  TileBinsHost tile_bins;
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
};

constexpr int PRT_TILE_NODES = 128;

void *ws_buffer(prt_workspace *ws, int slot, size_t bytes, int *rc);
int prt_mesh_build_tiles(prt_mesh *m, const prt_mesh_desc *d);
