"""ctypes binding of libprt.so (the C ABI declared in include/prt.h).

The library is the product path: there is no fallback. If ``libprt.so`` is
missing or fails to load, importing anything that needs it raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libprt.so"

INVALID_ELEMENT = 0xFFFFFFFF
INVALID_AXIS = 0xFFFFFFFF

PRT_OK = 0
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of device memory",
    -4: "no best normal found--weird",
    -5: "particle has no containing element",
    -6: "size exceeds the fixed scratch capacity",
    -7: "a kernel's bounded wait on its tensor-core work timed out",
}
PRT_WARN_ZERO_MASS = 1
PRT_WARN_ZERO_AVERAGE = 2
PRT_ERR_CAPACITY = -6
NOALLOC_SCRATCH_BYTES = 64 << 20

TIME_DEPOSIT_GATHER = 0
TIME_DEPOSIT_STAGE = 1
TIME_LSRK_STAGE = 2
TIME_SORT = 3
TIME_STAGE_ADJOINT = 4
TIME_DEPOSIT_ADJOINT = 5
TIME_DEPOSIT_NORMALIZE = 6
MAX_FIELD_BASIS = 4
BEAM_MOMENTS = 25
BM = dict(count=0, charge=1, p=2, ke=5, ke2=6, x=7, x2=10, xp=13, xp2=16, xxp=19, qv=22)

DEPOSIT_PLAIN = 0
DEPOSIT_NORMALIZED = 1
GRID_SHAPE = 0
GRID_TRILINEAR = 1

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)


class MeshDesc(C.Structure):
    _fields_ = [
        ("element_count", C.c_int64),
        ("vertex_count", C.c_int64),
        ("nodes_per_element", C.c_int32),
        ("reserved0", C.c_int32),
        ("vertices", _dp),
        ("element_vertices", _u32p),
        ("inverse_maps", _dp),
        ("jacobians", _dp),
        ("face_normals", _dp),
        ("face_plane_rhs", _dp),
        ("face_centroids", _dp),
        ("face_radii", _dp),
        ("face_neighbors", _u32p),
        ("face_periodicity_axes", _u32p),
        ("vertex_adj_starts", _u32p),
        ("vertex_adj_elements", _u32p),
        ("periodicity_min", C.c_double * 3),
        ("periodicity_max", C.c_double * 3),
        ("nodes", _dp),
        ("bin_origin", C.c_double * 3),
        ("bin_inv_width", C.c_double * 3),
        ("bin_dims", C.c_int32 * 3),
        ("reserved1", C.c_int32),
        ("bin_starts", _u32p),
        ("bin_elements", _u32p),
    ]


class FindCounters(C.Structure):
    _fields_ = [("find_same", C.c_uint64), ("find_by_neighbor", C.c_uint64),
                ("find_by_vertex", C.c_uint64), ("find_global", C.c_uint64)]


class ShapeFunctionDesc(C.Structure):
    _fields_ = [("radius", C.c_double), ("alpha", C.c_double), ("normalizer", C.c_double)]


class DepositStats(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "norm_count", "norm_sum", "norm_sum_sq", "norm_min", "norm_max",
        "el_count", "el_sum", "el_sum_sq", "el_min", "el_max", "pair_count",
        "node_pair_count", "evaluated_pairs")]


class Brick(C.Structure):
    _fields_ = [("origin", C.c_double * 3), ("stepwidths", C.c_double * 3),
                ("dims", C.c_int32 * 3), ("reserved", C.c_int32),
                ("start_index", C.c_int64)]


class GridDesc(C.Structure):
    _fields_ = [
        ("brick_count", C.c_int32),
        ("nodes_per_element", C.c_int32),
        ("bricks", C.POINTER(Brick)),
        ("eog_count", C.c_int64),
        ("eog_elements", _u32p),
        ("eog_starts", _u64p),
        ("eog_grid_nodes", _u32p),
        ("eog_weights", _dp),
        ("eog_matrix_starts", _u64p),
        ("eog_matrices", _dp),
        ("avg_group_count", C.c_int64),
        ("avg_group_starts", _u32p),
        ("avg_group_nodes", _u32p),
        ("point_origins", _dp),
    ]


_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_d = C.c_double

# name -> (restype, argtypes); every function declared in include/prt.h
SIGNATURES = {
    "prt_mesh_create": (_i32, [C.POINTER(MeshDesc), C.POINTER(_vp)]),
    "prt_mesh_destroy": (_i32, [_vp]),
    "prt_workspace_create": (_i32, [C.POINTER(_vp)]),
    "prt_workspace_destroy": (_i32, [_vp]),
    "prt_workspace_status": (_i32, [_vp, _vp, C.POINTER(_i32), C.POINTER(_i64),
                                    C.POINTER(_i32), C.POINTER(_i64), _i32]),
    "prt_workspace_counters": (_i32, [_vp, _vp, C.POINTER(FindCounters), _i32]),
    "prt_workspace_timing": (_i32, [_vp, _i32]),
    "prt_workspace_timing_read": (_i32, [_vp, _i32, C.POINTER(_d), C.POINTER(_i64), _i32]),
    "prt_get_velocities": (_i32, [_i64, _vp, _vp, _d, _vp, _vp]),
    "prt_find_containing_elements": (_i32, [_vp, _i64, _vp, _vp, _vp]),
    "prt_update_containing_elements": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp, _vp]),
    "prt_monomial_pusher_create": (_i32, [_vp, _i32, _u32p, _dp, C.POINTER(_vp)]),
    "prt_monomial_pusher_destroy": (_i32, [_vp]),
    "prt_forces": (_i32, [_vp, _i64, _vp, _vp, _vp, _vp, C.POINTER(_vp), _vp, _vp, _vp]),
    "prt_lsrk_stage": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                              C.POINTER(_vp), _d, _d, _d, _d, _i32, _vp]),
    "prt_deposit_shape": (_i32, [_vp, _vp, _i32, ShapeFunctionDesc, _dp, _i64, _vp, _vp,
                                 _vp, _vp, _vp, _vp, _i32, C.POINTER(DepositStats), _vp]),
    "prt_deposit_shape_noalloc": (_i32, [_vp, ShapeFunctionDesc, _i64, _vp, _vp, _vp, _vp,
                                         _vp, _vp, _vp]),
    "prt_mesh_position_count": (_i32, [_vp, C.POINTER(_i64)]),
    "prt_deposit_shape_charges": (_i32, [_vp, _vp, _i32, ShapeFunctionDesc, _dp, _i64, _vp,
                                         _vp, _vp, _vp, _vp, C.POINTER(DepositStats), _vp]),
    "prt_deposit_shape_sums": (_i32, [_vp, _vp, ShapeFunctionDesc, _i64, _vp, _vp, _vp]),
    "prt_deposit_shape_combine": (_i32, [_vp, _vp, ShapeFunctionDesc, _vp, _vp, _vp, _vp,
                                         _vp]),
    "prt_grid_create": (_i32, [_vp, C.POINTER(GridDesc), C.POINTER(_vp)]),
    "prt_grid_destroy": (_i32, [_vp]),
    "prt_deposit_grid": (_i32, [_vp, _vp, _i32, ShapeFunctionDesc, _i64, _vp, _vp, _vp,
                                _vp, _vp, _vp, _vp]),
    "prt_deposit_grid_mixed": (_i32, [_vp, _vp, ShapeFunctionDesc, _i64, _vp, _vp, _vp, _vp,
                                      _vp, _vp, _vp]),
    "prt_remap_grid_to_mesh": (_i32, [_vp, _vp, _vp, _i64, _i64, _vp]),
    "prt_remap_grid_to_mesh_components": (_i32, [_vp, _vp, _vp, _i32, _vp]),
    "prt_sort_by_element": (_i32, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "prt_lsrk_stage_record": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                     _vp, _vp, _vp, C.POINTER(_vp), _d, _d, _d, _d, _vp]),
    "prt_lsrk_stage_adjoint": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                      _vp, _vp, C.POINTER(_vp), _d, _d, _d, _d,
                                      C.POINTER(_vp), _i32, C.POINTER(_vp), _vp, _vp]),
    "prt_velocities_adjoint": (_i32, [_i64, _vp, _vp, _d, _vp, _vp, _vp]),
    "prt_fields_to_monomial": (_i32, [_vp, _i32, C.POINTER(_vp), C.POINTER(_vp), _vp]),
    "prt_deposit_shape_adjoint": (_i32, [_vp, _vp, ShapeFunctionDesc, _i64, _vp, _vp, _vp,
                                         _vp, _vp, _vp, _vp, _vp, _vp]),
    "prt_average_forces": (_i32, [_vp, _vp, ShapeFunctionDesc, _dp, _i64, _vp, _vp, _vp, _vp,
                                  C.POINTER(_vp), _vp, _vp, _vp, _vp]),
    "prt_lsrk_update": (_i32, [_vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _d, _d, _d,
                               _d, _vp]),
    "prt_kinetic_energies": (_i32, [_i64, _vp, _vp, _vp, _d, _vp, _vp]),
    "prt_beam_moments": (_i32, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _d, _i32, _d, _dp, _vp]),
    "prt_version": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Load libprt.so once; raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m pyrticle_b200.build` "
            "(there is no CPU fallback for this path)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib.prt_last_error_message.restype = C.c_char_p
    lib.prt_last_error_message.argtypes = []
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != PRT_OK:
        msg = ERRORS.get(rc, f"error {rc}")
        if rc == -2:
            detail = load().prt_last_error_message()
            msg += f": {detail.decode() if detail else ''}"
        raise RuntimeError(f"{what}: {msg}" if what else msg)


def ptr(arr, ctype=C.c_double):
    """ctypes pointer to a contiguous numpy array (host)."""
    if arr is None:
        return None
    assert arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(ctype))


def dptr(t) -> int | None:
    """Device address of a torch tensor (or None)."""
    if t is None:
        return None
    return t.data_ptr()


def mesh_desc(mesh, nodes: np.ndarray, bins, keep: list) -> MeshDesc:
    """Fill a MeshDesc from a meshgen.Mesh; arrays are appended to ``keep``."""

    def arr(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a

    d = MeshDesc()
    d.element_count = mesh.element_count
    d.vertex_count = mesh.vertex_count
    d.nodes_per_element = len(nodes) // mesh.element_count
    d.vertices = ptr(arr(mesh.points, np.float64))
    d.element_vertices = ptr(arr(mesh.elements, np.uint32), C.c_uint32)
    d.inverse_maps = ptr(arr(mesh.inverse_maps, np.float64))
    d.jacobians = ptr(arr(mesh.jacobians, np.float64))
    d.face_normals = ptr(arr(mesh.face_normals, np.float64))
    d.face_plane_rhs = ptr(arr(mesh.face_plane_rhs, np.float64))
    d.face_centroids = ptr(arr(mesh.face_centroids, np.float64))
    d.face_radii = ptr(arr(mesh.face_radii, np.float64))
    d.face_neighbors = ptr(arr(mesh.face_neighbors, np.uint32), C.c_uint32)
    d.face_periodicity_axes = ptr(arr(mesh.face_periodicity_axes, np.uint32), C.c_uint32)
    d.vertex_adj_starts = ptr(arr(mesh.vertex_adj_starts, np.uint32), C.c_uint32)
    d.vertex_adj_elements = ptr(arr(mesh.vertex_adj_elements, np.uint32), C.c_uint32)
    for a in range(3):
        d.periodicity_min[a] = float(mesh.periodicity_min[a])
        d.periodicity_max[a] = float(mesh.periodicity_max[a])
    d.nodes = ptr(arr(nodes, np.float64))
    lo, inv, dims, starts, els = bins
    for a in range(3):
        d.bin_origin[a] = float(lo[a])
        d.bin_inv_width[a] = float(inv[a])
        d.bin_dims[a] = int(dims[a])
    d.bin_starts = ptr(arr(starts, np.uint32), C.c_uint32)
    d.bin_elements = ptr(arr(els, np.uint32), C.c_uint32)
    return d


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)
