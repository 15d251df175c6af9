"""Device mesh tables (the reference's ``MeshData``, meshdata.py:37-133 and
meshdata.hpp:53-216), held by libprt."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, meshgen

INVALID_ELEMENT = _lib.INVALID_ELEMENT
INVALID_AXIS = _lib.INVALID_AXIS


class MeshData:
    """Owns a ``prt_mesh`` handle built from a :class:`Discretization`."""

    INVALID_ELEMENT = INVALID_ELEMENT
    INVALID_AXIS = INVALID_AXIS

    def __init__(self, dimensions: int = 3):
        if dimensions != 3:
            raise ValueError("only 3D meshes are supported")
        self.dimensions = dimensions
        self.handle = None
        self.discr = None

    def fill_from_hedge(self, discr) -> None:
        """Build the tables from a discretisation (name kept from the reference)."""
        self.fill_from_discretization(discr)

    def fill_from_discretization(self, discr) -> None:
        lib = _lib.load()
        self.discr = discr
        mesh = discr.mesh
        self.bins = meshgen.element_bins(mesh)
        keep: list = []
        desc = _lib.mesh_desc(mesh, np.ascontiguousarray(discr.nodes), self.bins, keep)
        h = C.c_void_p()
        _lib.check(lib.prt_mesh_create(C.byref(desc), C.byref(h)), "prt_mesh_create")
        self.handle = h
        self.element_count = mesh.element_count
        self.nodes_per_element = discr.nodes_per_element

    def __del__(self):
        if getattr(self, "handle", None) is not None and _lib._lib is not None:
            _lib._lib.prt_mesh_destroy(self.handle)
            self.handle = None

    # --- helpers of the reference's Python MeshData (meshdata.py:135-152)
    def min_vertex_distance_for_el(self, el: int) -> float:
        pts = self.discr.mesh.points[self.discr.mesh.elements[el]]
        d = np.linalg.norm(pts[:, None] - pts[None], axis=-1)
        return float(d[d > 0].min())

    def advisable_particle_radius(self) -> float:
        m = self.discr.mesh
        p = m.points[m.elements]
        d = np.linalg.norm(p[:, :, None] - p[:, None], axis=-1)
        d[d == 0] = np.inf
        dist = np.sort(d.reshape(len(p), -1).min(axis=1))
        return 0.6 * float(dist[int(0.25 * len(dist))])
