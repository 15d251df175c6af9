"""Brick generators for grid deposition (the reference's
``deposition/grid_base.py:30-151``)."""

from __future__ import annotations

import numpy as np


class SingleBrickGenerator:
    """One brick over the mesh bounding box (+ margin), with about
    ``overresolve`` grid points per DG node, or explicit ``dims``."""

    def __init__(self, overresolve=1.5, mesh_margin=0, dims=None):
        self.overresolve = overresolve
        self.mesh_margin = mesh_margin
        self.dims = dims

    def __call__(self, discr):
        mesh = discr.mesh
        bbox_min = mesh.bbox_min - self.mesh_margin
        bbox_max = mesh.bbox_max + self.mesh_margin
        size = bbox_max - bbox_min
        if self.dims is None:
            volume = float(mesh.jacobians.sum() * 4 / 3)
            dx = (volume / len(discr) / self.overresolve) ** (1 / discr.dimensions)
            dims = np.asarray(size / dx, dtype=np.int32)
        else:
            dims = np.asarray(self.dims, dtype=np.int32)
        stepwidths = size / dims
        yield stepwidths, bbox_min, dims
