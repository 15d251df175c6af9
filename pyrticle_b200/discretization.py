"""A minimal stand-in for the parts of hedge's ``Discretization`` that the
particle side reads.

The reference's plugins take a hedge discretisation and use: ``dimensions``,
``nodes`` and ``len(discr)`` (cloud.py, meshdata.py:133), ``mesh``
(periodicity, bounding box), ``element_groups[i].local_discretization`` with
``node_tuples``, ``unit_nodes``, ``mass_matrix``, ``vandermonde``,
``basis_functions`` and ``generate_mode_identifiers`` (pusher.py:94-114,
shape.py:64-69, grid.py:195-273), ``find_el_range`` and ``volume_zeros``.
This module provides exactly those, on top of :mod:`meshgen` and
:mod:`refelement`.
"""

from __future__ import annotations

import numpy as np

from . import meshgen, refelement


class LocalDiscretization:
    """Order-N nodal tetrahedron (reference element of :mod:`refelement`)."""

    dimensions = 3

    def __init__(self, order: int):
        self.order = int(order)

    def node_count(self) -> int:
        return refelement.node_count(self.order)

    def node_tuples(self):
        return refelement.node_tuples(self.order)

    def unit_nodes(self) -> np.ndarray:
        return refelement.unit_nodes(self.order)

    def generate_mode_identifiers(self):
        return refelement.mode_identifiers(self.order)

    def basis_functions(self):
        return [(lambda pts, m=m: refelement.orthonormal_mode(np.atleast_2d(pts), m))
                for m in self.generate_mode_identifiers()]

    def vandermonde(self) -> np.ndarray:
        return refelement.orthonormal_vandermonde(self.unit_nodes(),
                                                  self.generate_mode_identifiers())

    def mass_matrix(self) -> np.ndarray:
        return refelement.mass_matrix(self.order)

    def integration_weights(self) -> np.ndarray:
        return refelement.integration_weights(self.order)


class ElementGroup:
    def __init__(self, ldis: LocalDiscretization, members):
        self.local_discretization = ldis
        self.members = members


class Discretization:
    """Nodes of a single-order DG discretisation on a :class:`meshgen.Mesh`."""

    dimensions = 3

    def __init__(self, mesh: meshgen.Mesh, order: int, nodes: np.ndarray | None = None):
        self.mesh = mesh
        self.order = int(order)
        self.ldis = LocalDiscretization(order)
        self.nodes = meshgen.element_nodes(mesh, order) if nodes is None else nodes
        self.element_groups = [ElementGroup(self.ldis, range(mesh.element_count))]

    def __len__(self) -> int:
        return len(self.nodes)

    @property
    def nodes_per_element(self) -> int:
        return self.ldis.node_count()

    def find_el_range(self, el: int) -> slice:
        np_ = self.nodes_per_element
        return slice(el * np_, (el + 1) * np_)

    def volume_zeros(self, shape=()) -> np.ndarray:
        return np.zeros(tuple(shape) + (len(self),), dtype=np.float64)

    def integral(self, vec: np.ndarray) -> float:
        """Integral of a nodal vector (w = M 1 per element, times |J|)."""
        w = self.ldis.integration_weights()
        return float((vec.reshape(-1, len(w)) @ w * self.mesh.jacobians).sum())

    def interpolate_volume_function(self, f) -> np.ndarray:
        return np.array([f(x, None) for x in self.nodes])
