"""Grid-find deposition (the reference's ``deposition/grid_find.py`` and
``dep_grid_find.hpp``).

The reference sorts the mesh nodes into the cells of one or more bricks
(grid_find.py:55-104) and deposits every particle onto the nodes listed in
the cells of its box [x - a, x + a] (dep_grid_find.hpp:73-112), periodic
copies included (dep_grid_base.hpp:285-347). A node within the shape radius
of a particle always lies in a cell of that box, and the reference requires
every node to lie in some brick, so the result is the plain shape deposition
over all mesh nodes within the radius: on the device it runs as the same
gather over distinct node positions as ShapeFunctionDepositor. The brick
cell -> node lists are still built here, with the reference's order and its
error for nodes that no brick covers, and exposed under the reference's
names (``node_number_list_starts``, ``node_number_lists``)."""

from __future__ import annotations

import numpy as np

from .grid import BrickInfo
from .grid_base import SingleBrickGenerator
from .shape import ShapeFunctionDepositor


def grid_node_lists(mesh, nodes, nodes_per_element, bricks):
    """The brick cell -> mesh node lists of grid_find.py:63-104.

    Per element (ascending), per brick whose box meets the element's vertex
    box, every node of the element that lies in a cell of the brick
    (brick.which_cell, grid.hpp:270-280) is appended to that cell's list.
    Returns (starts [G+1], lists) as uint32 arrays, G the grid node count."""
    E = mesh.element_count
    Np = nodes_per_element
    p = mesh.points[mesh.elements]
    elo, ehi = p.min(axis=1), p.max(axis=1)
    node_el = np.arange(E * Np) // Np
    keys, els, brk_no, node_no = [], [], [], []
    for brk in bricks:
        blo, bhi = brk.bounding_box()
        # box::intersect(...).is_empty() (tools.hpp:119-125, 142-160)
        meets = np.all(np.maximum(elo, blo) < np.minimum(ehi, bhi), axis=1)
        cell = np.floor((nodes - brk.origin) / brk.stepwidths).astype(np.int64)
        inside = np.all((cell >= 0) & (cell < brk.dims), axis=1) & meets[node_el]
        idx = np.nonzero(inside)[0]
        keys.append(brk.start_index + cell[idx] @ brk.strides)
        els.append(node_el[idx])
        brk_no.append(np.full(len(idx), brk.number))
        node_no.append(idx)
    keys = np.concatenate(keys)
    els = np.concatenate(els)
    brk_no = np.concatenate(brk_no)
    node_no = np.concatenate(node_no)
    if len(np.unique(node_no)) != len(nodes):
        raise RuntimeError("dep_grid_find: unassigned mesh nodes found. "
                           "you should specify a mesh_margin when generating bricks")
    if len(node_no) != len(nodes):
        # a node listed twice would receive a particle's charge once per
        # brick the particle's box meets (depending on the brick cache)
        raise NotImplementedError("dep_grid_find: overlapping bricks (a mesh node lies in "
                                  "cells of two bricks)")
    # append order of the reference: element, then brick, then node
    order = np.lexsort((node_no, brk_no, els, keys))
    G = bricks[-1].start_index + len(bricks[-1])
    starts = np.zeros(G + 1, dtype=np.int64)
    starts[1:] = np.cumsum(np.bincount(keys, minlength=G))
    return starts.astype(np.uint32), node_no[order].astype(np.uint32)


class GridFindDepositor(ShapeFunctionDepositor):
    """Deposit through brick cells' node lists (grid_find.py:34-151).

    @arg brick_generator: yields (stepwidths, origin, dims) per brick;
      default one brick over the mesh box with a margin of 1e-3 of its
      largest extent and 0.2 grid points per node (grid_find.py:55-60).
    @arg precision: "fp64" (default) or "mixed", as for ShapeFunctionDepositor.
    """

    name = "GridFind"

    def __init__(self, brick_generator=None, precision="fp64"):
        ShapeFunctionDepositor.__init__(self, precision=precision)
        self.brick_generator = brick_generator

    def initialize(self, method):
        ShapeFunctionDepositor.initialize(self, method)
        discr = method.discretization
        mesh = discr.mesh
        if self.brick_generator is None:
            self.brick_generator = SingleBrickGenerator(
                mesh_margin=1e-3 * float(np.max(mesh.bbox_max - mesh.bbox_min)),
                overresolve=0.2)
        self.bricks = []
        start = 0
        for i, (sw, origin, dims) in enumerate(self.brick_generator(discr)):
            b = BrickInfo(i, start, sw, origin, dims)
            self.bricks.append(b)
            start += len(b)
        self.grid_node_count = start
        self.node_number_list_starts, self.node_number_lists = grid_node_lists(
            mesh, np.asarray(discr.nodes), discr.nodes_per_element, self.bricks)
        # nodes per grid cell (the reference's "usecounts" debug field)
        self.usecounts = np.diff(self.node_number_list_starts.astype(np.int64))
