"""The grid depositor's host set-up runs on all host cores: point finding in
element chunks, Vandermonde rows in blocks and the basis reduction per point
count run in threads. The results must be bitwise those of one thread (the
reference's serial set-up, grid.py:217-273, 552-669)."""

import numpy as np

from pyrticle_b200 import problems
from pyrticle_b200.deposition import grid as G


def _setup(mesh, order, brick, chunk):
    starts, gidx, pts, w = G.find_points_in_elements(mesh, [brick], 0.12, chunk=chunk)
    mats, mstarts, kept = G.basis_reduction_matrices(mesh, order, starts, pts, w)
    return starts, gidx, pts, w, mats, mstarts, kept


def test_threaded_grid_setup_is_bitwise_serial(monkeypatch):
    w = problems.make("config1", scale=1e-5, cubes=(4, 4, 16))
    mesh = w.mesh
    dims = np.array([16, 16, 64])
    brick = G.BrickInfo(0, 0, (mesh.bbox_max - mesh.bbox_min) / dims, mesh.bbox_min, dims)
    # small chunks and blocks so that several threads take part
    monkeypatch.setattr(G.os, "cpu_count", lambda: 1)
    serial = _setup(mesh, w.order, brick, chunk=97)
    monkeypatch.setattr(G.os, "cpu_count", lambda: 8)
    threaded = _setup(mesh, w.order, brick, chunk=97)
    for a, b in zip(serial, threaded):
        assert np.array_equal(a, b)
    # the Vandermonde rows in blocks equal one evaluation
    pts = np.random.default_rng(3).random((1000, 3)) * 0.3
    modes = G.refelement.mode_identifiers(w.order)
    one = G.refelement.orthonormal_vandermonde(pts, modes)
    assert np.array_equal(G.orthonormal_vandermonde_fast(pts, modes, block=97), one)
