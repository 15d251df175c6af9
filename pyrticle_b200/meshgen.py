"""Seeded tetrahedral box meshes and the per-element tables the particle side needs.

The reference fills its ``mesh_data`` from a hedge discretisation
(``meshdata.py:37-133``): per element the inverse affine map to the unit
simplex, ``|J|``, the node range, the vertices, and per face the outward
normal, neighbour, periodicity axis, plane right-hand side and bounding
circle; plus a vertex -> element CSR and the periodicity intervals. hedge is
not available, so this module builds the same tables for jittered Kuhn-split
box meshes, with these fixed conventions:

* face ``f`` of element ``(v0, v1, v2, v3)`` is ``(0,1,2), (0,1,3), (0,2,3),
  (1,2,3)`` for f = 0..3;
* element ``e`` owns nodes ``[e*Np, (e+1)*Np)`` (the layout the reference's
  monomial pusher assumes, ``push_monomial.hpp:104-110``);
* vertex-adjacent elements are listed in ascending element id (the reference
  takes them from a Python-2 ``set``, ``meshdata.py:330-352``, an order that
  cannot be reproduced; ascending id is the canonical replacement).

Host-side numpy set-up only: these tables are inputs, shared bit for bit by
the CPU oracle and the CUDA library.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import refelement

INVALID_ELEMENT = 0xFFFFFFFF
INVALID_AXIS = 0xFFFFFFFF

FACE_VERTICES = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))
FACE_OPPOSITE = (3, 2, 1, 0)

# Kuhn (Freudenthal) split of the unit cube into 6 tetrahedra along the
# main diagonal; conforming across neighbouring cubes.
_KUHN_PERMS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


@dataclasses.dataclass
class Mesh:
    """Tetrahedral mesh plus the particle-side tables (all numpy, host)."""

    points: np.ndarray              # [V, 3] f64
    elements: np.ndarray            # [E, 4] u32 vertex ids
    inverse_maps: np.ndarray        # [E, 12] f64: row-major A^{-1}, then -A^{-1} b
    forward_maps: np.ndarray        # [E, 12] f64: row-major A, then b (unit -> physical)
    jacobians: np.ndarray           # [E] |det A|
    face_normals: np.ndarray        # [E, 4, 3]
    face_plane_rhs: np.ndarray      # [E, 4]
    face_centroids: np.ndarray      # [E, 4, 3]
    face_radii: np.ndarray          # [E, 4]
    face_neighbors: np.ndarray      # [E, 4] u32 (INVALID_ELEMENT at the boundary)
    face_periodicity_axes: np.ndarray  # [E, 4] u32 (INVALID_AXIS unless periodic)
    vertex_adj_starts: np.ndarray   # [V+1] u32
    vertex_adj_elements: np.ndarray  # [nnz] u32, ascending element id per vertex
    periodicity_min: np.ndarray     # [3]; min == max means "not periodic"
    periodicity_max: np.ndarray     # [3]
    bbox_min: np.ndarray
    bbox_max: np.ndarray
    cube_dims: tuple = (0, 0, 0)    # (nx, ny, nz) for box meshes

    @property
    def element_count(self) -> int:
        return len(self.elements)

    @property
    def vertex_count(self) -> int:
        return len(self.points)

    def element_centroids(self) -> np.ndarray:
        return self.points[self.elements].mean(axis=1)

    def inradii(self) -> np.ndarray:
        p = self.points[self.elements]
        vol = np.abs(np.einsum("ij,ij->i", p[:, 1] - p[:, 0],
                               np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))) / 6
        area = np.zeros(len(p))
        for f in FACE_VERTICES:
            a, b, c = p[:, f[0]], p[:, f[1]], p[:, f[2]]
            area += 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
        return 3 * vol / area


def box_mesh(n=(8, 8, 32), lo=(0.0, 0.0, 0.0), hi=(0.01, 0.01, 0.04),
             jitter=0.15, seed=0, periodic=(False, False, False)) -> Mesh:
    """Box of ``nx*ny*nz`` cubes, 6 Kuhn tetrahedra each, interior vertices
    jittered uniformly by ``+-jitter`` cell sizes (seeded).

    Element id = 6 * cube id + Kuhn index, cube id x-fastest, so 6
    consecutive elements tile one (jittered) cube.
    """
    nx, ny, nz = (int(v) for v in n)
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    h = (hi - lo) / np.array([nx, ny, nz])

    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1),
                             indexing="ij")
    ii, jj, kk = (a.transpose(2, 1, 0).ravel() for a in (ii, jj, kk))  # x fastest
    idx = np.stack([ii, jj, kk], axis=1)
    pts = lo + idx * h
    # exact box faces
    for ax, cnt in enumerate((nx, ny, nz)):
        pts[idx[:, ax] == cnt, ax] = hi[ax]
    interior = ((ii > 0) & (ii < nx) & (jj > 0) & (jj < ny) & (kk > 0) & (kk < nz))
    rng = np.random.default_rng(seed)
    jit = rng.uniform(-jitter, jitter, size=pts.shape) * h
    pts[interior] += jit[interior]

    def vid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = (a.transpose(2, 1, 0).ravel() for a in (ci, cj, ck))
    ncubes = len(ci)
    elements = np.empty((ncubes, 6, 4), dtype=np.int64)
    corner = np.stack([ci, cj, ck], axis=1)
    for t, perm in enumerate(_KUHN_PERMS):
        c = corner.copy()
        elements[:, t, 0] = vid(c[:, 0], c[:, 1], c[:, 2])
        for s in range(3):
            c[:, perm[s]] += 1
            elements[:, t, s + 1] = vid(c[:, 0], c[:, 1], c[:, 2])
    elements = elements.reshape(-1, 4)

    p = pts[elements]
    det = np.einsum("ij,ij->i", p[:, 1] - p[:, 0],
                    np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))
    neg = det < 0
    elements[neg, 2], elements[neg, 3] = elements[neg, 3].copy(), elements[neg, 2].copy()

    per = np.asarray(periodic, dtype=bool)
    return _finish_mesh(pts, elements, lo, hi, per, (nx, ny, nz), idx)


def _finish_mesh(pts, elements, lo, hi, periodic, cube_dims, vertex_index) -> Mesh:
    E = len(elements)
    V = len(pts)
    p = pts[elements]                                   # [E, 4, 3]
    A = np.stack([(p[:, 1] - p[:, 0]) / 2, (p[:, 2] - p[:, 0]) / 2,
                  (p[:, 3] - p[:, 0]) / 2], axis=2)     # columns
    b = p[:, 0] + A.sum(axis=2)
    Ainv = np.linalg.inv(A)
    binv = -np.einsum("eij,ej->ei", Ainv, b)
    inverse_maps = np.concatenate([Ainv.reshape(E, 9), binv], axis=1)
    forward_maps = np.concatenate([A.reshape(E, 9), b], axis=1)
    jac = np.abs(np.linalg.det(A))

    normals = np.empty((E, 4, 3))
    rhs = np.empty((E, 4))
    centroids = np.empty((E, 4, 3))
    radii = np.empty((E, 4))
    for f, (fa, fb, fc) in enumerate(FACE_VERTICES):
        a, bb, c = p[:, fa], p[:, fb], p[:, fc]
        d = p[:, FACE_OPPOSITE[f]]
        n = np.cross(bb - a, c - a)
        n /= np.linalg.norm(n, axis=1)[:, None]
        flip = np.einsum("ij,ij->i", n, d - a) > 0
        n[flip] *= -1
        normals[:, f] = n
        rhs[:, f] = (np.einsum("ij,ij->i", n, a) + np.einsum("ij,ij->i", n, bb)
                     + np.einsum("ij,ij->i", n, c)) / 3
        cen = (a + bb + c) / 3
        centroids[:, f] = cen
        radii[:, f] = np.maximum(np.maximum(np.linalg.norm(a - cen, axis=1),
                                            np.linalg.norm(bb - cen, axis=1)),
                                 np.linalg.norm(c - cen, axis=1))

    # face neighbours (periodic faces match after identifying opposite vertices)
    canon = np.arange(V, dtype=np.int64)
    per_axis_of_vertex = np.full(V, -1, dtype=np.int64)
    if periodic.any():
        dims = np.array(cube_dims)
        for ax in range(3):
            if periodic[ax]:
                top = vertex_index[:, ax] == dims[ax]
                partner = vertex_index[top].copy()
                partner[:, ax] = 0
                nx, ny = dims[0], dims[1]
                pid = partner[:, 0] + (nx + 1) * (partner[:, 1] + (ny + 1) * partner[:, 2])
                canon[top] = canon[pid]
                per_axis_of_vertex[top] = ax
    fv = np.stack([elements[:, list(f)] for f in FACE_VERTICES], axis=1)  # [E,4,3]
    fkey_v = np.sort(canon[fv], axis=2)
    key = (fkey_v[..., 0] * (V + 1) + fkey_v[..., 1]) * (V + 1) + fkey_v[..., 2]
    key = key.ravel()
    order = np.argsort(key, kind="stable")
    ks = key[order]
    neighbors = np.full(E * 4, INVALID_ELEMENT, dtype=np.uint32)
    axes = np.full(E * 4, INVALID_AXIS, dtype=np.uint32)
    same = ks[1:] == ks[:-1]
    i0 = order[:-1][same]
    i1 = order[1:][same]
    neighbors[i0] = (i1 // 4).astype(np.uint32)
    neighbors[i1] = (i0 // 4).astype(np.uint32)
    if periodic.any():
        # a matched pair is periodic when its raw vertex sets differ
        raw = np.sort(fv.reshape(E * 4, 3), axis=1)
        differs = np.any(raw[i0] != raw[i1], axis=1)
        for a_idx, b_idx in ((i0, i1), (i1, i0)):
            sel = a_idx[differs]
            oth = b_idx[differs]
            # axis along which the faces differ: the coordinate that is constant
            fp = pts[fv.reshape(E * 4, 3)[sel]]
            fq = pts[fv.reshape(E * 4, 3)[oth]]
            dax = np.argmax(np.abs(fp.mean(axis=1) - fq.mean(axis=1)), axis=1)
            axes[sel] = dax.astype(np.uint32)
    neighbors = neighbors.reshape(E, 4)
    axes = axes.reshape(E, 4)

    # vertex -> element CSR, ascending element id per vertex
    ve = np.stack([elements.ravel(), np.repeat(np.arange(E), 4)], axis=1)
    ord2 = np.lexsort((ve[:, 1], ve[:, 0]))
    ve = ve[ord2]
    counts = np.bincount(ve[:, 0], minlength=V)
    starts = np.zeros(V + 1, dtype=np.uint32)
    starts[1:] = np.cumsum(counts).astype(np.uint32)

    pmin = np.where(periodic, lo, 0.0).astype(np.float64)
    pmax = np.where(periodic, hi, 0.0).astype(np.float64)
    return Mesh(points=np.ascontiguousarray(pts), elements=elements.astype(np.uint32),
                inverse_maps=np.ascontiguousarray(inverse_maps),
                forward_maps=np.ascontiguousarray(forward_maps), jacobians=jac,
                face_normals=normals, face_plane_rhs=rhs, face_centroids=centroids,
                face_radii=radii, face_neighbors=neighbors, face_periodicity_axes=axes,
                vertex_adj_starts=starts,
                vertex_adj_elements=ve[:, 1].astype(np.uint32),
                periodicity_min=pmin, periodicity_max=pmax,
                bbox_min=pts.min(axis=0), bbox_max=pts.max(axis=0),
                cube_dims=tuple(cube_dims))


def element_nodes(mesh: Mesh, order: int) -> np.ndarray:
    """Physical node coordinates, element-contiguous, shape [E*Np, 3]."""
    r = refelement.unit_nodes(order)                    # [Np, 3]
    A = mesh.forward_maps[:, :9].reshape(-1, 3, 3)
    b = mesh.forward_maps[:, 9:]
    x = np.einsum("eij,nj->eni", A, r) + b[:, None, :]
    return np.ascontiguousarray(x.reshape(-1, 3))


def element_bins(mesh: Mesh, bins_per_axis=None, margin_rel=1e-6):
    """Uniform bins over the mesh box, each listing (ascending) every element
    whose bounding box, inflated by ``margin_rel`` of the box size, overlaps it.

    Used to answer the reference's global element search
    (``meshdata.hpp:208-215``: the first, i.e. lowest-id, element whose inverse
    map passes ``is_in_unit_simplex``) without an O(E) scan: the lowest id among
    the bin's elements that pass the same test is the same answer, because the
    bin lists every element that could contain the point. Returns
    (lo[3], inv_h[3], dims[3], starts[nb+1] u32, elements u32).
    """
    E = mesh.element_count
    lo = mesh.bbox_min.astype(np.float64)
    hi = mesh.bbox_max.astype(np.float64)
    size = hi - lo
    if bins_per_axis is None:
        target = max(1, E // 6)
        s = (target / np.prod(size)) ** (1 / 3)
        bins_per_axis = np.maximum(1, np.round(size * s)).astype(np.int64)
    dims = np.asarray(bins_per_axis, dtype=np.int64)
    h = size / dims
    p = mesh.points[mesh.elements]
    margin = margin_rel * np.max(size)
    emin = p.min(axis=1) - margin
    emax = p.max(axis=1) + margin
    b0 = np.clip(np.floor((emin - lo) / h).astype(np.int64), 0, dims - 1)
    b1 = np.clip(np.floor((emax - lo) / h).astype(np.int64), 0, dims - 1)
    cnt = np.prod(b1 - b0 + 1, axis=1)
    total = int(cnt.sum())
    el = np.repeat(np.arange(E, dtype=np.int64), cnt)
    # enumerate the bin boxes
    offs = np.arange(total) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    ext = (b1 - b0 + 1)[el]
    ox = offs % ext[:, 0]
    oy = (offs // ext[:, 0]) % ext[:, 1]
    oz = offs // (ext[:, 0] * ext[:, 1])
    bx = b0[el, 0] + ox
    by = b0[el, 1] + oy
    bz = b0[el, 2] + oz
    bid = bx + dims[0] * (by + dims[1] * bz)
    order = np.lexsort((el, bid))
    bid = bid[order]
    el = el[order]
    nb = int(np.prod(dims))
    starts = np.zeros(nb + 1, dtype=np.uint32)
    starts[1:] = np.cumsum(np.bincount(bid, minlength=nb)).astype(np.uint32)
    return lo, 1.0 / h, dims.astype(np.int32), starts, el.astype(np.uint32)
