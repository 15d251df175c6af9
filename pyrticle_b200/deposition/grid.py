"""Grid depositor: deposit onto brick grids, then remap element by element
onto the DG nodes (the reference's ``deposition/grid.py``, ``dep_grid.hpp``,
``dep_grid_base.hpp`` and ``grid.hpp``).

Set-up (host, numpy, batched over elements) follows the reference's
``prepare_with_pointwise_projection_and_basis_reduction`` (grid.py:552-669):
per element, the grid points inside the element (grown by ``el_tolerance``
times the norm of the element map, dep_grid.hpp:142-213) weighted by
sqrt(cell volume), the weighted orthonormal Vandermonde on them, and a
basis reduction that drops the highest-degree mode with the largest weight
in the last right singular vector while the system is underdetermined or its
condition number exceeds 10. The remap matrix is
``I_e = V_e[:, basis] pinv(W V_struct[:, basis])`` (grid.py:217-273).
"""

from __future__ import annotations

import ctypes as C

import os

import numpy as np
import torch

from .. import _lib, refelement
from . import Depositor
from .grid_base import SingleBrickGenerator


class BrickInfo:
    """One brick (grid.hpp:159-340): cell-centred points, x-fastest numbering."""

    def __init__(self, number, start_index, stepwidths, origin, dims):
        stepwidths = np.array(stepwidths, dtype=np.float64)
        origin = np.array(origin, dtype=np.float64)
        dims = np.array(dims, dtype=np.int64)
        neg = stepwidths < 0
        stepwidths[neg] *= -1
        origin[neg] -= stepwidths[neg] * dims[neg]
        if (dims <= 0).any():
            raise ValueError("zero dimensions for brick not supported")
        self.number = number
        self.start_index = int(start_index)
        self.stepwidths = stepwidths
        self.origin = origin
        self.dims = dims
        self.strides = np.array([1, dims[0], dims[0] * dims[1]], dtype=np.int64)

    def __len__(self):
        return int(np.prod(self.dims))

    def node_count(self):
        return len(self)

    def cell_volume(self):
        return float(np.prod(self.stepwidths))

    def bounding_box(self):
        return self.origin, self.origin + self.dims * self.stepwidths

    def point(self, idx):
        return self.origin + self.stepwidths / 2 + np.asarray(idx) * self.stepwidths

    def index(self, idx):
        return self.start_index + int(np.dot(idx, self.strides))

    def as_struct(self) -> _lib.Brick:
        b = _lib.Brick()
        for a in range(3):
            b.origin[a] = self.origin[a]
            b.stepwidths[a] = self.stepwidths[a]
            b.dims[a] = int(self.dims[a])
        b.start_index = self.start_index
        return b


class MT19937:
    """The 32-bit Mersenne Twister (Matsumoto and Nishimura, 1998), the
    engine of the reference's jiggly bricks (boost::mt19937, default seed
    5489). Known answer: the 10000th output from the default seed is
    4123659995."""

    def __init__(self, seed=5489):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            prev = self.mt[i - 1]
            self.mt[i] = (1812433253 * (prev ^ (prev >> 30)) + i) & 0xFFFFFFFF
        self.index = 624

    def _twist(self):
        mt = self.mt
        for i in range(624):
            y = (mt[i] & 0x80000000) | (mt[(i + 1) % 624] & 0x7FFFFFFF)
            v = mt[(i + 397) % 624] ^ (y >> 1)
            if y & 1:
                v ^= 0x9908B0DF
            mt[i] = v
        self.index = 0

    def __call__(self):
        if self.index >= 624:
            self._twist()
        y = self.mt[self.index]
        self.index += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


def uniform_real(engine, lo, hi):
    """boost::uniform_real<>(lo, hi) over a 32-bit engine:
    lo + (hi - lo) * k / 2^32 for the engine's output k."""
    return float(engine()) / 4294967296.0 * (hi - lo) + lo


class JigglyBrickInfo(BrickInfo):
    """A brick whose points are jittered (grid.hpp:345-449): three point
    origins origin + h/2 + offset_i, offset_i = U(-r, r) * h per axis drawn
    from a fresh MT19937 (i outer, axis inner), and point idx taking origin
    (i + j + k) % 3. Every brick draws the same offsets (in cell units).

    The reference's jiggly iterator advances along x by the offset of the
    origin after the next one, so the points it visits along a row depend on
    where the row starts; this build uses point(idx) everywhere (setup and
    deposition), which is the brick's own definition of its points."""

    def __init__(self, number, start_index, stepwidths, origin, dims, jiggle_radius):
        BrickInfo.__init__(self, number, start_index, stepwidths, origin, dims)
        if not 0 < jiggle_radius <= 0.5:
            # beyond half a cell a point can leave its cell, and the index
            # ranges the reference walks would miss points within the radius
            raise ValueError("jiggle_radius must be in (0, 0.5]")
        self.jiggle_radius = float(jiggle_radius)
        eng = MT19937()
        oph = self.origin + self.stepwidths / 2
        po = np.empty((3, 3))
        for i in range(3):
            for a in range(3):
                po[i, a] = uniform_real(eng, -jiggle_radius, jiggle_radius) * self.stepwidths[a]
            po[i] = oph + po[i]
        self.point_origins = po

    def point(self, idx):
        idx = np.asarray(idx)
        return self.point_origins[int(idx.sum()) % 3] + idx * self.stepwidths

    def points(self, idx):
        """point() of an [..., 3] index array."""
        idx = np.asarray(idx)
        return self.point_origins[idx.sum(axis=-1) % 3] + idx * self.stepwidths


def find_points_in_elements(mesh, bricks, el_tolerance, chunk=20000):
    """Per element, the grid points within the tolerance-grown element
    (dep_grid.hpp:142-213). Returns (starts[E+1], grid_index, points, weights)."""
    E = mesh.element_count
    A = mesh.forward_maps[:, :9].reshape(E, 3, 3)
    scaled_tol = el_tolerance * np.linalg.norm(A, ord=2, axis=(1, 2))
    p = mesh.points[mesh.elements]
    elo = p.min(axis=1) - scaled_tol[:, None]
    ehi = p.max(axis=1) + scaled_tol[:, None]
    per_el_idx = [[] for _ in range(E)]
    per_el_pts = [[] for _ in range(E)]
    per_el_w = [[] for _ in range(E)]
    counts = np.zeros(E, dtype=np.int64)
    all_idx, all_pts, all_w, all_el = [], [], [], []
    for brk in bricks:
        blo, bhi = brk.bounding_box()
        dV = brk.cell_volume()
        ilo_box = np.maximum(elo, blo)
        ihi_box = np.minimum(ehi, bhi)
        nonempty = np.all(ilo_box < ihi_box, axis=1)
        lo_i = np.floor((ilo_box - brk.origin) / brk.stepwidths).astype(np.int64)
        hi_i = np.ceil((ihi_box - brk.origin) / brk.stepwidths).astype(np.int64)
        ext = np.where(nonempty[:, None], np.maximum(hi_i - lo_i, 0), 0)
        mx = ext.max(axis=0)

        def chunk_points(c0):
            sl = slice(c0, min(E, c0 + chunk))
            ee = np.arange(sl.start, sl.stop)
            ox, oy, oz = np.meshgrid(np.arange(mx[0]), np.arange(mx[1]), np.arange(mx[2]),
                                     indexing="ij")
            # x fastest, like the brick iterator (grid.hpp:104-125)
            off = np.stack([ox.transpose(2, 1, 0).ravel(), oy.transpose(2, 1, 0).ravel(),
                            oz.transpose(2, 1, 0).ravel()], axis=1)      # [K, 3]
            idx = lo_i[sl][:, None, :] + off[None]                          # [e, K, 3]
            valid = np.all(off[None] < ext[sl][:, None, :], axis=2)
            if isinstance(brk, JigglyBrickInfo):
                pts = brk.points(idx)
            else:
                pts = brk.origin + brk.stepwidths / 2 + idx * brk.stepwidths   # [e, K, 3]
            n = mesh.face_normals[sl]                                       # [e, 4, 3]
            rhs = mesh.face_plane_rhs[sl]
            dist = np.einsum("eki,efi->ekf", pts, n) - rhs[:, None, :]
            inside = valid & np.all(dist <= scaled_tol[sl][:, None, None], axis=2)
            e_i, k_i = np.nonzero(inside)                                   # row-major
            gidx = brk.start_index + idx[e_i, k_i] @ brk.strides
            return ee[e_i], gidx, pts[e_i, k_i], np.full(len(e_i), np.sqrt(dV))

        # the element chunks on all host cores, collected in chunk order
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
            for a_el, a_idx, a_pts, a_w in ex.map(chunk_points, range(0, E, chunk)):
                all_el.append(a_el)
                all_idx.append(a_idx)
                all_pts.append(a_pts)
                all_w.append(a_w)
    el = np.concatenate(all_el)
    order = np.argsort(el, kind="stable")   # bricks in order, points in iterator order
    el = el[order]
    gidx = np.concatenate(all_idx)[order]
    pts = np.concatenate(all_pts)[order]
    w = np.concatenate(all_w)[order]
    starts = np.zeros(E + 1, dtype=np.int64)
    starts[1:] = np.cumsum(np.bincount(el, minlength=E))
    return starts, gidx, pts, w


def basis_reduction_matrices(mesh, order, starts, pts, w, max_condition=10.0):
    """Batched basis reduction + pseudoinverse (grid.py:217-273, 552-669).

    Returns per element the column-major Np x P_e interpolation matrix
    (flattened, concatenated) and the kept-mode count."""
    E = mesh.element_count
    modes = refelement.mode_identifiers(order)
    Np = len(modes)
    degree = np.array([sum(m) for m in modes])
    el_vdm = refelement.orthonormal_vandermonde(refelement.unit_nodes(order), modes)
    A_inv = mesh.inverse_maps[:, :9].reshape(E, 3, 3)
    b_inv = mesh.inverse_maps[:, 9:]
    counts = np.diff(starts)
    el_of_pt = np.repeat(np.arange(E), counts)
    unit = np.einsum("pij,pj->pi", A_inv[el_of_pt], pts) + b_inv[el_of_pt]
    vfull = orthonormal_vandermonde_fast(unit, modes) * w[:, None]       # [Ptot, Np]
    mats = [None] * E
    kept = np.zeros(E, dtype=np.int64)
    eps = np.finfo(float).eps

    def reduce_group(P):
        """The elements with P points: basis reduction and pseudoinverse."""
        els = np.nonzero(counts == P)[0]
        if P == 0:
            raise RuntimeError("grid depositor: element %d contains no grid points" % els[0])
        rows = starts[els][:, None] + np.arange(P)[None]                    # [G, P]
        V = vfull[rows]                                                    # [G, P, Np]
        mask = np.ones((len(els), Np), dtype=bool)
        active = np.arange(len(els))
        B = Np
        while len(active):
            cols = np.nonzero(mask[active])[1].reshape(len(active), B)
            Vs = np.take_along_axis(V[active], cols[:, None, :], axis=2)  # [g, P, B]
            u, s, vt = _batched_svd(Vs)
            ratio = np.abs(s[:, 0] / s[:, -1]) if s.shape[1] else np.full(len(active), np.inf)
            retry = (B > P) | ~(ratio <= max_condition)
            done = active[~retry]
            if len(done):
                g = ~retry
                ss = s[g]
                thresh = eps * max(P, B) * ss[:, :1]
                inv_s = np.where(np.abs(ss) >= thresh, 1.0 / np.where(ss == 0, 1, ss), 0.0)
                k = ss.shape[1]
                # V diag(1/s) U^T over the k = min(P, B) singular triplets
                vk = np.transpose(vt[g][:, :k, :], (0, 2, 1))               # [d, B, k]
                uk = u[g][:, :, :k]                                        # [d, P, k]
                pinv = (vk * inv_s[:, None, :]) @ np.transpose(uk, (0, 2, 1))
                ev = el_vdm[:, cols[g]].transpose(1, 0, 2)                  # [d, Np, B]
                imat = ev @ pinv                                            # [d, Np, P]
                for t, gi in enumerate(done):
                    e = els[gi]
                    mats[e] = np.asfortranarray(imat[t]).ravel(order="F")
                    kept[e] = B
            if not retry.any():
                break
            if B == 1:
                raise RuntimeError("basis reduction has killed almost the entire basis on "
                                   "element %d" % els[active[retry][0]])
            ra = active[retry]
            vti = vt[retry][:, -1, :]                                       # [r, B]
            deg = degree[cols[retry]]                                       # [r, B]
            killable = deg == deg.max(axis=1, keepdims=True)
            score = np.where(killable, np.abs(vti), -1.0)
            kill_pos = np.argmax(score, axis=1)                             # first max
            kill_col = cols[retry][np.arange(len(ra)), kill_pos]
            mask[ra, kill_col] = False
            active = ra
            B -= 1

    # the groups are independent: all host cores (LAPACK releases the
    # interpreter lock; each group's results do not depend on the others)
    from concurrent.futures import ThreadPoolExecutor
    sizes = np.unique(counts)
    order = sorted(sizes, key=lambda P: -int(np.count_nonzero(counts == P)) * int(P))
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        for _ in ex.map(reduce_group, order):
            pass
    mstarts = np.zeros(E + 1, dtype=np.int64)
    mstarts[1:] = np.cumsum(counts * Np)
    return np.concatenate(mats), mstarts, kept


def _batched_svd(A):
    """SVD of a batch [g, P, B]. With P >= B the thin U (P x B) suffices: the
    pseudoinverse uses its first B columns only, and V is square either way;
    with P < B the full V is needed (its last row spans the null space the
    mode killing reads)."""
    full = A.shape[1] < A.shape[2]
    try:
        return np.linalg.svd(A, full_matrices=full)
    except np.linalg.LinAlgError:
        outs = [np.linalg.svd(a, full_matrices=full) for a in A]
        return (np.stack([o[0] for o in outs]), np.stack([o[1] for o in outs]),
                np.stack([o[2] for o in outs]))


def orthonormal_vandermonde_fast(points, modes, block=262144):
    """refelement.orthonormal_vandermonde in blocks of points on all host
    cores (row by row the same values)."""
    if len(points) <= block:
        return refelement.orthonormal_vandermonde(points, modes)
    from concurrent.futures import ThreadPoolExecutor
    parts = [points[i:i + block] for i in range(0, len(points), block)]
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return np.concatenate(list(ex.map(
            lambda p: refelement.orthonormal_vandermonde(p, modes), parts)))


def average_groups(mesh, nodes, nodes_per_element, chunk=None):
    """The continuity groups of prepare_average_groups (grid.py:143-183): the
    DG nodes that face pairs identify, merged into connected sets. For every
    interior face (periodic ones included: positions compared modulo the
    period) the nodes of both elements lying on it are matched by position;
    the groups are the connected components of those matches with two or
    more nodes, each in ascending node order. Returns (starts[G+1], nodes)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components

    E, Np = mesh.element_count, nodes_per_element
    X = nodes.reshape(E, Np, 3)
    h = float(np.median(mesh.inradii()))
    tol = 1e-6 * h
    # [E, 4, Np]: node on face f of its element
    dist = np.einsum("enk,efk->efn", X, mesh.face_normals) - mesh.face_plane_rhs[:, :, None]
    on_face = np.abs(dist) <= tol
    nb = mesh.face_neighbors.astype(np.int64)
    inval = np.iinfo(np.uint32).max
    e_idx, f_idx = np.nonzero((nb != inval) & (nb > np.arange(E)[:, None]))
    per = mesh.periodicity_max - mesh.periodicity_min
    # face pairs per chunk: the [F, Np, Np, 3] differences stay near 160 MB
    chunk = chunk or max(1, int(2e7) // (Np * Np))
    rows, cols = [], []
    for c0 in range(0, len(e_idx), chunk):
        e1 = e_idx[c0:c0 + chunk]
        f1 = f_idx[c0:c0 + chunk]
        e2 = nb[e1, f1]
        # the face of e2 that points back at e1
        f2 = np.argmax(mesh.face_neighbors[e2].astype(np.int64) == e1[:, None], axis=1)
        m1 = on_face[e1, f1]                    # [F, Np]
        m2 = on_face[e2, f2]
        d = X[e1][:, :, None, :] - X[e2][:, None, :, :]   # [F, Np, Np, 3]
        for ax in range(3):
            if per[ax] > 0:
                d[..., ax] -= np.round(d[..., ax] / per[ax]) * per[ax]
        close = (np.abs(d).max(axis=-1) <= tol) & m1[:, :, None] & m2[:, None, :]
        fi, a, b = np.nonzero(close)
        rows.append(e1[fi] * Np + a)
        cols.append(e2[fi] * Np + b)
    rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    nn = E * Np
    g = coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(nn, nn))
    ncomp, labels = connected_components(g, directed=False)
    sizes = np.bincount(labels, minlength=ncomp)
    member = sizes[labels] >= 2
    order = np.lexsort((np.arange(nn), labels))     # by group, ascending node inside
    order = order[member[order]]
    lab = labels[order]
    starts = np.concatenate([[0], np.nonzero(np.diff(lab))[0] + 1, [len(order)]])
    return starts.astype(np.uint32), order.astype(np.uint32)


class GridDepositor(Depositor):
    """Deposit on brick grids (shape-function values at the points, or
    trilinear weights with ``grid_weights="trilinear"``), then remap.

    ``precision``: ``"fp64"`` (the reference's arithmetic) or ``"mixed"``
    (the chosen form: the shape-weight grid deposition on the tensor cores,
    split-FP16 scores, 23-bit integer weights, exact int8 sums; shape
    weights with exponent 2 only). The remap is FP64 in both."""

    PRECISIONS = ("fp64", "mixed")

    def __init__(self, brick_generator=None, el_tolerance=0.12, max_extra_points=20,
                 enforce_continuity=False, submethod="simplex_reduce",
                 filter_min_amplification=None, filter_order=None, jiggle_radius=0.0,
                 grid_weights="shape", precision="fp64"):
        Depositor.__init__(self)
        if precision not in self.PRECISIONS:
            raise ValueError(f"precision must be one of {self.PRECISIONS}")
        self.precision = precision
        self.brick_generator = brick_generator or SingleBrickGenerator()
        self.el_tolerance = el_tolerance
        self.max_extra_points = max_extra_points
        self.enforce_continuity = enforce_continuity
        self.submethod = submethod
        if submethod != "simplex_reduce":
            raise NotImplementedError("only submethod='simplex_reduce' (the reference default)")
        if filter_min_amplification is not None:
            raise NotImplementedError("DG filters are not supported")
        if grid_weights not in ("shape", "trilinear"):
            raise ValueError("grid_weights must be 'shape' or 'trilinear'")
        if jiggle_radius and grid_weights != "shape":
            raise ValueError("trilinear weights need the regular cell-centred points")
        self.jiggle_radius = jiggle_radius
        self.grid_weights = grid_weights

    @property
    def name(self):
        return "GridJiggly" if self.jiggle_radius else "GridRegular"

    def initialize(self, method):
        Depositor.initialize(self, method)
        discr = method.discretization
        self.bricks = []
        start = 0
        for i, (sw, origin, dims) in enumerate(self.brick_generator(discr)):
            if self.jiggle_radius:
                b = JigglyBrickInfo(i, start, sw, origin, dims, self.jiggle_radius)
            else:
                b = BrickInfo(i, start, sw, origin, dims)
            self.bricks.append(b)
            start += len(b)
        self.grid_node_count = start
        starts, gidx, pts, w = find_points_in_elements(discr.mesh, self.bricks,
                                                       self.el_tolerance)
        mats, mstarts, kept = basis_reduction_matrices(discr.mesh, discr.order, starts, pts, w)
        self.eog = dict(starts=starts, grid_nodes=gidx, weights=w, matrices=mats,
                        matrix_starts=mstarts, kept=kept)
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a

        d = _lib.GridDesc()
        d.brick_count = len(self.bricks)
        d.nodes_per_element = discr.nodes_per_element
        barr = (_lib.Brick * len(self.bricks))(*[b.as_struct() for b in self.bricks])
        keep.append(barr)
        d.bricks = C.cast(barr, C.POINTER(_lib.Brick))
        E = discr.mesh.element_count
        d.eog_count = E
        d.eog_elements = _lib.ptr(arr(np.arange(E), np.uint32), C.c_uint32)
        d.eog_starts = _lib.ptr(arr(starts, np.uint64), C.c_uint64)
        d.eog_grid_nodes = _lib.ptr(arr(gidx, np.uint32), C.c_uint32)
        d.eog_weights = _lib.ptr(arr(w, np.float64))
        d.eog_matrix_starts = _lib.ptr(arr(mstarts, np.uint64), C.c_uint64)
        d.eog_matrices = _lib.ptr(arr(mats, np.float64))
        d.avg_group_count = 0
        if self.enforce_continuity:
            ag_starts, ag_nodes = average_groups(discr.mesh, np.asarray(discr.nodes),
                                                 discr.nodes_per_element)
            self.average_group_starts, self.average_groups = ag_starts, ag_nodes
            d.avg_group_count = len(ag_starts) - 1
            d.avg_group_starts = _lib.ptr(arr(ag_starts, np.uint32), C.c_uint32)
            d.avg_group_nodes = _lib.ptr(arr(ag_nodes, np.uint32), C.c_uint32)
        if self.jiggle_radius:
            d.point_origins = _lib.ptr(arr(np.stack([b.point_origins for b in self.bricks]),
                                           np.float64))
        self.grid_desc = d
        self._keep = keep
        h = C.c_void_p()
        _lib.check(self.lib.prt_grid_create(method.mesh_data.handle, C.byref(d), C.byref(h)),
                   "prt_grid_create")
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) is not None and _lib._lib is not None:
            _lib._lib.prt_grid_destroy(self.handle)
            self.handle = None

    def grid_node_count_with_extra(self):
        return self.grid_node_count

    def _shape_desc(self):
        sf = self.shape_function
        if sf is None:
            return _lib.ShapeFunctionDesc(0.0, 2.0, 0.0)
        return _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer)

    def deposit_grid_densities_device(self, state, rho=True, j=True):
        if self.grid_weights == "shape":
            self.deposit_hook()
        m = self.method
        G = self.grid_node_count
        dev = state.x.device
        gr = torch.empty((G,), dtype=torch.float64, device=dev) if rho else None
        gj = torch.empty((3, G), dtype=torch.float64, device=dev) if j else None
        v = m.velocities_device(state) if j else None
        if self.precision == "mixed":
            if self.grid_weights != "shape" or self.shape_function is None or \
                    self.shape_function.exponent != 2:
                raise ValueError("the mixed grid deposition needs shape weights with exponent 2")
            _lib.check(self.lib.prt_deposit_grid_mixed(
                self.handle, m.workspace, self._shape_desc(), len(state),
                state.x.data_ptr(), state.q.data_ptr(), v.data_ptr() if v is not None else None,
                state.el.data_ptr(), gr.data_ptr() if rho else None,
                gj.data_ptr() if j else None, self._stream()), "prt_deposit_grid_mixed")
            return gr, gj
        wmode = _lib.GRID_SHAPE if self.grid_weights == "shape" else _lib.GRID_TRILINEAR
        _lib.check(self.lib.prt_deposit_grid(
            self.handle, m.workspace, wmode, self._shape_desc(), len(state),
            state.x.data_ptr(), state.q.data_ptr(), v.data_ptr() if v is not None else None,
            state.el.data_ptr(), gr.data_ptr() if rho else None,
            gj.data_ptr() if j else None, self._stream()), "prt_deposit_grid")
        return gr, gj

    def remap_grid_to_mesh_device(self, q_grid: torch.Tensor) -> torch.Tensor:
        """[G] -> [Nn]; [3, G] -> [3, Nn] (each component remapped)."""
        nn = len(self.method.discretization)
        if q_grid.dim() == 1:
            out = torch.zeros((nn,), dtype=torch.float64, device=q_grid.device)
            _lib.check(self.lib.prt_remap_grid_to_mesh(self.handle, q_grid.data_ptr(),
                                                       out.data_ptr(), 0, 1, self._stream()))
            return out
        out = torch.zeros((q_grid.shape[0], nn), dtype=torch.float64, device=q_grid.device)
        q = q_grid.contiguous()
        for c0 in range(0, q.shape[0], 4):
            k = min(4, q.shape[0] - c0)
            _lib.check(self.lib.prt_remap_grid_to_mesh_components(
                self.handle, q[c0].data_ptr(), out[c0].data_ptr(), k, self._stream()))
        return out

    def deposit_densities_device(self, state, rho=True, j=True):
        gr, gj = self.deposit_grid_densities_device(state, rho, j)
        if rho and j:
            # rho and the three j components in one remap pass
            out = self.remap_grid_to_mesh_device(torch.cat([gr[None], gj]))
            return out[0], out[1:]
        r = self.remap_grid_to_mesh_device(gr) if rho else None
        jj = self.remap_grid_to_mesh_device(gj) if j else None
        return r, jj

    # host entry points with the reference's names
    def deposit_grid_rho(self, state, pslice=None):
        return self.deposit_grid_densities_device(state, True, False)[0].cpu().numpy()

    def deposit_grid_j(self, state, velocities=None, pslice=None):
        return self.deposit_grid_densities_device(state, False, True)[1].T.contiguous().cpu().numpy()

    def deposit_grid_densities(self, state, velocities=None, pslice=None):
        """(rho_grid [G], j_grid [G, 3]) in one pass (grid.py:820-829)."""
        gr, gj = self.deposit_grid_densities_device(state, True, True)
        return gr.cpu().numpy(), gj.T.contiguous().cpu().numpy()

    # grid debug quantities (grid.py:848-858)
    def ones_on_grid(self):
        return np.ones((self.grid_node_count_with_extra(),), dtype=float)

    def grid_usecount(self):
        """How many elements' interpolation uses each grid point."""
        return np.bincount(np.asarray(self.eog["grid_nodes"], dtype=np.int64),
                           minlength=self.grid_node_count_with_extra()).astype(float)

    def remap_grid_to_mesh(self, q_grid):
        t = torch.as_tensor(np.ascontiguousarray(q_grid), device=self.method.dev)
        if t.dim() == 2:
            t = t.T.contiguous()
            return self.remap_grid_to_mesh_device(t).T.contiguous().cpu().numpy()
        return self.remap_grid_to_mesh_device(t).cpu().numpy()
