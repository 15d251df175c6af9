"""ctypes wrapper of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU
baseline of bench.py as the checker. The product (pyrticle_b200) never
imports this module. Arrays follow the reference layout: positions and
momenta [n, 3], j [Nn, 3].
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from pyrticle_b200 import _lib as L

HERE = Path(__file__).resolve().parent
SERIAL = HERE / "_build" / "liboracle.so"
PARALLEL = HERE / "_build" / "liboracle_omp.so"

_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_i64p = C.POINTER(C.c_int64)

_libs: dict = {}


def build() -> None:
    subprocess.run(["make", "-C", str(HERE)], check=True, stdout=subprocess.DEVNULL)


def lib(parallel: bool = False) -> C.CDLL:
    path = PARALLEL if parallel else SERIAL
    if path in _libs:
        return _libs[path]
    if not path.exists():
        build()
    h = C.CDLL(str(path))
    md = C.POINTER(L.MeshDesc)
    h.orc_get_velocities.argtypes = [C.c_int64, _dp, _dp, C.c_double, _dp]
    h.orc_find_containing_elements.argtypes = [md, C.c_int64, _dp, _u32p, C.c_int]
    h.orc_update_containing_elements.argtypes = [md, _i64p, _dp, _dp, _dp, _dp, _u32p, _dp,
                                                 _dp, _i64p, C.POINTER(L.FindCounters),
                                                 C.c_int]
    h.orc_pusher_create.restype = C.c_void_p
    h.orc_pusher_create.argtypes = [C.c_int, _u32p, _dp]
    h.orc_pusher_destroy.argtypes = [C.c_void_p]
    h.orc_forces.argtypes = [C.c_void_p, md, C.c_int64, _dp, _u32p, _dp, _dp] + [_dp] * 6 + [_dp, _dp]
    h.orc_lsrk_steps.argtypes = [C.c_void_p, md, _i64p, _dp, _dp, _dp, _dp, _u32p, _dp, _dp,
                                 _i64p, C.POINTER(_dp), C.c_int, _dp, _dp, C.c_double,
                                 C.c_double, C.c_int, C.POINTER(L.FindCounters), C.c_int]
    h.orc_deposit_shape.restype = C.c_int64
    h.orc_deposit_shape.argtypes = [md, C.c_int, L.ShapeFunctionDesc, _dp, C.c_int64, _dp, _dp,
                                    _dp, _u32p, _dp, _dp, _dp]
    h.orc_walk_elements.argtypes = [md, _dp, C.c_uint32, C.c_double, _u32p, C.c_int]
    h.orc_deposit_grid.argtypes = [md, C.c_int, C.POINTER(L.Brick), _dp, C.c_int,
                                   L.ShapeFunctionDesc, C.c_int64, _dp, _dp, _dp, C.c_int64,
                                   _dp, _dp, _u32p]
    h.orc_deposit_grid_find.argtypes = [md, C.c_int, C.POINTER(L.Brick), _u32p, _u32p, _dp,
                                        C.c_int64, L.ShapeFunctionDesc, C.c_int64, _dp, _dp,
                                        _dp, _dp, _dp, _u32p]
    h.orc_remap_grid_to_mesh.argtypes = [C.POINTER(L.GridDesc), _dp, _dp, C.c_int64, C.c_int64]
    h.orc_pic_steps_parallel.argtypes = [C.c_void_p, md, C.c_int64, _dp, _dp, _dp, _dp, _u32p,
                                         _dp, _dp, C.POINTER(_dp), C.c_int, _dp, _dp,
                                         C.c_double, C.c_double, C.c_int, L.ShapeFunctionDesc,
                                         _dp, _dp, C.c_int]
    h.orc_max_threads.restype = C.c_int
    _libs[path] = h
    return h


def _p(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class OracleMesh:
    """Mesh tables held for the oracle (host)."""

    def __init__(self, mesh, nodes, bins):
        self.keep: list = []
        self.mesh = mesh
        self.nodes = np.ascontiguousarray(nodes)
        self.desc = L.mesh_desc(mesh, self.nodes, bins, self.keep)
        self.np = len(nodes) // mesh.element_count

    @property
    def ref(self):
        return C.byref(self.desc)


def velocities(p, m, c):
    p = np.ascontiguousarray(p, dtype=np.float64)
    v = np.empty_like(p)
    lib().orc_get_velocities(len(p), _p(p), _p(np.ascontiguousarray(m, dtype=np.float64)), c, _p(v))
    return v


def find_containing_elements(om: OracleMesh, x, linear=True):
    x = np.ascontiguousarray(x, dtype=np.float64)
    el = np.empty(len(x), dtype=np.uint32)
    lib().orc_find_containing_elements(om.ref, len(x), _p(x), _p(el, C.c_uint32), int(linear))
    return el


def update_containing_elements(om: OracleMesh, x, p, q, m, el, kx=None, kp=None, ids=None,
                               linear_global=False):
    """In place on copies; returns (n, x, p, q, m, el, kx, kp, ids, counters, rc)."""
    x, p = x.copy(), p.copy()
    q, m, el = q.copy(), m.copy(), el.copy()
    kx = None if kx is None else kx.copy()
    kp = None if kp is None else kp.copy()
    ids = np.arange(len(x), dtype=np.int64) if ids is None else ids.copy()
    n = C.c_int64(len(x))
    ctr = L.FindCounters()
    rc = lib().orc_update_containing_elements(om.ref, C.byref(n), _p(x), _p(p), _p(q), _p(m),
                                              _p(el, C.c_uint32), _p(kx), _p(kp),
                                              _p(ids, C.c_int64), C.byref(ctr), int(linear_global))
    k = n.value
    return dict(n=k, x=x[:k], p=p[:k], q=q[:k], m=m[:k], el=el[:k],
                kx=None if kx is None else kx[:k], kp=None if kp is None else kp[:k],
                ids=ids[:k], counters=ctr, rc=rc)


class OraclePusher:
    """Monomial pusher set-up; `parallel` selects the library it lives in."""

    def __init__(self, order_exponents, vandermonde, parallel=False):
        ex = np.ascontiguousarray(order_exponents, dtype=np.uint32)
        v = np.ascontiguousarray(vandermonde, dtype=np.float64)
        self.lib = lib(parallel)
        self.h = self.lib.orc_pusher_create(len(ex), _p(ex, C.c_uint32), _p(v))
        if not self.h:
            raise RuntimeError("singular Vandermonde")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_pusher_destroy(self.h)
            self.h = None


def forces(pusher: OraclePusher, om: OracleMesh, x, el, q, v, fields, vis=False):
    x = np.ascontiguousarray(x)
    n = len(x)
    out = np.empty((n, 3))
    visarr = np.empty((4, n, 3)) if vis else None
    f = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in fields]
    lib().orc_forces(pusher.h, om.ref, n, _p(x), _p(np.ascontiguousarray(el, dtype=np.uint32), C.c_uint32),
                     _p(np.ascontiguousarray(q)), _p(np.ascontiguousarray(v)),
                     *[_p(a) for a in f], _p(out), _p(visarr))
    return (out, visarr) if vis else out


def lsrk_steps(pusher, om, x, p, q, m, el, fields, rk_a, rk_b, dt, c, steps, kx=None,
               kp=None, ids=None, linear_global=False):
    n0 = len(x)
    x, p, q, m, el = (np.ascontiguousarray(a).copy() for a in (x, p, q, m, el))
    kx = np.zeros((n0, 3)) if kx is None else kx.copy()
    kp = np.zeros((n0, 3)) if kp is None else kp.copy()
    ids = np.arange(n0, dtype=np.int64) if ids is None else ids.copy()
    f = [np.ascontiguousarray(a, dtype=np.float64) for a in fields]
    farr = (_dp * 6)(*[_p(a) for a in f])
    ca = np.ascontiguousarray(rk_a, dtype=np.float64)
    cb = np.ascontiguousarray(rk_b, dtype=np.float64)
    n = C.c_int64(n0)
    ctr = L.FindCounters()
    rc = lib().orc_lsrk_steps(pusher.h, om.ref, C.byref(n), _p(x), _p(p), _p(q), _p(m),
                              _p(el, C.c_uint32), _p(kx), _p(kp), _p(ids, C.c_int64), farr,
                              len(ca), _p(ca), _p(cb), dt, c, steps, C.byref(ctr),
                              int(linear_global))
    k = n.value
    return dict(n=k, x=x[:k], p=p[:k], q=q[:k], m=m[:k], el=el[:k], kx=kx[:k], kp=kp[:k],
                ids=ids[:k], counters=ctr, rc=rc)


def deposit_shape(om: OracleMesh, mode, shape, x, q, v, el, integral_weights=None,
                  rho=True, j=True):
    nn = om.mesh.element_count * om.np
    r = np.empty(nn) if rho else None
    jj = np.empty((nn, 3)) if j else None
    stats = np.zeros(15)
    iw = None if integral_weights is None else np.ascontiguousarray(integral_weights, dtype=np.float64)
    sd = L.ShapeFunctionDesc(shape.radius, shape.alpha, shape.normalizer)
    zm = lib().orc_deposit_shape(om.ref, mode, sd, _p(iw), len(x),
                                 _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(q)),
                                 _p(None if v is None else np.ascontiguousarray(v)),
                                 _p(np.ascontiguousarray(el, dtype=np.uint32), C.c_uint32),
                                 _p(r), _p(jj), _p(stats))
    return r, jj, stats, zm


def walk_elements(om: OracleMesh, pos, start, radius, cap=100000):
    out = np.empty(cap, dtype=np.uint32)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    cnt = lib().orc_walk_elements(om.ref, _p(pos), int(start), radius, _p(out, C.c_uint32), cap)
    return out[:min(cnt, cap)]


def deposit_grid(om: OracleMesh, bricks, weights, shape, x, q, v, gnc, rho=True, j=True,
                 brick_cache=None, point_origins=None):
    """point_origins: [bricks, 3, 3] for jiggly bricks, or None."""
    arr = (L.Brick * len(bricks))(*bricks)
    r = np.empty(gnc) if rho else None
    jj = np.empty((gnc, 3)) if j else None
    cache = np.zeros(len(x), dtype=np.uint32) if brick_cache is None else brick_cache
    sd = L.ShapeFunctionDesc(shape.radius, shape.alpha, shape.normalizer)
    po = None if point_origins is None else np.ascontiguousarray(point_origins, dtype=np.float64)
    lib().orc_deposit_grid(om.ref, len(bricks), arr, _p(po), weights, sd, len(x),
                           _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(q)),
                           _p(None if v is None else np.ascontiguousarray(v)), gnc, _p(r), _p(jj),
                           _p(cache, C.c_uint32))
    return r, jj


def deposit_grid_find(om: OracleMesh, bricks, cell_starts, cell_nodes, nodes, shape, x, q, v,
                      rho=True, j=True, brick_cache=None):
    """GridFindDepositor: rho [Nn], j [Nn, 3] through the brick cells' node
    lists (cell_starts [G+1], cell_nodes)."""
    arr = (L.Brick * len(bricks))(*bricks)
    nn = len(nodes)
    r = np.empty(nn) if rho else None
    jj = np.empty((nn, 3)) if j else None
    cache = np.zeros(len(x), dtype=np.uint32) if brick_cache is None else brick_cache
    sd = L.ShapeFunctionDesc(shape.radius, shape.alpha, shape.normalizer)
    cs = np.ascontiguousarray(cell_starts, dtype=np.uint32)
    cn = np.ascontiguousarray(cell_nodes, dtype=np.uint32)
    lib().orc_deposit_grid_find(om.ref, len(bricks), arr, _p(cs, C.c_uint32), _p(cn, C.c_uint32),
                                _p(np.ascontiguousarray(nodes, dtype=np.float64)), nn, sd, len(x),
                                _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(q)),
                                _p(None if v is None else np.ascontiguousarray(v)), _p(r), _p(jj),
                                _p(cache, C.c_uint32))
    return r, jj


def remap_grid_to_mesh(grid_desc, from_vec, to_vec, offset=0, increment=1):
    lib().orc_remap_grid_to_mesh(C.byref(grid_desc), _p(from_vec), _p(to_vec), offset, increment)
    return to_vec


def pic_steps_parallel(pusher, om, x, p, q, m, el, fields, rk_a, rk_b, dt, c, steps, shape,
                       threads=0):
    """Multi-core baseline: `steps` LSRK steps + one rho/j deposition each."""
    n = len(x)
    x, p, q, m, el = (np.ascontiguousarray(a).copy() for a in (x, p, q, m, el))
    kx = np.zeros((n, 3))
    kp = np.zeros((n, 3))
    f = [np.ascontiguousarray(a, dtype=np.float64) for a in fields]
    farr = (_dp * 6)(*[_p(a) for a in f])
    nn = om.mesh.element_count * om.np
    rho = np.empty(nn)
    j = np.empty((nn, 3))
    ca = np.ascontiguousarray(rk_a, dtype=np.float64)
    cb = np.ascontiguousarray(rk_b, dtype=np.float64)
    sd = L.ShapeFunctionDesc(shape.radius, shape.alpha, shape.normalizer)
    h = lib(parallel=True)
    assert pusher.lib is h, "create the pusher with parallel=True"
    rc = h.orc_pic_steps_parallel(pusher.h, om.ref, n, _p(x), _p(p), _p(q), _p(m),
                                  _p(el, C.c_uint32), _p(kx), _p(kp), farr, len(ca), _p(ca),
                                  _p(cb), dt, c, steps, sd, _p(rho), _p(j), threads)
    return dict(x=x, p=p, el=el, rho=rho, j=j, rc=rc)


def max_threads() -> int:
    return lib(parallel=True).orc_max_threads()
