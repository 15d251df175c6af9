"""Reference tetrahedron: interpolation nodes, monomial and orthonormal bases.

The reference element is the simplex with vertices (-1,-1,-1), (1,-1,-1),
(-1,1,-1), (-1,-1,1), the same unit element the reference's mesh layer maps
every tetrahedron onto (``meshdata.hpp:38-48`` tests membership in it).

Everything here replaces pieces of the un-vendored ``hedge`` package that the
reference calls during set-up (``pusher.py:95-109`` uses ``node_tuples``,
``unit_nodes`` and ``generic_vandermonde``; ``shape.py:64-69`` the mass
matrix; ``grid.py:207-273`` the orthonormal ``basis_functions`` and
``vandermonde``). They are written from the published methods:

* nodes: Warburton (2006), "An explicit construction of interpolation nodes
  on the simplex" (warp & blend), as given in Hesthaven & Warburton,
  *Nodal Discontinuous Galerkin Methods* (2008), section 6.2;
* orthonormal basis: the Proriol-Koornwinder-Dubiner-Owens polynomials in
  collapsed coordinates (same book, section 6.1).

All of it is host-side numpy set-up; nothing here runs per time step.
"""

from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

import numpy as np


def node_tuples(order: int) -> list[tuple[int, int, int]]:
    """Index tuples (i, j, k), i + j + k <= order, i fastest.

    These double as the monomial exponents of the reference's monomial
    pusher (``pusher.py:104-105``: one ``MonomialBasisFunction`` per node
    tuple) and as the orthonormal-mode identifiers of the grid depositor
    (``grid.py:571-577``).
    """
    return [(i, j, k)
            for k in range(order + 1)
            for j in range(order + 1 - k)
            for i in range(order + 1 - j - k)]


def node_count(order: int) -> int:
    return (order + 1) * (order + 2) * (order + 3) // 6


def mode_identifiers(order: int) -> list[tuple[int, int, int]]:
    """Orthonormal-mode identifiers (i, j, k), i outermost (Vandermonde3D order)."""
    return [(i, j, k)
            for i in range(order + 1)
            for j in range(order + 1 - i)
            for k in range(order + 1 - i - j)]


# --- 1D helpers -------------------------------------------------------------

def gauss_lobatto_nodes(order: int) -> np.ndarray:
    """Legendre-Gauss-Lobatto nodes on [-1, 1], ascending."""
    if order == 1:
        return np.array([-1.0, 1.0])
    from numpy.polynomial import legendre
    c = np.zeros(order + 1)
    c[order] = 1.0
    interior = np.sort(legendre.legroots(legendre.legder(c)).real)
    return np.concatenate([[-1.0], interior, [1.0]])


def jacobi_p(x: np.ndarray, alpha: float, beta: float, n: int) -> np.ndarray:
    """Orthonormal Jacobi polynomial P_n^(alpha,beta) on [-1, 1]."""
    x = np.asarray(x, dtype=np.float64)
    gamma0 = (2.0 ** (alpha + beta + 1) / (alpha + beta + 1)
              * math.gamma(alpha + 1) * math.gamma(beta + 1)
              / math.gamma(alpha + beta + 1))
    p_prev = np.full_like(x, 1.0 / math.sqrt(gamma0))
    if n == 0:
        return p_prev
    gamma1 = (alpha + 1) * (beta + 1) / (alpha + beta + 3) * gamma0
    p_cur = ((alpha + beta + 2) * x / 2 + (alpha - beta) / 2) / math.sqrt(gamma1)
    if n == 1:
        return p_cur
    a_old = 2 / (2 + alpha + beta) * math.sqrt(
        (alpha + 1) * (beta + 1) / (alpha + beta + 3))
    for i in range(1, n):
        h1 = 2 * i + alpha + beta
        a_new = 2 / (h1 + 2) * math.sqrt(
            (i + 1) * (i + 1 + alpha + beta) * (i + 1 + alpha) * (i + 1 + beta)
            / (h1 + 1) / (h1 + 3))
        b_new = -(alpha ** 2 - beta ** 2) / h1 / (h1 + 2)
        p_next = (-a_old * p_prev + (x - b_new) * p_cur) / a_new
        p_prev, p_cur = p_cur, p_next
        a_old = a_new
    return p_cur


# --- warp & blend nodes -----------------------------------------------------

_ALPHA_OPT = [0.0, 0.0, 0.0, 0.1002, 1.1332, 1.5608, 1.3413, 1.2577, 1.1603,
              1.10153, 0.6080, 0.4523, 0.8856, 0.8717, 0.9655]


def _equidistant_rst(order: int) -> np.ndarray:
    return np.array([[-1 + 2 * i / order, -1 + 2 * j / order, -1 + 2 * k / order]
                     for (i, j, k) in node_tuples(order)])


def _eval_warp(p: int, xnodes: np.ndarray, xout: np.ndarray) -> np.ndarray:
    """1D warp: interpolant of (GLL - equidistant) displacement."""
    warp = np.zeros_like(xout)
    xeq = np.array([-1 + 2 * (p - i) / p for i in range(p + 1)])
    for i in range(p + 1):
        d = np.full_like(xout, xnodes[i] - xeq[i])
        for j in range(1, p):
            if i != j:
                d = d * (xout - xeq[j]) / (xeq[i] - xeq[j])
        if i != 0:
            d = -d / (xeq[i] - xeq[0])
        if i != p:
            d = d / (xeq[i] - xeq[p])
        warp = warp + d
    return warp


def _eval_shift(p, pval, l1, l2, l3):
    gauss_x = -gauss_lobatto_nodes(p)
    warp1 = _eval_warp(p, gauss_x, l3 - l2)
    warp2 = _eval_warp(p, gauss_x, l1 - l3)
    warp3 = _eval_warp(p, gauss_x, l2 - l1)
    blend1 = 4 * l2 * l3
    blend2 = 4 * l1 * l3
    blend3 = 4 * l1 * l2
    wf1 = blend1 * warp1 * (1 + (pval * l1) ** 2)
    wf2 = blend2 * warp2 * (1 + (pval * l2) ** 2)
    wf3 = blend3 * warp3 * (1 + (pval * l3) ** 2)
    dx = wf1 + math.cos(2 * math.pi / 3) * wf2 + math.cos(4 * math.pi / 3) * wf3
    dy = math.sin(2 * math.pi / 3) * wf2 + math.sin(4 * math.pi / 3) * wf3
    return dx, dy


_V1 = np.array([-1.0, -1 / math.sqrt(3), -1 / math.sqrt(6)])
_V2 = np.array([1.0, -1 / math.sqrt(3), -1 / math.sqrt(6)])
_V3 = np.array([0.0, 2 / math.sqrt(3), -1 / math.sqrt(6)])
_V4 = np.array([0.0, 0.0, 3 / math.sqrt(6)])


def _xyz_to_rst(xyz: np.ndarray) -> np.ndarray:
    rhs = xyz - 0.5 * (_V2 + _V3 + _V4 - _V1)
    a = np.column_stack([0.5 * (_V2 - _V1), 0.5 * (_V3 - _V1), 0.5 * (_V4 - _V1)])
    return np.linalg.solve(a, rhs.T).T


@lru_cache(maxsize=None)
def _unit_nodes_cached(order: int) -> bytes:
    if order == 0:
        return np.array([[-0.5, -0.5, -0.5]]).tobytes()
    alpha = _ALPHA_OPT[order - 1] if order <= 15 else 1.0
    tol = 1e-10
    rst = _equidistant_rst(order)
    r, s, t = rst[:, 0], rst[:, 1], rst[:, 2]
    l1 = (1 + t) / 2
    l2 = (1 + s) / 2
    l3 = -(1 + r + s + t) / 2
    l4 = (1 + r) / 2
    t1 = np.array([_V2 - _V1, _V2 - _V1, _V3 - _V2, _V3 - _V1])
    t2 = np.array([_V3 - 0.5 * (_V1 + _V2), _V4 - 0.5 * (_V1 + _V2),
                   _V4 - 0.5 * (_V2 + _V3), _V4 - 0.5 * (_V1 + _V3)])
    t1 /= np.linalg.norm(t1, axis=1)[:, None]
    t2 /= np.linalg.norm(t2, axis=1)[:, None]
    xyz = np.outer(l3, _V1) + np.outer(l4, _V2) + np.outer(l2, _V3) + np.outer(l1, _V4)
    shift = np.zeros_like(xyz)
    faces = [(l1, l2, l3, l4), (l2, l1, l3, l4), (l3, l1, l4, l2), (l4, l1, l3, l2)]
    for face, (la, lb, lc, ld) in enumerate(faces):
        warp1, warp2 = _eval_shift(order, alpha, lb, lc, ld)
        blend = lb * lc * ld
        denom = (lb + 0.5 * la) * (lc + 0.5 * la) * (ld + 0.5 * la)
        ids = denom > tol
        blend[ids] = (1 + (alpha * la[ids]) ** 2) * blend[ids] / denom[ids]
        shift += np.outer(blend * warp1, t1[face]) + np.outer(blend * warp2, t2[face])
        ids = (la < tol) & (((lb > tol).astype(int) + (lc > tol) + (ld > tol)) < 3)
        shift[ids] = (np.outer(warp1[ids], t1[face]) + np.outer(warp2[ids], t2[face]))
    return _xyz_to_rst(xyz + shift).tobytes()


def unit_nodes(order: int) -> np.ndarray:
    """Warp & blend nodes on the reference tetrahedron, shape [Np, 3]."""
    return np.frombuffer(_unit_nodes_cached(order)).reshape(-1, 3).copy()


# --- bases ------------------------------------------------------------------

def monomial_vandermonde(points: np.ndarray, exponents) -> np.ndarray:
    """V[i, k] = prod_d points[i, d] ** exponents[k][d] (``push_monomial.hpp:60-69``)."""
    pts = np.asarray(points, dtype=np.float64)
    v = np.empty((len(pts), len(exponents)))
    for k, (a, b, c) in enumerate(exponents):
        v[:, k] = pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c
    return v


def _rst_to_abc(rst: np.ndarray):
    r, s, t = rst[:, 0], rst[:, 1], rst[:, 2]
    a = np.full_like(r, -1.0)
    den = -s - t
    ok = den != 0
    a[ok] = 2 * (1 + r[ok]) / den[ok] - 1
    b = np.full_like(r, -1.0)
    ok = t != 1
    b[ok] = 2 * (1 + s[ok]) / (1 - t[ok]) - 1
    return a, b, t


def orthonormal_mode(rst: np.ndarray, mode: tuple[int, int, int]) -> np.ndarray:
    """PKDO orthonormal polynomial on the reference tetrahedron."""
    i, j, k = mode
    a, b, c = _rst_to_abc(np.asarray(rst, dtype=np.float64))
    h1 = jacobi_p(a, 0, 0, i)
    h2 = jacobi_p(b, 2 * i + 1, 0, j)
    h3 = jacobi_p(c, 2 * (i + j) + 2, 0, k)
    return 2 * math.sqrt(2) * h1 * h2 * (1 - b) ** i * h3 * (1 - c) ** (i + j)


def orthonormal_vandermonde(points: np.ndarray, modes) -> np.ndarray:
    pts = np.asarray(points, dtype=np.float64)
    return np.column_stack([orthonormal_mode(pts, m) for m in modes])


@lru_cache(maxsize=None)
def _monomial_integral(a: int, b: int, c: int) -> Fraction:
    """Exact integral of r^a s^b t^c over the reference tetrahedron."""
    # r = 2u - 1 etc. on the unit simplex u, v, w >= 0, u + v + w <= 1
    # (Jacobian 8), then Dirichlet: int u^i v^j w^k = i! j! k! / (i+j+k+3)!.
    total = Fraction(0)
    for i in range(a + 1):
        ci = math.comb(a, i) * 2 ** i * (-1) ** (a - i)
        for j in range(b + 1):
            cj = math.comb(b, j) * 2 ** j * (-1) ** (b - j)
            for k in range(c + 1):
                ck = math.comb(c, k) * 2 ** k * (-1) ** (c - k)
                total += Fraction(ci * cj * ck * math.factorial(i) * math.factorial(j)
                                  * math.factorial(k), math.factorial(i + j + k + 3))
    return 8 * total


def integration_weights(order: int) -> np.ndarray:
    """w = M 1 on the reference element: w_i = integral of the i-th Lagrange
    function. The normalising depositor builds exactly this vector from the
    mass matrix (``dep_normshape.hpp:214-222``)."""
    ex = node_tuples(order)
    v = monomial_vandermonde(unit_nodes(order), ex)
    moments = np.array([float(_monomial_integral(*e)) for e in ex])
    # l_i(r) = sum_k C[k, i] m_k(r) with C = V^{-1}; integral = C^T moments.
    return np.linalg.solve(v.T, moments)


def mass_matrix(order: int) -> np.ndarray:
    """Reference-element mass matrix M = (V V^T)^{-1} from the orthonormal basis."""
    v = orthonormal_vandermonde(unit_nodes(order), mode_identifiers(order))
    return np.linalg.inv(v @ v.T)
