"""The CPU oracle against known answers (no GPU needed).

The reference's own tests pin this path only through analytic tolerances
(test/static_field.py:413-415) and the shape-function integral
(test/test_pyrticle.py:389-420); these tests restate those checks on the
oracle, plus hand-computed single-element cases and the committed golden
vectors.
"""

import math
from pathlib import Path

import numpy as np
import pytest

from oracle import pyoracle as O
from pyrticle_b200 import meshgen, problems, refelement
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
from pyrticle_b200.tools import PolynomialShapeFunction
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U

from conftest import rel_l2

GOLDEN = Path(__file__).parent / "golden"


def single_tet_mesh():
    pts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
    els = np.array([[0, 1, 2, 3]])
    m = meshgen._finish_mesh(pts, els, pts.min(0), pts.max(0), np.zeros(3, bool),
                             (1, 1, 1), np.zeros((4, 3), int))
    return m


def test_unit_simplex_membership_hand_computed():
    m = single_tet_mesh()
    nodes = meshgen.element_nodes(m, 1)
    om = O.OracleMesh(m, nodes, meshgen.element_bins(m))
    inside = np.array([[0.1, 0.1, 0.1], [0.25, 0.25, 0.25], [0.0, 0.0, 0.0]])
    outside = np.array([[0.5, 0.5, 0.5], [-0.01, 0.1, 0.1], [0.4, 0.4, 0.3]])
    assert (O.find_containing_elements(om, inside) == 0).all()
    assert (O.find_containing_elements(om, outside) == meshgen.INVALID_ELEMENT).all()
    # the 1e-10 tolerance in unit coordinates (meshdata.hpp:38-48):
    # unit coordinates are 2x the physical ones here
    assert O.find_containing_elements(om, np.array([[-0.4e-10, 0.2, 0.2]]))[0] == 0
    assert O.find_containing_elements(om, np.array([[-0.6e-10, 0.2, 0.2]]))[0] == meshgen.INVALID_ELEMENT


def test_shape_value_at_node_hand_computed():
    """One particle at distance r from a node: rho = q N (a - r^2/a)^2."""
    m = single_tet_mesh()
    nodes = meshgen.element_nodes(m, 1)
    om = O.OracleMesh(m, nodes, meshgen.element_bins(m))
    a = 0.6
    sf = PolynomialShapeFunction(a, 3, 2)
    x = np.array([[0.1, 0.2, 0.15]])
    rho, j, _, _ = O.deposit_shape(om, 0, sf, x, np.array([2.0]), np.array([[1.0, 2.0, 3.0]]),
                                   np.array([0], np.uint32))
    for i, xn in enumerate(nodes):
        r2 = float(np.sum((xn - x[0]) ** 2))
        want = 0.0 if r2 > a * a else 2.0 * sf.normalizer * (a - r2 / a) ** 2
        assert rho[i] == pytest.approx(want, rel=1e-14, abs=0)
        assert j[i] == pytest.approx(np.array([1.0, 2.0, 3.0]) * want, rel=1e-14)


def test_shape_normalizer_formula():
    # tools.cpp:54 for n = 3, alpha = 2 gives 105 / (32 pi a^5)
    for a in (1e-3, 0.1, 10.0):
        sf = PolynomialShapeFunction(a, 3, 2)
        assert sf.normalizer == pytest.approx(105 / (32 * math.pi * a ** 5), rel=1e-14)


@pytest.mark.parametrize("alpha", [2, 4])
def test_shape_function_integrates_to_one(alpha):
    """test_pyrticle.py:389-420: the shape function interpolated at order 3
    integrates to 1 within 4e-5 (here on a 14^3-cube Kuhn mesh of the box
    around the ball, tets of volume <= (r/10)^3 as in the reference)."""
    r = 0.1
    mesh = meshgen.box_mesh((14, 14, 14), (-r, -r, -r), (r, r, r), jitter=0.0)
    nodes = meshgen.element_nodes(mesh, 3)
    sf = PolynomialShapeFunction(r, 3, alpha)
    vals = sf.evaluate(nodes)
    w = refelement.integration_weights(3)
    integral = float((vals.reshape(-1, len(w)) @ w * mesh.jacobians).sum())
    assert abs(integral - 1) < 4e-5


def test_c_infinity_shape_function_integrates_to_one():
    """test_pyrticle.py:389-420 for the C-infinity shape, same mesh and bound."""
    from pyrticle_b200.tools import CInfinityShapeFunction
    r = 0.1
    mesh = meshgen.box_mesh((14, 14, 14), (-r, -r, -r), (r, r, r), jitter=0.0)
    nodes = meshgen.element_nodes(mesh, 3)
    sf = CInfinityShapeFunction(r, 3)
    vals = sf.evaluate(nodes)
    w = refelement.integration_weights(3)
    integral = float((vals.reshape(-1, len(w)) @ w * mesh.jacobians).sum())
    assert abs(integral - 1) < 4e-5
    assert sf(np.zeros(3)) == pytest.approx(sf.normalizer * math.exp(-1))
    assert sf(np.array([r, 0, 0])) == 0.0


def test_global_search_bins_equal_linear_scan(small_workload, oracle_mesh):
    w = small_workload
    rng = np.random.default_rng(5)
    pts = rng.uniform(w.mesh.bbox_min - 1e-4, w.mesh.bbox_max + 1e-4, size=(3000, 3))
    # plus points exactly on vertices and faces
    pts = np.concatenate([pts, w.mesh.points[:500], w.mesh.face_centroids[:200, 0]])
    lin = O.find_containing_elements(oracle_mesh, pts, linear=True)
    binned = O.find_containing_elements(oracle_mesh, pts, linear=False)
    assert np.array_equal(lin, binned)


def test_monomial_force_exact_on_linear_fields(small_workload, oracle_mesh):
    """Fields linear in x are reproduced exactly by the order-2 interpolant."""
    w = small_workload
    c = U.VACUUM_LIGHT_SPEED()
    ex = refelement.node_tuples(w.order)
    V = refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex)
    pu = O.OraclePusher(ex, V)
    el = O.find_containing_elements(oracle_mesh, w.positions)
    v = O.velocities(w.momenta, w.masses, c)
    F = O.forces(pu, oracle_mesh, w.positions, el, w.charges, v, list(w.fields))
    x, q = w.positions, w.charges
    E = np.stack([-1e6 * (x[:, 0] - 0.005), -1e6 * (x[:, 1] - 0.005), 0 * x[:, 0]], 1)
    Fa = q[:, None] * E + np.cross(v, q[:, None] * np.array([0, 0, 0.1]))
    assert rel_l2(F, Fa) < 1e-13


def test_velocity_formula():
    c = U.VACUUM_LIGHT_SPEED()
    p = np.array([[0.0, 0.0, 0.0], [1e-22, -2e-22, 3e-22]])
    m = np.full(2, U.EL_MASS)
    v = O.velocities(p, m, c)
    assert (v[0] == 0).all()
    want = c * p[1] / math.sqrt(m[1] ** 2 * c ** 2 + p[1] @ p[1])
    assert np.allclose(v[1], want, rtol=1e-15, atol=0)


def test_normalized_deposit_conserves_charge(small_workload, oracle_mesh):
    w = small_workload
    c = U.VACUUM_LIGHT_SPEED()
    el = O.find_containing_elements(oracle_mesh, w.positions)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    iw = refelement.integration_weights(w.order)
    v = O.velocities(w.momenta, w.masses, c)
    rho, j, st, zm = O.deposit_shape(oracle_mesh, 1, sf, w.positions, w.charges, v, el,
                                     integral_weights=iw)
    total = float((rho.reshape(-1, len(iw)) @ iw * w.mesh.jacobians).sum())
    assert total == pytest.approx(w.charges.sum(), rel=1e-13)
    assert zm == -1
    assert st[0] == len(w.positions)


def test_walk_reaches_every_element_with_a_node_in_the_ball(small_workload, oracle_mesh):
    """The face-based walk (element_finder.hpp:239-293) visits every element
    that has a node within the radius: the completeness the device gather
    relies on."""
    w = small_workload
    el = O.find_containing_elements(oracle_mesh, w.positions[:200])
    a = w.shape_radius
    nodes = w.nodes.reshape(w.mesh.element_count, -1, 3)
    for i in range(200):
        visited = set(O.walk_elements(oracle_mesh, w.positions[i], el[i], a).tolist())
        d2 = ((nodes - w.positions[i]) ** 2).sum(-1)
        need = set(np.nonzero((d2 < a * a).any(axis=1))[0].tolist())
        assert need <= visited


def test_oracle_against_golden_vectors():
    """Committed fixtures, made by tests/golden/make_golden.py."""
    path = GOLDEN / "config0_small.npz"
    g = np.load(path)
    w = problems.make("config0", scale=float(g["scale"]))
    assert np.array_equal(w.positions, g["x0"])
    om = O.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
    el = O.find_containing_elements(om, w.positions)
    assert np.array_equal(el, g["el0"])
    ex = refelement.node_tuples(w.order)
    V = refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex)
    pu = O.OraclePusher(ex, V)
    c = U.VACUUM_LIGHT_SPEED()
    r = O.lsrk_steps(pu, om, w.positions, w.momenta, w.charges, w.masses, el,
                     list(w.fields), LSRK4_A, LSRK4_B, w.dt, c, int(g["steps"]))
    assert np.array_equal(r["x"], g["x"]) and np.array_equal(r["p"], g["p"])
    assert np.array_equal(r["el"], g["el"])
    ctr = r["counters"]
    assert [ctr.find_same, ctr.find_by_neighbor, ctr.find_by_vertex,
            ctr.find_global] == list(g["counters"])
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    rho, j, _, _ = O.deposit_shape(om, 0, sf, r["x"], r["q"], O.velocities(r["p"], r["m"], c),
                                   r["el"])
    assert np.array_equal(rho, g["rho"]) and np.array_equal(j, g["j"])
