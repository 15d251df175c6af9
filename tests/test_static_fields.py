"""Restated reference integration test (test_pyrticle.py:331-384 with
static_field.py:264-417): particles in static uniform fields follow the
closed-form helix / E-parallel-B trajectories through 10^4 LSRK4 steps with
the monomial pusher, on a z-periodic mesh at order 1. Bounds as in the
reference: position rel-err < 2e-12, velocity rel-err < 2e-13.

The CPU oracle runs here; the same run through libprt is in
test_gpu_parity.py."""

import numpy as np
import pytest

from oracle import pyoracle as O
from pyrticle_b200 import meshgen, refelement
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U

import static_field as SF


@pytest.mark.parametrize("case", ["screw", "epb"])
def test_oracle_static_fields(case):
    setup = SF.make_setups()[case]
    mesh = SF.periodic_cylinder_box()
    order = 1
    nodes = meshgen.element_nodes(mesh, order)
    om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
    fields = SF.uniform_fields(nodes, setup.e(), setup.b())
    ex = refelement.node_tuples(order)
    V = refelement.monomial_vandermonde(refelement.unit_nodes(order), ex)
    pu = O.OraclePusher(ex, V)
    c = U.VACUUM_LIGHT_SPEED()
    x0 = setup.positions(0)
    x0[:, 2] = np.mod(x0[:, 2], 2.0)
    p0 = SF.momenta(setup, setup.velocities(0))
    n = len(x0)
    q = np.full(n, setup.charge)
    m = np.full(n, U.EL_MASS)
    el = O.find_containing_elements(om, x0)
    assert (el != meshgen.INVALID_ELEMENT).all()
    nsteps = setup.nsteps
    dt = setup.final_time() / nsteps
    chunk = nsteps // 300          # the reference checks every int(nsteps/300) steps
    kx = np.zeros((n, 3))
    kp = np.zeros((n, 3))
    x, p = x0, p0
    t = 0.0
    worst = (0.0, 0.0)
    for _ in range(nsteps // chunk):
        r = O.lsrk_steps(pu, om, x, p, q, m, el, list(fields), LSRK4_A, LSRK4_B, dt, c,
                         chunk, kx=kx, kp=kp)
        assert r["rc"] == 0 and r["n"] == n
        x, p, el, kx, kp = r["x"], r["p"], r["el"], r["kx"], r["kp"]
        t += chunk * dt
        v = O.velocities(p, m, c)
        xe, ve = SF.trajectory_errors(setup, t, x, v, 2.0)
        worst = (max(worst[0], xe), max(worst[1], ve))
    assert worst[0] < 2e-12, worst
    assert worst[1] < 2e-13, worst
