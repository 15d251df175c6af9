"""The averaging pusher (push_average.hpp; AverageParticlePusher,
pusher.py:167-207): device forces against the CPU restatement of the
reference's element-walk averaging, and the restated static-field
integration test (test_pyrticle.py:377-384, which runs it with the
averaging pusher too) through the device path."""

import warnings

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import average as OA  # noqa: E402
from oracle import pyoracle as O  # noqa: E402
from pyrticle_b200 import meshgen, problems  # noqa: E402
from pyrticle_b200.cloud import PicMethod  # noqa: E402
from pyrticle_b200.deposition.shape import ShapeFunctionDepositor  # noqa: E402
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import AverageParticlePusher  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

pytestmark = pytest.mark.gpu
C_LIGHT = U.VACUUM_LIGHT_SPEED()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def test_average_forces_match_the_restated_walk():
    w = problems.make("config0", scale=0.02)
    m = PicMethod(Discretization(w.mesh, w.order), U, ShapeFunctionDepositor(),
                  AverageParticlePusher(), 3, 3, debug={"verbose_vis"})
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    m.depositor.set_shape_function(None, sf)
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    v = m.velocities(s)
    f = m.pusher.forces(s, v, *w.fields)
    om = O.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
    el = O.find_containing_elements(om, s.positions)
    fo, eo, bo = OA.average_forces(om, sf, m.pusher.integral_weights, s.positions, s.charges,
                                   v, el, w.fields)
    assert rel(f, fo) < 1e-12
    vis = s.vis_listener.particle_vis_map
    assert rel(vis["pt_e"], eo) < 1e-12
    assert rel(vis["pt_b"], bo) < 1e-12
    assert rel(vis["el_force"] + vis["mag_force"], fo) < 1e-12
    st = s.pusher_state.e_normalization_stats
    assert st.count() == len(s)


def test_zero_charge_particle_gets_no_force_and_a_warning():
    w = problems.make("config0", scale=0.002)
    m = PicMethod(Discretization(w.mesh, w.order), U, ShapeFunctionDepositor(),
                  AverageParticlePusher(), 3, 3)
    m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    s = m.make_state()
    q = w.charges.copy()
    q[0] = 0.0
    m.add_particles_from_arrays(s, w.positions, w.momenta, q, w.masses)
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        f = m.pusher.forces(s, m.velocities(s), *w.fields)
    assert np.all(f[0] == 0) and np.any(f[1:] != 0)
    assert any("zero reconstructed charge" in str(c.message) for c in caught)


def test_average_pusher_static_fields():
    """Uniform fields average to themselves: the closed-form helix and
    E-parallel-B trajectories within the reference's bounds."""
    import static_field as SF
    for case, setup_ in SF.make_setups().items():
        mesh = SF.periodic_cylinder_box()
        m = PicMethod(Discretization(mesh, 1), U, ShapeFunctionDepositor(),
                      AverageParticlePusher(), 3, 3)
        # the order-1 nodes are 0.5 apart: a radius of 0.6 always reaches some
        m.depositor.set_shape_function(None, PolynomialShapeFunction(0.6, 3, 2))
        nodes = m.discretization.nodes
        fields = torch.as_tensor(SF.uniform_fields(nodes, setup_.e(), setup_.b()), device="cuda")
        x0 = setup_.positions(0)
        x0[:, 2] = np.mod(x0[:, 2], 2.0)
        p0 = SF.momenta(setup_, setup_.velocities(0))
        s = m.make_state()
        n = len(x0)
        m.add_particles_from_arrays(s, x0, p0, np.full(n, setup_.charge), np.full(n, U.EL_MASS))
        dt = setup_.final_time() / setup_.nsteps
        chunk = setup_.nsteps // 300
        t = 0.0
        worst = (0.0, 0.0)
        for _ in range(setup_.nsteps // chunk):
            m.step(s, fields, dt, steps=chunk, deposit=False, sort_every=0)
            t += chunk * dt
            xe, ve = SF.trajectory_errors(setup_, t, s.positions, m.velocities(s), 2.0)
            worst = (max(worst[0], xe), max(worst[1], ve))
        assert worst[0] < 2e-12, (case, worst)
        assert worst[1] < 2e-13, (case, worst)
