"""The reference's RK coupling of the particle side (cloud.py:159-311): a
low-storage RK4 stepper advancing a TimesteppablePicState with
FieldToParticleRhsCalculator + ParticleRhsCalculator right-hand sides
(host arithmetic on number-shiftable vectors, relocation through
advance_state) against the fused device step (PicMethod.step) on the same
particles: positions and momenta within 1e-12 relative L2, element ids equal.
A second run sends particles out of the mesh in mid-step: the RK residuals
follow the removals through the number-shift signalling.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyrticle_b200 import problems  # noqa: E402
from pyrticle_b200.cloud import (LSRK4_A, LSRK4_B, FieldToParticleRhsCalculator,  # noqa: E402
                                 ParticleRhsCalculator, PicMethod, TimesteppablePicState)
from pyrticle_b200.deposition.shape import ShapeFunctionDepositor  # noqa: E402
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

from conftest import rel_l2  # noqa: E402

pytestmark = pytest.mark.gpu


class StaticMaxwell:
    """The three members of a Maxwell operator the particle RHS reads."""

    mu = U.MU0

    def split_eh(self, fields):
        return fields[0:3], [f / self.mu for f in fields[3:6]]

    def get_eh_subset(self):
        return (True, True, True, True, True, True)


def rk_steps(m, state, fields, dt, steps):
    maxwell = StaticMaxwell()
    f_rhs = FieldToParticleRhsCalculator(m, maxwell)
    p_rhs = ParticleRhsCalculator(m, maxwell)
    y = TimesteppablePicState(m, state)
    residual = 0
    t = 0.0
    for _ in range(steps):
        for a, b in zip(LSRK4_A, LSRK4_B):
            rhs = f_rhs(t, lambda: fields, lambda: y.state) + p_rhs(t, lambda: fields,
                                                                     lambda: y.state)
            residual = a * residual + dt * rhs
            y = y + b * residual
        t += dt
    return y.state


def test_rk_coupling_matches_fused_step():
    w = problems.make("config0", scale=0.05)
    m = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    s_ref = m.make_state()
    m.add_particles_from_arrays(s_ref, w.positions, w.momenta, w.charges, w.masses)
    s_dev = m.make_state()
    m.add_particles_from_arrays(s_dev, w.positions, w.momenta, w.charges, w.masses)
    fields = [np.ascontiguousarray(f) for f in w.fields]
    out = rk_steps(m, s_ref, fields, w.dt, 3)
    m.step(s_dev, torch.as_tensor(w.fields, device="cuda"), w.dt, steps=3, deposit=False)
    assert np.array_equal(out.particle_ids, s_dev.particle_ids)
    assert np.array_equal(out.containing_elements, s_dev.containing_elements)
    assert rel_l2(out.positions, s_dev.positions) < 1e-12
    assert rel_l2(out.momenta, s_dev.momenta) < 1e-12


def test_rk_residuals_follow_removals():
    """Twenty particles start next to the x = 0 wall moving out of the mesh
    and are removed in mid-step; the survivors' trajectories equal a run of
    the same stepper on the survivors alone, which holds only if every
    residual row moved with its particle."""
    w = problems.make("config0", scale=0.05)
    m = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    fields = [np.ascontiguousarray(f) for f in w.fields]
    x = w.positions.copy()
    p = w.momenta.copy()
    pz = float(np.abs(p[:, 2]).mean())
    x[:20, 0] = 2e-6
    p[:20, 0] = -pz
    s = m.make_state()
    m.add_particles_from_arrays(s, x, p, w.charges, w.masses)
    n0 = len(s)
    out = rk_steps(m, s, fields, w.dt, 2)
    assert len(out) == n0 - 20
    keep = np.isin(np.arange(n0), out.particle_ids)
    assert not keep[:20].any()
    s2 = m.make_state()
    m.add_particles_from_arrays(s2, x[keep], p[keep], w.charges[keep], w.masses[keep])
    out2 = rk_steps(m, s2, fields, w.dt, 2)
    assert len(out2) == len(out)
    assert rel_l2(out.positions, out2.positions) < 1e-13
    assert rel_l2(out.momenta, out2.momenta) < 1e-13


def test_state_helpers_and_instrumentation():
    w = problems.make("config0", scale=0.02)
    m = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)

    class Mgr:
        def __init__(self):
            self.quantities, self.constants = [], {}

        def add_quantity(self, q):
            self.quantities.append(q)

        def set_constant(self, k, v):
            self.constants[k] = v

    mgr = Mgr()
    m.add_instrumentation(mgr, None)
    assert mgr.constants == {"depositor": "ShapeFunctionDepositor",
                             "pusher": "MonomialParticlePusher"}
    s = m.make_state()
    sizes = []

    class Rec:
        def note_change_size(self, n):
            sizes.append(n)

        def note_move(self, *a):
            pass

        def note_reset(self, *a):
            pass

    rec = Rec()
    s.particle_number_shift_signaller.subscribe(rec)
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    n = len(s)
    assert sizes == [n]
    dx = np.zeros((n, 3))
    dx[:, 2] = 0.3 * w.shape_radius  # moves into neighbouring elements
    s = m.advance_state(s, dx, np.zeros((n, 3)), None)
    found = {q.name: q() for q in mgr.quantities}
    assert sum(found.values()) == n and found["n_find_global"] >= 0
    assert all(q() == 0 for q in mgr.quantities)  # events since the last reading
    with pytest.raises(ValueError):
        s.resize(n - 1)
    s.resize(2 * n)
    s.clear()
    assert len(s) == 0 and sizes[-1] == 0
    assert m.get_shape_function_class().__name__ == "PolynomialShapeFunction"


def test_shape_bandwidth_helpers():
    """guess_shape_bandwidth and optimize_shape_bandwidth (cloud.py:680-824)
    on the config0 beam (uniform in a cylinder of radius 0.25 cm over
    z in [0.5, 3.5] cm) against its analytic charge density."""
    from pyrticle_b200.cloud import guess_shape_bandwidth, optimize_shape_bandwidth
    w = problems.make("config0", scale=1.0)
    m = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    guess_shape_bandwidth(m, s, 2)
    assert m.depositor.shape_function.radius == m.mesh_data.advisable_particle_radius()
    CM = 1e-2
    nodes = np.asarray(m.discretization.nodes)
    r2 = (nodes[:, 0] - 0.5 * CM) ** 2 + (nodes[:, 1] - 0.5 * CM) ** 2
    inside = (r2 < (0.25 * CM) ** 2) & (nodes[:, 2] > 0.5 * CM) & (nodes[:, 2] < 3.5 * CM)
    rho0 = float(np.sum(w.charges)) / (np.pi * (0.25 * CM) ** 2 * 3 * CM)
    analytic = np.where(inside, rho0, 0.0)
    chosen, tried, errors = optimize_shape_bandwidth(m, s, analytic, 2)
    i = tried.index(chosen)
    assert 0 < i < len(tried) - 1 and errors[i] < errors[i - 1] and errors[i] < errors[i + 1]
    assert m.depositor.shape_function.radius == chosen
    assert errors[i] / abs(m.discretization.integral(analytic)) < 0.5
