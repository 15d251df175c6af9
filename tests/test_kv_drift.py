"""The reference's force-free KV drift (test_pyrticle.py:62-74 and 77-183),
restated on this build's meshes.

A Kapchinskij-Vladimirskij beam (uniform on the 4D ellipsoid surface in
(x, y, x', y'), uniform in z; distribution.py:233-400) drifts through a
z-periodic tube without fields for 1 m of flight: the device particle path
(PicMethod.step: five LSRK stages with relocation and periodic wrap, element
sort) and the device beam diagnostics (rms_beam_size) each step. The rms
radius must follow the chargeless KV envelope a(s) = sqrt(a0^2 + (eps/a0)^2
s^2) (distribution.py:411-420) within 1%, as in the reference. The envelope
itself is checked against an RK4 integration of the KV envelope equation
a'' = eps^2 / a^3 (distribution.py:423-449 with no focusing and no space
charge), the reference's predictor test.

The reference meshes a cylinder of radius 25 mm and length 100 mm at order 3
with hedge's DG time step; here a 50 x 50 x 100 mm box, z-periodic, order 3,
with this build's stable step (0.3 inradius / c): the drift is force free, so
the step size only sets how often the radius is checked.
"""

import math

import numpy as np
import pytest

from pyrticle_b200.units import SIUnitsWithNaturalConstants as U


def chargeless_kv_radius(a0, eps, s):
    return math.sqrt(a0 ** 2 + (eps / a0) ** 2 * s ** 2)


def kv_envelope_rk4(a0, eps, s_values, substeps=200):
    """a'' = eps^2 / a^3 from a(0) = a0, a'(0) = 0, by classical RK4."""
    def f(y):
        return np.array([y[1], eps ** 2 / y[0] ** 3])

    out = []
    y = np.array([a0, 0.0])
    s = 0.0
    for target in s_values:
        h = (target - s) / substeps
        for _ in range(substeps):
            k1 = f(y)
            k2 = f(y + h / 2 * k1)
            k3 = f(y + h / 2 * k2)
            k4 = f(y + h * k3)
            y = y + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        s = target
        out.append(y[0])
    return np.array(out)


def kv_beam(n, rng, radii, emittances, z_length, z_pos, beta, c):
    """Positions and velocities of a KV beam centred on the z axis."""
    s = rng.normal(size=(n, 4))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    radii = np.asarray(radii)
    emittances = np.asarray(emittances)
    x = s[:, :2] * radii
    xp = s[:, 2:] / radii * emittances
    one = (x ** 2 / radii ** 2).sum(1) + (xp ** 2 * radii ** 2 / emittances ** 2).sum(1)
    assert np.all(np.abs(one - 1) < 1e-14)
    z = rng.uniform(z_pos - z_length / 2, z_pos + z_length / 2, n)
    vz = beta * c
    pos = np.column_stack([x, z])
    vel = np.column_stack([xp * vz, np.full(n, vz)])
    return pos, vel


def test_kv_predictors():
    """The closed-form chargeless envelope against the integrated envelope
    equation (test_pyrticle.py:62-74: 1e-3)."""
    a0, eps = 2.5e-3, 5e-6
    s_values = np.linspace(0, 50 * (a0 ** 2 / eps) / 7, 50)
    exact = np.array([chargeless_kv_radius(a0, eps, s) for s in s_values])
    num = kv_envelope_rk4(a0, eps, s_values)
    assert np.max(np.abs(exact - num) / exact) < 1e-3


@pytest.mark.gpu
def test_kv_with_no_charge():
    pytest.importorskip("torch")
    from pyrticle_b200 import meshgen, problems
    from pyrticle_b200.cloud import PicMethod
    from pyrticle_b200.deposition.shape import ShapeFunctionDepositor
    from pyrticle_b200.diagnostics import rms_beam_size
    from pyrticle_b200.discretization import Discretization
    from pyrticle_b200.pusher import MonomialParticlePusher

    units = U
    c = units.VACUUM_LIGHT_SPEED()
    MM = 1e-3
    mesh = meshgen.box_mesh((8, 8, 16), (-25 * MM, -25 * MM, 0.0), (25 * MM, 25 * MM, 100 * MM),
                            periodic=(False, False, True))
    discr = Discretization(mesh, 3)
    method = PicMethod(discr, units, ShapeFunctionDepositor(), MonomialParticlePusher(), 3, 3)

    final_time = 1.0 / c
    dt = problems.stable_dt(mesh)
    nsteps = int(final_time / dt) + 1
    dt = final_time / nsteps

    nparticles = 10000
    cloud_charge = 1e-9
    electrons_per_particle = cloud_charge / nparticles / units.EL_CHARGE
    el_energy = 5.2e6 * units.EV
    gamma = el_energy / units.EL_REST_ENERGY()
    beta = (1 - 1 / gamma ** 2) ** 0.5
    radii = 2 * [2.5 * MM]
    emittances = 2 * [5 * MM * 1e-3]
    pos, vel = kv_beam(nparticles, np.random.default_rng(0), radii, emittances,
                       z_length=5 * MM, z_pos=10 * MM, beta=beta, c=c)
    mass = electrons_per_particle * units.EL_MASS
    state = method.make_state()
    method.add_particles(state, zip(pos, vel, np.zeros(nparticles), np.full(nparticles, mass)),
                         nparticles)
    assert len(state) == nparticles

    # rms radius and emittance of the KV beam: half the radius, a quarter of
    # the emittance (distribution.py:248-254)
    a0, eps = radii[0] / 2, emittances[0] / 4
    worst = 0.0
    t = 0.0
    for step in range(nsteps + 1):
        if step % 10 == 0 or step == nsteps:
            rx = rms_beam_size(state, 0)
            theory = chargeless_kv_radius(a0, eps, beta * c * t)
            worst = max(worst, abs(rx - theory) / theory)
        if step < nsteps:
            method.step(state, None, dt, steps=1, deposit=False)
            t += dt
    assert len(state) == nparticles  # nothing left the periodic tube
    assert worst < 0.01, worst
    # the beam really spread: 1.25 mm -> 1.6 mm rms over the metre
    assert rms_beam_size(state, 0) > 1.25 * a0
