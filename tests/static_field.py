"""Closed-form trajectories in static fields (restated from the reference's
test/static_field.py:45-259, after Jackson, Classical Electrodynamics, 3rd
ed.: section 12.2 and problem 12.6b)."""

import math

import numpy as np

from pyrticle_b200.units import SIUnitsWithNaturalConstants as U


class LarmorScrew:
    """Helix in a uniform Bz (static_field.py:45-117)."""

    def __init__(self, mass, charge, c, vpar, vperp, bz, nparticles):
        self.mass, self.charge, self.c = mass, charge, c
        self.vpar, self.vperp, self.bz = vpar, vperp, bz
        gamma = (1 - (vpar ** 2 + vperp ** 2) / c ** 2) ** (-0.5)
        self.omega_b = charge * bz / (gamma * mass)
        self.gyration_rad = vperp / abs(self.omega_b)
        self.angles = np.arange(0, 2 * math.pi, 2 * math.pi / nparticles)

    nsteps = 10 ** 4

    def final_time(self):
        return 1 / self.vperp

    def e(self):
        return np.zeros(3)

    def b(self):
        return np.array([0, 0, self.bz])

    def positions(self, t):
        a = self.angles + self.omega_b * t
        return np.stack([self.gyration_rad * np.sin(a), self.gyration_rad * np.cos(a),
                         np.full_like(a, self.vpar * t)], axis=1)

    def velocities(self, t):
        a = self.angles + self.omega_b * t
        w = self.omega_b * self.gyration_rad
        return np.stack([w * np.cos(a), -w * np.sin(a), np.full_like(a, self.vpar)], axis=1)


class EBParallel:
    """Parallel E and B along z (static_field.py:122-259), one particle."""

    def __init__(self, mass, charge, c, ez, bz, radius):
        self.mass, self.charge, self.c = mass, charge, c
        self.ez, self.bz = ez, bz
        self.R = mass * c / (charge * bz)
        self.rho = ez / (c * bz)
        self.scaling = radius / self.R
        self.shift = np.zeros(3)
        self.shift[2] = self.positions(0)[0, 2]

    nsteps = 10 ** 4

    def final_time(self):
        return self.R / self.c

    def e(self):
        return np.array([0, 0, self.ez])

    def b(self):
        return np.array([0, 0, self.bz])

    def t(self, phi):
        return (self.R / self.rho * math.sqrt(1 + self.scaling ** 2)
                * math.sinh(self.rho * phi) / self.c)

    def phi(self, t):
        return math.asinh(self.rho * t * self.c
                          / (self.R * math.sqrt(1 + self.scaling ** 2))) / self.rho

    def tprime(self, phi):
        return self.R * math.sqrt(1 + self.scaling ** 2) * math.cosh(self.rho * phi) / self.c

    def positions(self, t):
        phi = self.phi(t)
        zconst = self.R / self.rho * math.sqrt(1 + self.scaling ** 2)
        pos = np.array([self.scaling * self.R * math.sin(phi),
                        self.scaling * self.R * math.cos(phi),
                        zconst * math.cosh(self.rho * phi)]) - self.shift
        return pos[None]

    def velocities(self, t):
        phi = self.phi(t)
        phip = 1 / self.tprime(phi)
        zconst = self.R / self.rho * math.sqrt(1 + self.scaling ** 2)
        return np.array([[self.scaling * self.R * math.cos(phi) * phip,
                          -self.scaling * self.R * math.sin(phi) * phip,
                          zconst * math.sinh(self.rho * phi) * self.rho * phip]])


def momenta(setup, v):
    c = setup.c
    g = 1 / np.sqrt(1 - np.sum(v * v, axis=1) / c ** 2)
    return setup.mass * g[:, None] * v


def make_setups():
    c = U.VACUUM_LIGHT_SPEED()
    return {
        "screw": LarmorScrew(U.EL_MASS, U.EL_CHARGE, c, vpar=0.8 * c, vperp=0.1 * c,
                             bz=1e-3, nparticles=4),
        "epb": EBParallel(U.EL_MASS, U.EL_CHARGE, c, ez=1e5, bz=1e-3, radius=0.5),
    }


def periodic_cylinder_box():
    """Stand-in for the reference's periodic cylinder (radius 1 m, height
    2 m, test_pyrticle.py:344-346): a z-periodic box [-1,1]^2 x [0,2]."""
    from pyrticle_b200 import meshgen
    return meshgen.box_mesh((4, 4, 4), (-1.0, -1.0, 0.0), (1.0, 1.0, 2.0), jitter=0.15,
                            seed=3, periodic=(False, False, True))


def uniform_fields(nodes, e, b):
    f = np.zeros((6, len(nodes)))
    for d in range(3):
        f[d] = e[d]
        f[3 + d] = b[d]
    return f


def trajectory_errors(setup, t, x, v, z_period):
    """Max relative position and velocity errors (static_field.py:323-378);
    z is compared on the period circle so that a particle sitting on the
    periodic seam matches either image."""
    true_x = setup.positions(t).copy()
    true_x[:, 2] = np.mod(true_x[:, 2], z_period)
    true_v = setup.velocities(t)
    d = true_x - x
    d[:, 2] = np.mod(d[:, 2] + z_period / 2, z_period) - z_period / 2
    xe = np.max(np.linalg.norm(d, axis=1) / np.linalg.norm(true_x, axis=1))
    ve = np.max(np.linalg.norm(true_v - v, axis=1) / np.linalg.norm(true_v, axis=1))
    return xe, ve
