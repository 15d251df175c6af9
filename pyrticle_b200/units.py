"""SI units and natural constants, with the values the reference uses
(``units.py:27-89``)."""

from __future__ import annotations

import math

import numpy as np


class SIUnits:
    RAD = 1
    M = 1
    N = 1
    A = 1
    S = 1
    KG = 1

    C = A * S
    J = N * M
    V = J / C
    F = C / V
    T = V * S / M ** 2

    MM = 1e-3 * M
    MRAD = 1e-3 * RAD
    M_S = M / S

    EPSILON0 = 1.0
    MU0 = 1.0
    EL_MASS = 1.0
    EL_CHARGE = 1.0

    @classmethod
    def VACUUM_LIGHT_SPEED(cls):
        return 1 / (cls.EPSILON0 * cls.MU0) ** 0.5

    @classmethod
    def EL_REST_ENERGY(cls):
        return cls.EL_MASS * cls.VACUUM_LIGHT_SPEED() ** 2

    @classmethod
    def gamma_from_beta(cls, beta):
        return (1 - np.dot(beta, beta)) ** (-0.5)

    @classmethod
    def gamma_from_v(cls, v):
        value = 1 - np.dot(v, v) / cls.VACUUM_LIGHT_SPEED() ** 2
        if value <= 0:
            raise RuntimeError("particle velocity >= speed of light")
        return value ** (-0.5)

    @classmethod
    def v_from_p(cls, m, p):
        c = cls.VACUUM_LIGHT_SPEED()
        return c * p * (np.dot(p, p) + c * c * m * m) ** (-0.5)


class SIUnitsWithNaturalConstants(SIUnits):
    EPSILON0 = 8.8541878176e-12 * SIUnits.F / SIUnits.M
    MU0 = 4 * math.pi * 1e-7 * SIUnits.N / SIUnits.A ** 2

    EL_MASS = 9.10938215e-31 * SIUnits.KG
    EL_CHARGE = 1.602176487e-19 * SIUnits.C
    PROTON_MASS = 1.672621637e-27 * SIUnits.KG

    EV = EL_CHARGE * SIUnits.V


class SIUnitsWithUnityConstants(SIUnits):
    EPSILON0 = 1 * SIUnits.F / SIUnits.M
    MU0 = 1 * SIUnits.N / SIUnits.A ** 2

    EL_MASS = 1 * SIUnits.KG
    EL_CHARGE = 1 * SIUnits.C
    PROTON_MASS = 1 * SIUnits.KG
