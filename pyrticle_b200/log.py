"""Particle and beam log quantities (the reference's ``pyrticle/log.py``
particle and beam sections, log.py:107-325), computed by libprt's fused
reduction (``pyrticle_b200.diagnostics``). pytools' LogManager is not
required: each quantity is a callable with the reference's name, unit and
description, and the ``add_*`` helpers register them with any manager that
has ``add_quantity``."""

from __future__ import annotations

import numpy as np

from . import diagnostics as D


def axis_name(axis):
    return "xyz"[axis]


class StateObserver:
    """Holds the current method and state (log.py:33-70, particle part)."""

    def __init__(self, method, maxwell_op=None):
        self.method = method
        self.maxwell_op = maxwell_op
        self.state = None

    def set_fields_and_state(self, fields, state):
        self.fields = fields
        self.state = state


class _Quantity:
    def __init__(self, name, unit, description):
        self.name, self.unit, self.description = name, unit, description


class ParticleCount(_Quantity):
    def __init__(self, observer, name="n_part"):
        super().__init__(name, "1", "Particle Count")
        self.observer = observer

    def __call__(self):
        return len(self.observer.state)


class ParticleMomentum(_Quantity):
    def __init__(self, observer, names=None):
        vdim = observer.method.dimensions_velocity
        self.names = names or ["p%s_part" % axis_name(i) for i in range(vdim)]
        super().__init__(self.names, ["N*s"] * vdim, ["Particle Momentum"] * vdim)
        self.observer = observer

    def __call__(self):
        return D.particle_momentum(self.observer.state)


class KineticEnergy(_Quantity):
    def __init__(self, observer, name="W_part"):
        super().__init__(name, "J", "Kinetic Energy")
        self.observer = observer

    def __call__(self):
        c = self.observer.method.units.VACUUM_LIGHT_SPEED()
        return float(D.beam_moments(self.observer.state, c)[D.BM["ke"]])


class ParticleCharge(_Quantity):
    def __init__(self, observer, name="Q_part"):
        super().__init__(name, "C", "Total particle charge")
        self.observer = observer

    def __call__(self):
        return D.total_charge(self.observer.state)


class RMSBeamRadius(_Quantity):
    def __init__(self, observer, axis, name=None):
        super().__init__(name or "r%s_rms" % axis_name(axis), "m",
                         "RMS Beam Radius along %s" % axis_name(axis))
        self.observer, self.axis = observer, axis

    def __call__(self):
        return D.rms_beam_size(self.observer.state, self.axis)


class RMSBeamEmittance(_Quantity):
    def __init__(self, observer, axis, beam_axis, name=None):
        super().__init__(name or "eps%s_rms" % axis_name(axis), "m*rad",
                         "RMS Beam Emittance along %s" % axis_name(axis))
        self.observer, self.axis, self.beam_axis = observer, axis, beam_axis

    def __call__(self):
        return D.rms_beam_emittance(self.observer.state, self.axis, self.beam_axis)


class RMSBeamEnergySpread(_Quantity):
    def __init__(self, observer, name="Espread"):
        super().__init__(name, "J", "RMS Beam Energy Spread")
        self.observer = observer

    def __call__(self):
        return D.rms_energy_spread(self.observer.state,
                                   self.observer.method.units.VACUUM_LIGHT_SPEED())


class ParticleCurrent(_Quantity):
    def __init__(self, observer, direction, tube_length, name="I_part"):
        super().__init__(name, "A", "Particle Current along %s" % str(list(direction)))
        self.observer = observer
        self.direction = np.asarray(direction)
        self.tube_length = tube_length

    def __call__(self):
        return float(np.dot(D.particle_current(self.observer.state, None, self.tube_length,
                                               self.observer.method.units.VACUUM_LIGHT_SPEED()),
                            self.direction))


class FindCounter(_Quantity):
    """Particles located by one branch of the element finder since the last
    reading (the reference's EventCounter quantities, cloud.py:340-378)."""

    def __init__(self, method, attr, name, description):
        super().__init__(name, "1", description)
        self.method = method
        self.attr = attr
        self.last = getattr(method, attr)

    def __call__(self):
        now = getattr(self.method, self.attr)
        value, self.last = now - self.last, now
        return value


def add_particle_quantities(mgr, observer):
    mgr.add_quantity(ParticleCount(observer))
    mgr.add_quantity(ParticleMomentum(observer))
    mgr.add_quantity(KineticEnergy(observer))
    mgr.add_quantity(ParticleCharge(observer))


def add_beam_quantities(mgr, observer, axis=0, beam_axis=2):
    mgr.add_quantity(RMSBeamRadius(observer, axis))
    mgr.add_quantity(RMSBeamEmittance(observer, axis, beam_axis))
    mgr.add_quantity(RMSBeamEnergySpread(observer))


def add_currents(mgr, observer, direction, tube_length):
    mgr.add_quantity(ParticleCurrent(observer, direction, tube_length))
