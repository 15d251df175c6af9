"""Beam diagnostics (the reference's diagnostics.hpp / log.py quantities):
the CPU restatement on hand-computed cases, and the fused device reduction
against it on a config0 state with removed particles."""

import math

import numpy as np
import pytest

from oracle import diagnostics as OD
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U

C_LIGHT = U.VACUUM_LIGHT_SPEED()


def test_oracle_known_answers():
    a = 1e-3
    x = [[a, 0, 0], [-a, 0, 0], [a, 0, 0], [-a, 0, 0]]
    pz = 1e-21
    p = [[0.01 * pz, 0, pz], [0.01 * pz, 0, pz], [-0.01 * pz, 0, pz], [-0.01 * pz, 0, pz]]
    assert OD.rms_beam_size(x, 0) == pytest.approx(a, rel=1e-15)
    # uncorrelated x = +-a, x' = +-0.01: emittance = a * 0.01
    assert OD.rms_beam_emittance(x, p, 0, 2) == pytest.approx(a * 0.01, rel=1e-12)
    # x' = 0.01 x / a (fully correlated): zero emittance
    pc = [[0.01 * pz * xi[0] / a, 0, pz] for xi in x]
    e = OD.rms_beam_emittance(x, pc, 0, 2)
    assert math.isnan(e) or abs(e) < 1e-12
    m = U.EL_MASS
    gamma = 2.0
    pg = gamma * m * C_LIGHT * math.sqrt(1 - 1 / gamma ** 2)
    assert OD.kinetic_energies([[0, 0, pg]], [m], C_LIGHT)[0] == pytest.approx(
        m * C_LIGHT ** 2, rel=1e-12)
    assert OD.total_charge([1.0, -2.0, 0.5]) == -0.5
    assert OD.rms_beam_size([], 0) == 0.0 and OD.rms_energy_spread([], [], C_LIGHT) == 0.0
    with pytest.raises(RuntimeError):
        OD.std_dev([])


@pytest.mark.gpu
def test_device_diagnostics_match_the_oracle():
    torch = pytest.importorskip("torch")
    from pyrticle_b200 import diagnostics as D, log, problems
    from pyrticle_b200.cloud import PicMethod
    from pyrticle_b200.deposition.shape import ShapeFunctionDepositor
    from pyrticle_b200.discretization import Discretization
    from pyrticle_b200.pusher import MonomialParticlePusher
    w = problems.make("config0", scale=0.2)
    m = PicMethod(Discretization(w.mesh, w.order), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    # a removed (not yet compacted) particle is excluded like a dropped one
    s.el[::7] = -1
    live = s.el[s.id_order()].cpu().numpy() != -1
    x = s.positions[live].tolist()
    p = s.momenta[live].tolist()
    q = s.charges[live].tolist()
    mm = s.masses[live].tolist()

    def close(a, b, tol=1e-12):
        a, b = np.asarray(a, float), np.asarray(b, float)
        assert np.all(np.abs(a - b) <= tol * np.maximum(np.abs(b), 1e-300)), (a, b)

    close(D.total_charge(s), OD.total_charge(q))
    close(D.particle_momentum(s), OD.particle_momentum(p), 1e-11)
    ke = D.kinetic_energies(s, C_LIGHT)
    close(ke[live], OD.kinetic_energies(p, mm, C_LIGHT), 1e-12)
    assert np.all(ke[~live] == 0)
    for axis in range(3):
        close(D.rms_beam_size(s, axis), OD.rms_beam_size(x, axis))
    for axis in (0, 1):
        close(D.rms_beam_emittance(s, axis, 2), OD.rms_beam_emittance(x, p, axis, 2), 1e-9)
    # the reference's <KE^2> - <KE>^2 keeps only ~4 digits here (the spread is
    # 1.5e-6 of the mean); the device sums the squares about the mean
    kes = OD.kinetic_energies(p, mm, C_LIGHT)
    kmean = math.fsum(kes) / len(kes)
    exact = math.sqrt(math.fsum((k - kmean) ** 2 for k in kes) / len(kes))
    close(D.rms_energy_spread(s, C_LIGHT), exact, 1e-9)
    close(OD.rms_energy_spread(p, mm, C_LIGHT), exact, 1e-2)
    v = m.velocities(s)[live].tolist()
    close(D.particle_current(s, None, 0.04), OD.particle_current(q, v, 0.04), 1e-11)
    # the log quantities
    obs = log.StateObserver(m)
    obs.set_fields_and_state(None, s)

    class Mgr:
        def __init__(self):
            self.q = []

        def add_quantity(self, qty, interval=1):
            self.q.append(qty)

    mgr = Mgr()
    log.add_particle_quantities(mgr, obs)
    log.add_beam_quantities(mgr, obs)
    log.add_currents(mgr, obs, (0, 0, 1), 0.04)
    vals = {str(qt.name): qt() for qt in mgr.q}
    close(vals["Q_part"], OD.total_charge(q))
    close(vals["W_part"], sum(OD.kinetic_energies(p, mm, C_LIGHT)), 1e-11)
    close(vals["rx_rms"], OD.rms_beam_size(x, 0))
    close(vals["I_part"], OD.particle_current(q, v, 0.04)[2], 1e-11)
    assert vals["n_part"] == len(s)
