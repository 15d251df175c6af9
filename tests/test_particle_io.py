"""Particle files (cloud.py:606-671 as files; checkpoint and resume):
VTK output round trip on the host; checkpoint save/load of the device store
with removed particles, then identical steps from the saved and the
restored state."""

import numpy as np
import pytest

from pyrticle_b200.particle_io import read_vtk_points, write_vtk


def test_vtk_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    x = rng.normal(size=(17, 3))
    q = rng.normal(size=17)
    v = rng.normal(size=(17, 3))
    path = tmp_path / "p.vtk"
    write_vtk(path, x, {"charge": q, "velocity": v})
    pos, data = read_vtk_points(path)
    assert np.array_equal(pos, x)
    assert np.array_equal(data["charge"], q) and np.array_equal(data["velocity"], v)
    with pytest.raises(ValueError):
        write_vtk(tmp_path / "bad.vtk", x, {"bad": np.zeros((17, 2))})


@pytest.mark.gpu
def test_checkpoint_resume(tmp_path):
    torch = pytest.importorskip("torch")
    from pyrticle_b200 import problems
    from pyrticle_b200.cloud import PicMethod
    from pyrticle_b200.deposition.shape import ShapeFunctionDepositor
    from pyrticle_b200.discretization import Discretization
    from pyrticle_b200.particle_io import load_checkpoint, save_checkpoint, write_particles_vtk
    from pyrticle_b200.pusher import MonomialParticlePusher
    from pyrticle_b200.tools import PolynomialShapeFunction
    from pyrticle_b200.units import SIUnitsWithNaturalConstants as U
    w = problems.make("config0", scale=0.05)
    m = PicMethod(Discretization(w.mesh, w.order), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    fields = torch.as_tensor(w.fields, device="cuda")
    m.step(s, fields, w.dt, steps=3)
    s.el[::9] = -1  # removed, not yet compacted: dropped by the checkpoint
    path = tmp_path / "ck.npz"
    save_checkpoint(s, path)
    r = load_checkpoint(m, path)
    m.compact(s)
    assert len(r) == len(s)
    for a, b in ((r.positions, s.positions), (r.momenta, s.momenta),
                 (r.particle_ids, s.particle_ids), (r.containing_elements, s.containing_elements)):
        assert np.array_equal(a, b)
    rho1, j1 = m.step(s, fields, w.dt, steps=2)
    rho2, j2 = m.step(r, fields, w.dt, steps=2)
    assert np.array_equal(s.positions, r.positions)
    assert float(torch.linalg.norm(rho1 - rho2)) <= 1e-14 * float(torch.linalg.norm(rho1))
    write_particles_vtk(m, r, tmp_path / "p.vtk")
    pos, data = read_vtk_points(tmp_path / "p.vtk")
    assert np.array_equal(pos, r.positions) and "velocity" in data
