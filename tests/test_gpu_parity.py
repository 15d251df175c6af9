"""Parity of the CUDA path (libprt through the PicMethod API and the C ABI)
with the CPU oracle on the same seeded inputs.

Bars: element ids and find counters bit-exact; forces, trajectories, rho
and j within 1e-12 relative L2 (FP64 plain form); deposition deterministic
(bitwise equal on repeat).
"""


import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import pyoracle as O  # noqa: E402
from pyrticle_b200 import _lib, meshgen, problems, refelement  # noqa: E402
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B, PicMethod  # noqa: E402
from pyrticle_b200.deposition.grid import GridDepositor  # noqa: E402
from pyrticle_b200.deposition.grid_base import SingleBrickGenerator  # noqa: E402
from pyrticle_b200.deposition.shape import (NormalizedShapeFunctionDepositor,  # noqa: E402
                                            ShapeFunctionDepositor)
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

from conftest import rel_l2  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-12
C_LIGHT = U.VACUUM_LIGHT_SPEED()


def make_method(w, depositor=None, order=None, mesh=None, nodes=None):
    mesh = mesh or w.mesh
    discr = Discretization(mesh, order or w.order, nodes=nodes)
    m = PicMethod(discr, U, depositor or ShapeFunctionDepositor(), MonomialParticlePusher(), 3, 3)
    return m


def make_state(m, w, x=None, p=None):
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions if x is None else x,
                                w.momenta if p is None else p, w.charges, w.masses)
    return s


@pytest.fixture(scope="module")
def setup(small_workload, oracle_mesh):
    w = small_workload
    m = make_method(w)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    m.depositor.set_shape_function(None, sf)
    ex = refelement.node_tuples(w.order)
    V = refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex)
    return dict(w=w, m=m, sf=sf, om=oracle_mesh, pu=O.OraclePusher(ex, V))


def test_library_version():
    lib = _lib.load()
    assert b"sm_100a" in lib.prt_version()


def test_find_containing_elements_bitexact(setup):
    w, m, om = setup["w"], setup["m"], setup["om"]
    rng = np.random.default_rng(11)
    pts = np.concatenate([w.positions,
                          rng.uniform(w.mesh.bbox_min - 1e-4, w.mesh.bbox_max + 1e-4, (4000, 3)),
                          w.mesh.points, w.mesh.face_centroids[:, 0]])
    x = torch.as_tensor(pts, device="cuda").T.contiguous()
    el = m.find_containing_elements_device(x).cpu().numpy().view(np.uint32)
    assert np.array_equal(el, O.find_containing_elements(om, pts, linear=True))


def test_velocities_match(setup):
    w, m = setup["w"], setup["m"]
    s = make_state(m, w)
    v = m.velocities(s)
    vo = O.velocities(s.momenta, s.masses, C_LIGHT)
    assert np.array_equal(v, vo)          # same IEEE operations in the same order


def test_relocation_bitexact_with_counters_and_kills(setup):
    """update_containing_elements after a random displacement that sends
    some particles into neighbours, vertex neighbours, far elements (global
    search) and out of the mesh (removed)."""
    w, m, om = setup["w"], setup["m"], setup["om"]
    s = make_state(m, w)
    el0 = s.containing_elements.copy()
    rng = np.random.default_rng(3)
    h = 0.01 / 8
    scale = np.where(rng.random(len(w.positions)) < 0.9, 0.05 * h, 1.5 * h)
    dx = rng.normal(size=w.positions.shape) * scale[:, None]
    dx[:20] = rng.normal(size=(20, 3)) * 0.02        # far moves, some leave the box
    dp = np.zeros_like(dx)
    before = (m.find_same_counter, m.find_by_neighbor_counter, m.find_by_vertex_counter,
              m.find_global_counter)

    class ShiftRecorder:
        """A per-particle array kept in step through the number shifts."""

        def __init__(self, ids):
            self.ids = list(ids)

        def note_move(self, orig, dest, size):
            self.ids[dest:dest + size] = self.ids[orig:orig + size]

        def note_change_size(self, n):
            del self.ids[n:]

        def note_reset(self, start, size):
            pass

    rec = ShiftRecorder(s.particle_ids)
    s.particle_number_shift_signaller.subscribe(rec)
    new = m.advance_state(s, dx, dp, None)
    # the kills reached the subscribers as moves + a size change (id order)
    assert rec.ids == list(new.particle_ids)
    got = (m.find_same_counter - before[0], m.find_by_neighbor_counter - before[1],
           m.find_by_vertex_counter - before[2], m.find_global_counter - before[3])
    r = O.update_containing_elements(om, w.positions + dx, w.momenta, w.charges, w.masses, el0)
    assert r["rc"] == 0
    order = np.argsort(r["ids"])
    assert np.array_equal(new.particle_ids, r["ids"][order])
    assert np.array_equal(new.containing_elements, r["el"][order])
    assert np.array_equal(new.positions, r["x"][order])
    c = r["counters"]
    assert got == (c.find_same, c.find_by_neighbor, c.find_by_vertex, c.find_global)
    assert len(new) < len(s)      # some particles left the mesh
    assert c.find_global > 0 and c.find_by_vertex > 0 and c.find_by_neighbor > 0


def test_forces_and_vis_vectors(setup):
    w, m, om, pu = setup["w"], setup["m"], setup["om"], setup["pu"]
    m.debug.add("verbose_vis")
    try:
        s = make_state(m, w)
        v = m.velocities(s)
        F = m.pusher.forces(s, v, *w.fields)
        Fo, vis = O.forces(pu, om, s.positions, s.containing_elements, s.charges, v,
                           list(w.fields), vis=True)
        assert rel_l2(F, Fo) < TOL
        for k, name in enumerate(("pt_e", "pt_b", "el_force", "mag_force")):
            assert rel_l2(s.vis_listener.particle_vis_map[name], vis[k]) < TOL
        # a missing component (the reference's ZeroVector) counts as zero
        F2 = m.pusher.forces(s, v, w.fields[0], w.fields[1], None, None, None, w.fields[5])
        f = list(w.fields)
        f[2] = f[3] = f[4] = np.zeros_like(f[0])
        assert rel_l2(F2, O.forces(pu, om, s.positions, s.containing_elements, s.charges, v,
                                   f)) < TOL
    finally:
        m.debug.discard("verbose_vis")


def test_lsrk_steps_match_oracle(setup):
    w, m, om, pu = setup["w"], setup["m"], setup["om"], setup["pu"]
    s = make_state(m, w)
    fields = torch.as_tensor(w.fields, device="cuda")
    steps = 20
    m.step(s, fields, w.dt, steps=steps, deposit=False)
    el0 = O.find_containing_elements(om, w.positions)
    r = O.lsrk_steps(pu, om, w.positions, w.momenta, w.charges, w.masses, el0, list(w.fields),
                     LSRK4_A, LSRK4_B, w.dt, C_LIGHT, steps)
    order = np.argsort(r["ids"])
    assert np.array_equal(s.particle_ids, r["ids"][order])
    assert rel_l2(s.positions, r["x"][order]) < TOL
    assert rel_l2(s.momenta, r["p"][order]) < TOL
    flips = int((s.containing_elements != r["el"][order]).sum())
    assert flips == 0


def test_deposit_plain_matches_oracle_and_golden(setup):
    w, m, om = setup["w"], setup["m"], setup["om"]
    s = make_state(m, w)
    rho, j = m.deposit_densities(s)
    v = m.velocities(s)
    ro, jo, _, _ = O.deposit_shape(om, 0, setup["sf"], s.positions, s.charges, v,
                                   s.containing_elements)
    assert rel_l2(rho, ro) < TOL
    assert rel_l2(j, jo.T) < TOL
    # reference-layout host entry points
    assert rel_l2(m.depositor.deposit_j(s), jo) < TOL
    assert rel_l2(m.depositor.deposit_rho(s), ro) < TOL


def test_deposit_is_deterministic(setup):
    w, m = setup["w"], setup["m"]
    s = make_state(m, w)
    r1, j1 = m.depositor.deposit_densities_device(s)
    r2, j2 = m.depositor.deposit_densities_device(s)
    assert torch.equal(r1, r2) and torch.equal(j1, j2)
    # and independent of the store order
    m.sort_by_element(s)
    r3, j3 = m.depositor.deposit_densities_device(s)
    assert rel_l2(r3.cpu().numpy(), r1.cpu().numpy()) < 1e-14


def test_golden_fixture_through_gpu(setup):
    """The committed oracle fixture, reproduced through the device path."""
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "config0_small.npz")
    w = problems.make("config0", scale=float(g["scale"]))
    m = make_method(w)
    m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    s = make_state(m, w)
    assert np.array_equal(s.containing_elements, g["el0"])
    m.step(s, torch.as_tensor(w.fields, device="cuda"), w.dt, steps=int(g["steps"]),
           deposit=False)
    ctr = m.transfer_find_counters()
    order = np.argsort(g["ids"])
    assert np.array_equal(s.containing_elements, g["el"][order])
    assert [ctr.find_same, ctr.find_by_neighbor, ctr.find_by_vertex,
            ctr.find_global] == list(g["counters"])
    assert rel_l2(s.positions, g["x"][order]) < TOL
    rho, j = m.deposit_densities(s)
    assert rel_l2(rho, g["rho"]) < TOL
    assert rel_l2(j, g["j"].T) < TOL


def test_deposit_normalized_matches_oracle(setup):
    w, om = setup["w"], setup["om"]
    m = make_method(w, depositor=NormalizedShapeFunctionDepositor())
    m.depositor.set_shape_function(None, setup["sf"])
    s = make_state(m, w)
    rho, j = m.deposit_densities(s)
    v = m.velocities(s)
    iw = m.depositor.integral_weights
    ro, jo, st, zm = O.deposit_shape(om, 1, setup["sf"], s.positions, s.charges, v,
                                     s.containing_elements, integral_weights=iw)
    assert rel_l2(rho, ro) < TOL
    assert rel_l2(j, jo.T) < TOL
    total = float((rho.reshape(-1, len(iw)) @ iw * w.mesh.jacobians).sum())
    assert total == pytest.approx(float(w.charges.sum()), rel=1e-13)
    ns = s.depositor_state.normalization_stats
    assert ns.count() == int(st[0])
    assert ns.mean() == pytest.approx(st[1], rel=1e-12)


def test_empty_and_all_removed(setup):
    w, m = setup["w"], setup["m"]
    s = m.make_state()
    rho, j = m.deposit_densities(s)
    assert not rho.any() and not j.any()
    s = make_state(m, w)
    new = m.advance_state(s, np.full(w.positions.shape, 1.0), np.zeros_like(w.positions))
    assert len(new) == 0
    rho, j = m.deposit_densities(new)
    assert not rho.any()


def test_zero_momentum_raises_no_best_normal(setup):
    w, m = setup["w"], setup["m"]
    x = w.positions[:1]
    p = np.zeros((1, 3))
    s = m.make_state()
    m.add_particles_from_arrays(s, x, p, w.charges[:1], w.masses[:1])
    # move it out of its element with zero momentum: the reference throws
    with pytest.raises(RuntimeError, match="no best normal"):
        m.advance_state(s, np.array([[3e-4, 3e-4, 3e-4]]), np.zeros((1, 3)))


def test_static_fields_gpu():
    """The restated reference integration test through the device path."""
    import static_field as SF
    for case, setup_ in SF.make_setups().items():
        mesh = SF.periodic_cylinder_box()
        w = problems.Workload(name=case, mesh=mesh, order=1, positions=None, momenta=None,
                              charges=None, masses=None, fields=None, shape_radius=0.1,
                              dt=0.0, steps=0)
        m = make_method(w, order=1)
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


def test_periodic_deposit_images():
    """Particles near the periodic seam deposit through their images, as the
    walk does when it crosses a periodic face."""
    mesh = meshgen.box_mesh((4, 4, 8), (0, 0, 0), (0.01, 0.01, 0.02), periodic=(False, False, True))
    order = 2
    nodes = meshgen.element_nodes(mesh, order)
    om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
    w = problems.Workload(name="p", mesh=mesh, order=order, positions=None, momenta=None,
                          charges=None, masses=None, fields=None, shape_radius=0.003, dt=0,
                          steps=0)
    m = make_method(w)
    sf = PolynomialShapeFunction(0.003, 3, 2)
    m.depositor.set_shape_function(None, sf)
    rng = np.random.default_rng(2)
    n = 300
    x = np.stack([rng.uniform(0.003, 0.007, n), rng.uniform(0.003, 0.007, n),
                  np.concatenate([rng.uniform(0, 0.002, n // 2), rng.uniform(0.018, 0.02, n - n // 2)])], 1)
    p = rng.normal(size=(n, 3)) * 1e-22
    s = m.make_state()
    m.add_particles_from_arrays(s, x, p, np.full(n, -1.6e-19), np.full(n, 9.1e-31))
    rho, j = m.deposit_densities(s)
    ro, jo, _, _ = O.deposit_shape(om, 0, sf, s.positions, s.charges, m.velocities(s),
                                   s.containing_elements)
    assert rel_l2(rho, ro) < TOL and rel_l2(j, jo.T) < TOL


def grid_method(w, weights):
    gen = SingleBrickGenerator(dims=(24, 24, 96))
    dep = GridDepositor(brick_generator=gen, grid_weights=weights)
    m = make_method(w, depositor=dep)
    m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    return m


@pytest.mark.parametrize("weights", ["shape", "trilinear"])
def test_grid_deposit_and_remap(setup, weights):
    w, om = setup["w"], setup["om"]
    m = grid_method(w, weights)
    dep = m.depositor
    s = make_state(m, w)
    gr, gj = dep.deposit_grid_densities_device(s)
    v = m.velocities(s)
    bricks = [b.as_struct() for b in dep.bricks]
    wmode = _lib.GRID_SHAPE if weights == "shape" else _lib.GRID_TRILINEAR
    gro, gjo = O.deposit_grid(om, bricks, wmode, dep.shape_function, s.positions, s.charges, v,
                              dep.grid_node_count)
    assert rel_l2(gr.cpu().numpy(), gro) < TOL
    assert rel_l2(gj.cpu().numpy(), gjo.T) < TOL
    # remap onto the mesh
    rho = dep.remap_grid_to_mesh_device(gr).cpu().numpy()
    to = np.zeros(len(m.discretization))
    O.remap_grid_to_mesh(dep.grid_desc, np.ascontiguousarray(gro), to)
    assert rel_l2(rho, to) < TOL
    # total charge is carried through the grid for the trilinear weights
    if weights == "trilinear":
        dV = float(np.prod(dep.bricks[0].stepwidths))
        assert gro.sum() * dV == pytest.approx(float(s.charges.sum()), rel=1e-12)


@pytest.mark.parametrize("jiggle", [0.0, 0.3])
def test_grid_mixed_matches_fp64(setup, jiggle):
    """The chosen-form grid deposition (tensor cores) against the FP64 grid
    deposition: rho and j within 1e-5 relative L2 (the chosen form's bound;
    ~1e-7 expected), bitwise repeatable, and the same remapped values'
    relation."""
    import torch
    w = setup["w"]
    gen = SingleBrickGenerator(dims=(24, 24, 96))
    out = {}
    for prec in ("fp64", "mixed"):
        dep = GridDepositor(brick_generator=gen, jiggle_radius=jiggle, precision=prec)
        m = make_method(w, depositor=dep)
        m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
        s = make_state(m, w)
        out[prec] = dep.deposit_grid_densities_device(s)
        if prec == "mixed":
            again = dep.deposit_grid_densities_device(s)
            assert torch.equal(out[prec][0], again[0]) and torch.equal(out[prec][1], again[1])
    (r64, j64), (r32, j32) = out["fp64"], out["mixed"]
    assert float(torch.linalg.norm(r32 - r64) / torch.linalg.norm(r64)) < 1e-5
    assert float(torch.linalg.norm(j32 - j64) / torch.linalg.norm(j64)) < 1e-5


def test_grid_remap_components_equal_single_remaps(setup):
    """The four-component remap (rho and j in one pass) gives bitwise the
    values of four single-component remaps."""
    import torch
    w = setup["w"]
    m = grid_method(w, "shape")
    dep = m.depositor
    s = make_state(m, w)
    gr, gj = dep.deposit_grid_densities_device(s)
    q = torch.cat([gr[None], gj]).contiguous()
    one = torch.zeros((4, len(m.discretization)), dtype=torch.float64, device=q.device)
    for c in range(4):
        _lib.check(dep.lib.prt_remap_grid_to_mesh(dep.handle, q[c].data_ptr(), one[c].data_ptr(),
                                                  0, 1, dep._stream()))
    four = dep.remap_grid_to_mesh_device(q)
    assert torch.equal(one, four)
    rho, j = dep.deposit_densities_device(s)
    assert torch.equal(rho, one[0]) and torch.equal(j, one[1:])


def test_mixed_precision_deposit_error_bounds():
    """The chosen form (tensor-core deposition): rho and j within 1e-5
    relative L2 of the FP64 form (config2's bound), on a
    config2-like case (order 3, radius 0.08 cm) at reduced size."""
    w = problems.make("config2", scale=0.005, cubes=(16, 16, 64))
    m = make_method(w)
    m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    s = make_state(m, w)
    r64, j64 = m.depositor.deposit_densities_device(s, precision="fp64")
    r32, j32 = m.depositor.deposit_densities_device(s, precision="mixed")
    er = rel_l2(r32.cpu().numpy(), r64.cpu().numpy())
    ej = rel_l2(j32.cpu().numpy(), j64.cpu().numpy())
    assert er < 1e-5 and ej < 1e-5, (er, ej)
    assert er > 0  # it really ran in reduced precision


def test_mixed_precision_normalized_charge():
    w = problems.make("config0", scale=0.2)
    m = make_method(w, depositor=NormalizedShapeFunctionDepositor(precision="mixed"))
    m.depositor.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    s = make_state(m, w)
    rho, _ = m.deposit_densities(s)
    iw = m.depositor.integral_weights
    total = float((rho.reshape(-1, len(iw)) @ iw * w.mesh.jacobians).sum())
    # integer weights summed exactly against the same integer weights'
    # integrals: the deposited charge is exact to FP64 rounding
    assert total == pytest.approx(float(w.charges.sum()), rel=1e-14)
