"""GridFindDepositor and jiggly bricks (the reference's grid_find.py,
dep_grid_find.hpp and grid.hpp:345-449).

CPU: the MT19937 engine against the C++ standard's known answer, the
uniform_real mapping, the jiggled point origins, the brick cell -> node
lists (order and errors), and the oracle's restatements against independent
sums (the grid-find walk against the oracle's shape-function deposition, the
jiggly grid walk against a brute-force sum over all brick points).
GPU: libprt through the depositor classes against the oracle, rho and j
within 1e-12 relative L2 (FP64).
"""

import numpy as np
import pytest

from oracle import pyoracle as O
from pyrticle_b200 import _lib, meshgen
from pyrticle_b200.deposition.grid import (BrickInfo, JigglyBrickInfo, MT19937,
                                           uniform_real)
from pyrticle_b200.deposition.grid_base import SingleBrickGenerator
from pyrticle_b200.deposition.grid_find import grid_node_lists
from pyrticle_b200.tools import PolynomialShapeFunction
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U

from conftest import rel_l2

TOL = 1e-12
C_LIGHT = U.VACUUM_LIGHT_SPEED()


class _Discr:
    """The attributes a brick generator reads, without a device."""

    def __init__(self, mesh, nodes, np_):
        self.mesh = mesh
        self.nodes = nodes
        self.nodes_per_element = np_
        self.dimensions = 3

    def __len__(self):
        return len(self.nodes)


def default_bricks(mesh, nodes, np_):
    gen = SingleBrickGenerator(mesh_margin=1e-3 * float(np.max(mesh.bbox_max - mesh.bbox_min)),
                               overresolve=0.2)
    return [BrickInfo(i, 0, *b) for i, b in enumerate(gen(_Discr(mesh, nodes, np_)))]


def particles(mesh, n, seed, margin=0.0):
    rng = np.random.default_rng(seed)
    lo, hi = mesh.bbox_min + margin, mesh.bbox_max - margin
    x = rng.uniform(lo, hi, size=(n, 3))
    p = rng.normal(size=(n, 3)) * 1e-22
    return x, p, np.full(n, -1.6e-19), np.full(n, 9.1e-31)


# ------------------------------------------------------------------- CPU

def test_mt19937_known_answer():
    """C++ [rand.predef]: the 10000th output of a default-seeded mt19937
    is 4123659995."""
    e = MT19937()
    for _ in range(9999):
        e()
    assert e() == 4123659995


def test_uniform_real_mapping():
    e1, e2 = MT19937(), MT19937()
    k = e2()
    assert uniform_real(e1, -0.25, 0.25) == k / 2.0 ** 32 * 0.5 + -0.25


def test_jiggly_point_origins():
    b = JigglyBrickInfo(0, 0, (0.1, 0.2, 0.4), (1.0, 2.0, 3.0), (5, 6, 7), 0.3)
    oph = b.origin + b.stepwidths / 2
    off = (b.point_origins - oph) / b.stepwidths
    assert np.all(np.abs(off) <= 0.3)
    # a second brick draws the same offsets, in its own cell units
    b2 = JigglyBrickInfo(1, len(b), (0.3, 0.3, 0.3), (0.0, 0.0, 0.0), (2, 2, 2), 0.3)
    off2 = (b2.point_origins - (b2.origin + b2.stepwidths / 2)) / b2.stepwidths
    assert np.allclose(off, off2, rtol=0, atol=1e-14)
    # point(idx) takes origin (i + j + k) % 3
    for idx in [(0, 0, 0), (1, 0, 0), (1, 1, 0), (2, 3, 4), (4, 5, 6)]:
        exp = b.point_origins[sum(idx) % 3] + np.asarray(idx) * b.stepwidths
        assert np.array_equal(b.point(idx), exp)
    assert np.array_equal(b.points(np.array([[2, 3, 4]]))[0], b.point((2, 3, 4)))
    with pytest.raises(ValueError):
        JigglyBrickInfo(0, 0, (0.1, 0.1, 0.1), (0, 0, 0), (2, 2, 2), 0.6)


def test_grid_node_lists_order_and_errors(small_workload):
    w = small_workload
    np_ = w.nodes.shape[0] // w.mesh.element_count
    bricks = default_bricks(w.mesh, w.nodes, np_)
    starts, lists = grid_node_lists(w.mesh, w.nodes, np_, bricks)
    assert starts[-1] == len(w.nodes) == len(lists)
    assert np.array_equal(np.sort(lists), np.arange(len(w.nodes)))
    b = bricks[0]
    cell = np.floor((w.nodes - b.origin) / b.stepwidths).astype(np.int64) @ b.strides
    for g in np.unique(cell)[::97]:
        got = lists[starts[g]:starts[g + 1]]
        # one brick: a cell lists its nodes in ascending order
        assert np.array_equal(got, np.nonzero(cell == g)[0])
    # a brick that misses part of the mesh
    small = [BrickInfo(0, 0, b.stepwidths, b.origin, b.dims // 2)]
    with pytest.raises(RuntimeError, match="unassigned mesh nodes"):
        grid_node_lists(w.mesh, w.nodes, np_, small)
    # two bricks over the same region
    two = [BrickInfo(0, 0, b.stepwidths, b.origin, b.dims),
           BrickInfo(1, len(b), b.stepwidths, b.origin, b.dims)]
    with pytest.raises(NotImplementedError):
        grid_node_lists(w.mesh, w.nodes, np_, two)


def _periodic_case():
    mesh = meshgen.box_mesh((4, 4, 8), (0, 0, 0), (0.01, 0.01, 0.02),
                            periodic=(False, False, True))
    order = 2
    nodes = meshgen.element_nodes(mesh, order)
    return mesh, order, nodes


@pytest.mark.parametrize("case", ["config0", "periodic"])
def test_oracle_grid_find_equals_shape_deposition(small_workload, oracle_mesh, case):
    """The reference's grid-find walk and its element-walk shape deposition
    visit the same (particle, node) pairs within the radius."""
    if case == "config0":
        w, om = small_workload, oracle_mesh
        mesh, nodes, radius = w.mesh, w.nodes, w.shape_radius
        x, p, q, m = w.positions[:400], w.momenta[:400], w.charges[:400], w.masses[:400]
    else:
        mesh, order, nodes = _periodic_case()
        om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
        radius = 0.003
        x, p, q, m = particles(mesh, 300, 4)
        x[:100, 2] = np.random.default_rng(5).uniform(0, 0.002, 100)
    np_ = nodes.shape[0] // mesh.element_count
    sf = PolynomialShapeFunction(radius, 3, 2)
    el = O.find_containing_elements(om, x)
    assert np.all(el != 0xFFFFFFFF)
    v = O.velocities(p, m, C_LIGHT)
    rs, js, _, _ = O.deposit_shape(om, 0, sf, x, q, v, el)
    bricks = default_bricks(mesh, nodes, np_)
    starts, lists = grid_node_lists(mesh, nodes, np_, bricks)
    rg, jg = O.deposit_grid_find(om, [b.as_struct() for b in bricks], starts, lists, nodes, sf,
                                 x, q, v)
    assert rel_l2(rg, rs) < TOL and rel_l2(jg, js) < TOL
    assert np.count_nonzero(rs) > 0


def test_oracle_jiggly_grid_walk_is_complete():
    """The oracle's index-range walk over a jiggly brick against the sum of
    q S(x - pt) over every point of the brick."""
    lo, hi = np.zeros(3), np.array([0.01, 0.01, 0.02])
    b = JigglyBrickInfo(0, 0, (hi - lo) / (6, 6, 12), lo, (6, 6, 12), 0.4)
    mesh = meshgen.box_mesh((2, 2, 4), lo, hi)
    nodes = meshgen.element_nodes(mesh, 1)
    om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
    x, p, q, m = particles(mesh, 60, 8)
    sf = PolynomialShapeFunction(0.0025, 3, 2)
    v = O.velocities(p, m, C_LIGHT)
    gr, gj = O.deposit_grid(om, [b.as_struct()], _lib.GRID_SHAPE, sf, x, q, v, len(b),
                            point_origins=b.point_origins[None])
    ii, jj, kk = np.meshgrid(np.arange(6), np.arange(6), np.arange(12), indexing="ij")
    idx = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], 1)
    pts = b.points(idx)
    gidx = idx @ b.strides
    d2 = ((pts[:, None, :] - x[None]) ** 2).sum(-1)
    a = sf.radius
    S = np.where(d2 <= a * a, sf.normalizer * (a - d2 / a) ** 2, 0.0)
    exp_r = np.zeros(len(b))
    exp_r[gidx] = S @ q
    exp_j = np.zeros((len(b), 3))
    exp_j[gidx] = S @ (q[:, None] * v)
    assert rel_l2(gr, exp_r) < TOL and rel_l2(gj, exp_j) < TOL
    # and the jiggle moved the points: the regular grid gives other values
    gr0, _ = O.deposit_grid(om, [b.as_struct()], _lib.GRID_SHAPE, sf, x, q, v, len(b))
    assert rel_l2(gr0, exp_r) > 1e-3


# ------------------------------------------------------------------- GPU

def _gpu_imports():
    pytest.importorskip("torch")
    from pyrticle_b200.cloud import PicMethod
    from pyrticle_b200.deposition.grid import GridDepositor
    from pyrticle_b200.deposition.grid_find import GridFindDepositor
    from pyrticle_b200.discretization import Discretization
    from pyrticle_b200.pusher import MonomialParticlePusher
    return PicMethod, GridDepositor, GridFindDepositor, Discretization, MonomialParticlePusher


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["config0", "periodic"])
def test_grid_find_gpu_matches_oracle(small_workload, oracle_mesh, case):
    PicMethod, _, GridFindDepositor, Discretization, Pusher = _gpu_imports()
    if case == "config0":
        w, om = small_workload, oracle_mesh
        mesh, order, nodes, radius = w.mesh, w.order, w.nodes, w.shape_radius
        x, p, q, m = w.positions, w.momenta, w.charges, w.masses
    else:
        mesh, order, nodes = _periodic_case()
        om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
        radius = 0.003
        x, p, q, m = particles(mesh, 400, 6)
        x[:150, 2] = np.random.default_rng(7).uniform(0.0185, 0.02, 150)
    meth = PicMethod(Discretization(mesh, order, nodes=nodes), U, GridFindDepositor(), Pusher(),
                     3, 3)
    dep = meth.depositor
    assert dep.name == "GridFind"
    sf = PolynomialShapeFunction(radius, 3, 2)
    dep.set_shape_function(None, sf)
    s = meth.make_state()
    meth.add_particles_from_arrays(s, x, p, q, m)
    rho, j = meth.deposit_densities(s)
    v = meth.velocities(s)
    ro, jo = O.deposit_grid_find(om, [b.as_struct() for b in dep.bricks],
                                 dep.node_number_list_starts, dep.node_number_lists, nodes, sf,
                                 s.positions, s.charges, v)
    assert rel_l2(rho, ro) < TOL and rel_l2(j, jo.T) < TOL
    assert np.count_nonzero(ro) > 0


@pytest.mark.gpu
def test_jiggly_grid_gpu_matches_oracle(small_workload, oracle_mesh):
    PicMethod, GridDepositor, _, Discretization, Pusher = _gpu_imports()
    w, om = small_workload, oracle_mesh
    dep = GridDepositor(brick_generator=SingleBrickGenerator(dims=(24, 24, 96)),
                        jiggle_radius=0.35)
    meth = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, dep, Pusher(), 3, 3)
    assert dep.name == "GridJiggly"
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    dep.set_shape_function(None, sf)
    s = meth.make_state()
    meth.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    gr, gj = dep.deposit_grid_densities_device(s)
    v = meth.velocities(s)
    po = np.stack([b.point_origins for b in dep.bricks])
    gro, gjo = O.deposit_grid(om, [b.as_struct() for b in dep.bricks], _lib.GRID_SHAPE, sf,
                              s.positions, s.charges, v, dep.grid_node_count, point_origins=po)
    assert rel_l2(gr.cpu().numpy(), gro) < TOL
    assert rel_l2(gj.cpu().numpy(), gjo.T) < TOL
    # the remap onto the mesh, set up on the jiggled points
    rho = dep.remap_grid_to_mesh_device(gr).cpu().numpy()
    to = np.zeros(len(meth.discretization))
    O.remap_grid_to_mesh(dep.grid_desc, np.ascontiguousarray(gro), to)
    assert rel_l2(rho, to) < TOL
    # the points really moved: the regular brick deposits other values
    reg = GridDepositor(brick_generator=SingleBrickGenerator(dims=(24, 24, 96)))
    m2 = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, reg, Pusher(), 3, 3)
    reg.set_shape_function(None, sf)
    s2 = m2.make_state()
    m2.add_particles_from_arrays(s2, w.positions, w.momenta, w.charges, w.masses)
    gr2, _ = reg.deposit_grid_densities_device(s2)
    assert rel_l2(gr2.cpu().numpy(), gro) > 1e-3


@pytest.mark.gpu
def test_grid_remap_with_continuity_groups(small_workload, oracle_mesh):
    """GridDepositor(enforce_continuity=True): the averaging groups of
    prepare_average_groups (grid.py:143-183) applied after the remap, GPU
    against the oracle's remap (1e-12), and every group single-valued."""
    PicMethod, GridDepositor, _, Discretization, Pusher = _gpu_imports()
    w = small_workload
    dep = GridDepositor(brick_generator=SingleBrickGenerator(dims=(24, 24, 96)),
                        enforce_continuity=True)
    meth = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, dep, Pusher(), 3, 3)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    dep.set_shape_function(None, sf)
    s = meth.make_state()
    meth.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    gr, _ = dep.deposit_grid_densities_device(s, j=False)
    rho = dep.remap_grid_to_mesh_device(gr).cpu().numpy()
    to = np.zeros(len(meth.discretization))
    O.remap_grid_to_mesh(dep.grid_desc, np.ascontiguousarray(gr.cpu().numpy()), to)
    assert rel_l2(rho, to) < TOL
    st, nd = dep.average_group_starts, dep.average_groups
    assert len(st) > 1000
    for g in range(0, len(st) - 1, 7):
        vals = rho[nd[st[g]:st[g + 1]]]
        assert np.all(vals == vals[0])


@pytest.mark.gpu
def test_grid_host_entry_points(small_workload):
    """deposit_grid_densities / deposit_grid_rho / deposit_grid_j and the
    debug quantities (grid.py:820-858) agree with the device entry points."""
    PicMethod, GridDepositor, _, Discretization, Pusher = _gpu_imports()
    w = small_workload
    dep = GridDepositor(brick_generator=SingleBrickGenerator(dims=(24, 24, 96)))
    meth = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, dep, Pusher(), 3, 3)
    dep.set_shape_function(None, PolynomialShapeFunction(w.shape_radius, 3, 2))
    s = meth.make_state()
    meth.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    gr, gj = dep.deposit_grid_densities(s, meth.velocities(s))
    assert np.array_equal(gr, dep.deposit_grid_rho(s))
    assert np.array_equal(gj, dep.deposit_grid_j(s, meth.velocities(s)))
    assert gj.shape == (dep.grid_node_count, 3)
    rho = dep.remap_grid_to_mesh(gr)
    j = dep.remap_grid_to_mesh(gj)
    assert rho.shape == (len(meth.discretization),) and j.shape == (len(meth.discretization), 3)
    assert np.array_equal(rho, meth.deposit_rho(s))
    use = dep.grid_usecount()
    assert use.sum() == len(dep.eog["grid_nodes"]) and np.all(dep.ones_on_grid() == 1)
