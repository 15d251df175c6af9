"""The chosen form's shape deposition on the tensor cores (precision "mixed").

Bars (the chosen form's contract): rho and j within 1e-5 relative L2 of the
FP64 oracle (or of the FP64 GPU form, which equals the oracle to 1e-12, at
sizes the oracle would take minutes on); the normalising depositor's
deposited charge equal to the particles' charge within 1e-14 relative;
bitwise repeatable. Cases: config0 (order 2, radius comparable to the
element size), a config2-like and a config4-like mesh at reduced size, a
periodic seam, removed particles, and a dense cluster whose tiles see more
than 32,768 candidates (the int32 sums are folded into FP64 between windows).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import pyoracle as O  # noqa: E402
from pyrticle_b200 import meshgen, problems  # noqa: E402
from pyrticle_b200.cloud import PicMethod  # noqa: E402
from pyrticle_b200.deposition.shape import (NormalizedShapeFunctionDepositor,  # noqa: E402
                                            ShapeFunctionDepositor)
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

from conftest import rel_l2  # noqa: E402

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-5
CHARGE_TOL = 1e-14


def method(mesh, order, radius, depositor, nodes=None):
    discr = Discretization(mesh, order, nodes=nodes)
    m = PicMethod(discr, U, depositor, MonomialParticlePusher(), 3, 3)
    m.depositor.set_shape_function(None, PolynomialShapeFunction(radius, 3, 2))
    return m


def state(m, x, p, q, mass):
    s = m.make_state()
    m.add_particles_from_arrays(s, x, p, q, mass)
    return s


def deposited_charge(m, rho):
    iw = m.depositor.integral_weights
    jac = m.discretization.mesh.jacobians
    return float((np.asarray(rho).reshape(-1, len(iw)) @ iw * jac).sum())


def both(m, s):
    r64, j64 = m.depositor.deposit_densities_device(s, precision="fp64")
    r64, j64 = r64.cpu().numpy(), j64.cpu().numpy()
    rmx, jmx = m.depositor.deposit_densities_device(s, precision="mixed")
    return r64, j64, rmx.cpu().numpy(), jmx.cpu().numpy()


def test_tc_plain_matches_oracle(small_workload, oracle_mesh):
    w = small_workload
    m = method(w.mesh, w.order, w.shape_radius, ShapeFunctionDepositor("mixed"), w.nodes)
    s = state(m, w.positions, w.momenta, w.charges, w.masses)
    rho, j = m.deposit_densities(s)
    ro, jo, _, _ = O.deposit_shape(oracle_mesh, 0, m.depositor.shape_function, s.positions,
                                   s.charges, m.velocities(s), s.containing_elements)
    er, ej = rel_l2(rho, ro), rel_l2(j, jo.T)
    assert er < MIXED_TOL and ej < MIXED_TOL, (er, ej)
    assert er > 0  # the reduced-precision path really ran


def test_tc_normalized_charge_and_oracle(small_workload, oracle_mesh):
    w = small_workload
    m = method(w.mesh, w.order, w.shape_radius, NormalizedShapeFunctionDepositor("mixed"),
               w.nodes)
    s = state(m, w.positions, w.momenta, w.charges, w.masses)
    rho, j = m.deposit_densities(s)
    iw = m.depositor.integral_weights
    ro, jo, st, _ = O.deposit_shape(oracle_mesh, 1, m.depositor.shape_function, s.positions,
                                    s.charges, m.velocities(s), s.containing_elements,
                                    integral_weights=iw)
    er, ej = rel_l2(rho, ro), rel_l2(j, jo.T)
    assert er < MIXED_TOL and ej < MIXED_TOL, (er, ej)
    total = deposited_charge(m, rho)
    assert abs(total - float(w.charges.sum())) <= CHARGE_TOL * abs(float(w.charges.sum()))
    ns = s.depositor_state.normalization_stats
    assert ns.count() == int(st[0])
    assert ns.mean() == pytest.approx(st[1], rel=1e-5)
    # positions with a nonzero integer weight per particle: those within the
    # radius but for a thin rim where the weight rounds to zero
    el = s.depositor_state.el_per_particle_stats
    assert el.count() == len(w.positions)
    assert el.mean() > 0


def test_tc_deterministic(small_workload):
    w = small_workload
    m = method(w.mesh, w.order, w.shape_radius, NormalizedShapeFunctionDepositor("mixed"),
               w.nodes)
    s = state(m, w.positions, w.momenta, w.charges, w.masses)
    r1, j1 = m.deposit_densities(s)
    r2, j2 = m.deposit_densities(s)
    assert np.array_equal(r1, r2) and np.array_equal(j1, j2)


@pytest.mark.parametrize("name,scale,cubes", [("config2", 0.005, (16, 16, 64)),
                                              ("config4", 0.002, (24, 24, 48))])
def test_tc_config_like(name, scale, cubes):
    w = problems.make(name, scale=scale, cubes=cubes)
    for dep in (ShapeFunctionDepositor(), NormalizedShapeFunctionDepositor()):
        m = method(w.mesh, w.order, w.shape_radius, dep, w.nodes)
        s = state(m, w.positions, w.momenta, w.charges, w.masses)
        r64, j64, rmx, jmx = both(m, s)
        er, ej = rel_l2(rmx, r64), rel_l2(jmx, j64)
        assert er < MIXED_TOL and ej < MIXED_TOL, (name, dep.name, er, ej)
        if dep.name == "NormShape":
            q = float(w.charges.sum())
            assert abs(deposited_charge(m, rmx) - q) <= CHARGE_TOL * abs(q)


def test_tc_periodic_images():
    mesh = meshgen.box_mesh((4, 4, 8), (0, 0, 0), (0.01, 0.01, 0.02), periodic=(False, False, True))
    order, a = 2, 0.003
    nodes = meshgen.element_nodes(mesh, order)
    om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
    m = method(mesh, order, a, ShapeFunctionDepositor("mixed"), nodes)
    rng = np.random.default_rng(2)
    n = 300
    x = np.stack([rng.uniform(0.003, 0.007, n), rng.uniform(0.003, 0.007, n),
                  np.concatenate([rng.uniform(0, 0.002, n // 2),
                                  rng.uniform(0.018, 0.02, n - n // 2)])], 1)
    p = rng.normal(size=(n, 3)) * 1e-22
    s = state(m, x, p, np.full(n, -1.6e-19), np.full(n, 9.1e-31))
    rho, j = m.deposit_densities(s)
    ro, jo, _, _ = O.deposit_shape(om, 0, m.depositor.shape_function, s.positions, s.charges,
                                   m.velocities(s), s.containing_elements)
    er, ej = rel_l2(rho, ro), rel_l2(j, jo.T)
    assert er < MIXED_TOL and ej < MIXED_TOL, (er, ej)


def test_tc_removed_particles(small_workload):
    """Removed particles (element PRT_INVALID_ELEMENT, still in the store)
    deposit nothing: the same sums as a store without them."""
    w = small_workload
    m = method(w.mesh, w.order, w.shape_radius, ShapeFunctionDepositor(), w.nodes)
    s = state(m, w.positions, w.momenta, w.charges, w.masses)
    s.el[::3] = -1
    r64, j64, rmx, jmx = both(m, s)
    keep = np.ones(len(w.positions), bool)
    keep[s.ids[::3].cpu().numpy()] = False
    s2 = state(m, w.positions[keep], w.momenta[keep], w.charges[keep], w.masses[keep])
    r2, j2 = m.depositor.deposit_densities_device(s2, precision="mixed")
    assert np.array_equal(rmx, r2.cpu().numpy()) and np.array_equal(jmx, j2.cpu().numpy())
    er, ej = rel_l2(rmx, r64), rel_l2(jmx, j64)
    assert er < MIXED_TOL and ej < MIXED_TOL, (er, ej)


def test_tc_dense_cluster_folds_int32_windows(small_workload):
    """100,000 particles within 0.03 cm of one point: the tiles there stage
    far more than 256 chunks of 128 candidates, so the int32 sums are folded
    into FP64 several times per tile."""
    w = small_workload
    rng = np.random.default_rng(5)
    n = 100_000
    d = rng.normal(size=(n, 3))
    d *= (0.03e-2 * rng.random(n) ** (1 / 3) / np.linalg.norm(d, axis=1))[:, None]
    x = np.array([0.5e-2, 0.5e-2, 2e-2]) + d
    p = np.zeros((n, 3))
    p[:, 2] = 1e-22
    p[:, :2] = rng.normal(size=(n, 2)) * 1e-25
    q = np.full(n, -U.EL_CHARGE)
    mass = np.full(n, U.EL_MASS)
    for dep in (ShapeFunctionDepositor(), NormalizedShapeFunctionDepositor()):
        m = method(w.mesh, w.order, w.shape_radius, dep, w.nodes)
        s = state(m, x, p, q, mass)
        r64, j64, rmx, jmx = both(m, s)
        er, ej = rel_l2(rmx, r64), rel_l2(jmx, j64)
        assert er < MIXED_TOL and ej < MIXED_TOL, (dep.name, er, ej)
        if dep.name == "NormShape":
            assert abs(deposited_charge(m, rmx) - q.sum()) <= CHARGE_TOL * abs(q.sum())


def test_tc_and_simt_forms_agree(small_workload):
    """The tensor-core form and the FP32 CUDA-core form of the chosen
    precision agree within their two error bounds."""
    w = small_workload
    m = method(w.mesh, w.order, w.shape_radius, ShapeFunctionDepositor(), w.nodes)
    s = state(m, w.positions, w.momenta, w.charges, w.masses)
    r1, j1 = m.depositor.deposit_densities_device(s, precision="mixed")
    r2, j2 = m.depositor.deposit_densities_device(s, precision="mixed_simt")
    assert rel_l2(r1.cpu().numpy(), r2.cpu().numpy()) < 2 * MIXED_TOL
    assert rel_l2(j1.cpu().numpy(), j2.cpu().numpy()) < 2 * MIXED_TOL


@pytest.mark.parametrize("normalized", [False, True])
def test_tc_sharded_sums_are_bitwise_independent_of_the_split(small_workload, normalized):
    """Two ranks emulated on one GPU (two methods, each with its own
    workspace, the particles split in two): the charge maxima combined with
    max, the digit sums added, then combined, give bitwise the same rho and
    j as all particles on one GPU, by the single call and by the protocol."""
    from pyrticle_b200.sharding import deposit_densities_exact
    w = small_workload
    Dep = NormalizedShapeFunctionDepositor if normalized else ShapeFunctionDepositor
    ms = [method(w.mesh, w.order, w.shape_radius, Dep("mixed"), w.nodes) for _ in range(3)]
    full = state(ms[0], w.positions, w.momenta, w.charges, w.masses)
    rho1, j1 = ms[0].depositor.deposit_densities_device(full, precision="mixed")
    rho2, j2 = deposit_densities_exact(ms[0], full)
    assert torch.equal(rho1, rho2) and torch.equal(j1, j2)
    n = len(w.positions)
    cut = n // 3
    parts = [state(ms[1], w.positions[:cut], w.momenta[:cut], w.charges[:cut], w.masses[:cut]),
             state(ms[2], w.positions[cut:], w.momenta[cut:], w.charges[cut:], w.masses[cut:])]
    from pyrticle_b200 import _lib
    import ctypes as C
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    sf = ms[0].depositor.shape_function
    desc = _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer)
    iw = getattr(ms[0].depositor, "integral_weights", None)
    npos = C.c_int64()
    _lib.check(ms[0].lib.prt_mesh_position_count(ms[0].mesh_data.handle, C.byref(npos)))
    maxima = []
    for m, s in zip(ms[1:], parts):
        mx = torch.zeros(4, dtype=torch.float64, device="cuda")
        v = m.velocities_device(s)
        _lib.check(m.lib.prt_deposit_shape_charges(
            m.mesh_data.handle, m.workspace, m.depositor.mode, desc,
            _lib.ptr(iw) if iw is not None else None, len(s), s.x.data_ptr(), s.q.data_ptr(),
            v.data_ptr(), s.el.data_ptr(), mx.data_ptr(), None, stream))
        maxima.append(mx)
    gmax = torch.maximum(maxima[0], maxima[1])
    total = torch.zeros((16, npos.value), dtype=torch.float64, device="cuda")
    for m, s in zip(ms[1:], parts):
        part = torch.zeros_like(total)
        _lib.check(m.lib.prt_deposit_shape_sums(m.mesh_data.handle, m.workspace, desc, len(s),
                                                gmax.data_ptr(), part.data_ptr(), stream))
        total += part
    rho3 = torch.empty_like(rho1)
    j3 = torch.empty_like(j1)
    _lib.check(ms[0].lib.prt_deposit_shape_combine(
        ms[0].mesh_data.handle, ms[0].workspace, desc, gmax.data_ptr(), total.data_ptr(),
        rho3.data_ptr(), j3.data_ptr(), stream))
    ms[0].check_status()
    assert torch.equal(rho1, rho3) and torch.equal(j1, j3)
