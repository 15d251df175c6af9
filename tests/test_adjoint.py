"""Hand-written adjoint kernels (libprt) against an independent FP64 torch
autograd restatement of the same forward, against central finite
differences, and for internal consistency.

Set-up: the differentiable workload (focusing fields = Bz * basis[0] +
grad * basis[1]) on a 4x4x16-cube mesh, order 3, 400 electrons, 12 LSRK4
steps with a checkpoint every 5 (three segments, the last one partial).
Loss: random linear functionals of rho and j plus the sums over nodes of
(j - j_target)^2 and (rho - rho_target)^2 (each scaled to order one), the
targets from a run with 5% higher Bz. The linear part keeps the central
differences well conditioned: over 12 steps the 5% change of Bz moves j
only slightly, so the squared differences alone are small.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyrticle_b200 import _lib, problems  # noqa: E402
from pyrticle_b200.adjoint import (DifferentiableTrajectory, _field_components, _ptrs,  # noqa: E402
                                   monomial_coefficients)
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B, PicMethod, stream_handle  # noqa: E402
from pyrticle_b200.deposition.shape import ShapeFunctionDepositor  # noqa: E402
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

import adjoint_reference as R  # noqa: E402

pytestmark = pytest.mark.gpu

F64 = torch.float64
C_LIGHT = U.VACUUM_LIGHT_SPEED()
STEPS = 12
K = 5


def rel(a, b):
    a = a.detach().double().flatten()
    b = b.detach().double().flatten()
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.fixture(scope="module")
def S():
    w = problems.make("config3", scale=4e-4, cubes=(4, 4, 16), steps=STEPS)
    dev = torch.device("cuda", 0)
    discr = Discretization(w.mesh, w.order)
    m = PicMethod(discr, U, ShapeFunctionDepositor(), MonomialParticlePusher(), 3, 3)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    m.depositor.set_shape_function(None, sf)
    basis = torch.as_tensor(w.field_basis, dtype=F64, device=dev).contiguous()
    theta = torch.as_tensor(w.theta, dtype=F64, device=dev)
    q = torch.as_tensor(w.charges, dtype=F64, device=dev)
    mass = torch.as_tensor(w.masses, dtype=F64, device=dev)
    x0 = torch.as_tensor(w.positions.T.copy(), dtype=F64, device=dev).contiguous()
    p0 = torch.as_tensor(w.momenta.T.copy(), dtype=F64, device=dev).contiguous()
    traj = DifferentiableTrajectory(m, q, mass, w.dt, STEPS, checkpoint_every=K, basis=basis)
    with torch.no_grad():
        rho_t, j_t = traj(x0, p0, theta * torch.tensor([1.05, 1.0], dtype=F64, device=dev))
    scale_j = float((j_t ** 2).sum())
    scale_r = float((rho_t ** 2).sum())
    g = torch.Generator(device="cpu").manual_seed(7)
    wr = torch.randn(rho_t.shape, generator=g, dtype=F64).to(dev)
    wj = torch.randn(j_t.shape, generator=g, dtype=F64).to(dev)
    wr /= float(torch.linalg.norm(wr)) * scale_r ** 0.5
    wj /= float(torch.linalg.norm(wj)) * scale_j ** 0.5

    def loss(rho, j):
        return ((wr * rho).sum() + (wj * j).sum() + ((j - j_t) ** 2).sum() / scale_j
                + ((rho - rho_t) ** 2).sum() / scale_r)

    return dict(w=w, m=m, sf=sf, basis=basis, theta=theta, q=q, mass=mass, x0=x0, p0=p0,
                traj=traj, loss=loss, dev=dev)


def record(S, x0, p0, F, stages):
    """Run `stages` recorded stages from (x0, p0) in the given particle order;
    returns the per-stage input elements and the final state."""
    m = S["m"]
    lib = m.lib
    n = x0.shape[1]
    el = m.find_containing_elements_device(x0)
    x, p = x0.clone(), p0.clone()
    kx = torch.zeros_like(x)
    kp = torch.zeros_like(p)
    Fp = _ptrs(_field_components(F))
    els = []
    for t in range(stages):
        xo, po, elo = torch.empty_like(x), torch.empty_like(p), torch.empty_like(el)
        _lib.check(lib.prt_lsrk_stage_record(
            m.pusher.handle, m.workspace, n, x.data_ptr(), p.data_ptr(), el.data_ptr(),
            xo.data_ptr(), po.data_ptr(), elo.data_ptr(), S["q"].data_ptr(),
            S["mass"].data_ptr(), kx.data_ptr(), kp.data_ptr(), Fp, LSRK4_A[t % 5],
            LSRK4_B[t % 5], S["w"].dt, C_LIGHT, C.c_void_p(stream_handle())))
        els.append(el.long())
        x, p, el = xo, po, elo
    return els, (x, p, el, kx, kp)


def fields_of(S, theta):
    return torch.einsum("k,kcn->cn", theta, S["basis"]).contiguous()


def test_recorded_stage_is_bitwise_the_in_place_stage(S):
    m, lib = S["m"], S["m"].lib
    F = fields_of(S, S["theta"])
    els, (xr, pr, elr, kxr, kpr) = record(S, S["x0"], S["p0"], F, 7)
    x, p = S["x0"].clone(), S["p0"].clone()
    el = m.find_containing_elements_device(x)
    kx = torch.zeros_like(x)
    kp = torch.zeros_like(p)
    Fp = _ptrs(_field_components(F))
    for t in range(7):
        _lib.check(lib.prt_lsrk_stage(
            m.pusher.handle, m.workspace, x.shape[1], x.data_ptr(), p.data_ptr(),
            S["q"].data_ptr(), S["mass"].data_ptr(), el.data_ptr(), kx.data_ptr(),
            kp.data_ptr(), Fp, LSRK4_A[t % 5], LSRK4_B[t % 5], S["w"].dt, C_LIGHT, 0,
            C.c_void_p(stream_handle())))
    assert torch.equal(x, xr) and torch.equal(p, pr) and torch.equal(el, elr)
    assert torch.equal(kx, kxr) and torch.equal(kp, kpr)


def stage_adjoint(S, x, p, el, F, a, b, lam, basis_count=2):
    m, lib, w = S["m"], S["m"].lib, S["w"]
    lx, lp, lkx, lkp = [l.clone() for l in lam]
    gth = torch.zeros(2, dtype=F64, device=x.device)
    bcoef = monomial_coefficients(
        m, _field_components(S["basis"][0]) + _field_components(S["basis"][1]))
    fcoef = monomial_coefficients(m, _field_components(F))
    _lib.check(lib.prt_lsrk_stage_adjoint(
        m.pusher.handle, m.workspace, x.shape[1], x.data_ptr(), p.data_ptr(), el.data_ptr(),
        S["q"].data_ptr(), S["mass"].data_ptr(), lx.data_ptr(), lp.data_ptr(), lkx.data_ptr(),
        lkp.data_ptr(), _ptrs(fcoef), a, b, w.dt, C_LIGHT, None, basis_count,
        _ptrs(bcoef), gth.data_ptr(), C.c_void_p(stream_handle())))
    return lx, lp, lkx, lkp, gth


def stage_autograd(S, x, p, kx, kp, el, a, b, lam):
    w = S["w"]
    xr = x.clone().requires_grad_()
    pr = p.clone().requires_grad_()
    kxr = kx.clone().requires_grad_()
    kpr = kp.clone().requires_grad_()
    thr = S["theta"].clone().requires_grad_()
    Fr = torch.einsum("k,kcn->cn", thr, S["basis"])
    W = R.lagrange_weights(w.order, x.device)
    inv_maps = torch.as_tensor(w.mesh.inverse_maps, dtype=F64, device=x.device)
    xo, po, kxo, kpo = R.stage(xr, pr, kxr, kpr, el.long(), S["q"], S["mass"], Fr, inv_maps, W,
                               w.order, a, b, w.dt, C_LIGHT)
    (xo * lam[0] + po * lam[1] + kxo * lam[2] + kpo * lam[3]).sum().backward()
    return xr.grad, pr.grad, kxr.grad, kpr.grad, thr.grad


def test_stage_adjoint_matches_autograd(S):
    """One stage (a != 0: the third) from a state mid-step. Run A: adjoints
    only on the residuals, so every output is a pure derivative term (the
    field-gradient term is ~1e-7 of an identity term and would drown in it).
    Run B: all four adjoints, checking the b coupling."""
    F = fields_of(S, S["theta"])
    els, (x, p, el, kx, kp) = record(S, S["x0"], S["p0"], F, 2)
    assert bool((el >= 0).all())
    t = 2
    a, b = LSRK4_A[t], LSRK4_B[t]
    g = torch.Generator(device="cpu").manual_seed(3)
    xs = S["sf"].radius
    ps = float(torch.sqrt((p ** 2).sum(0).mean()))
    rnd = [torch.randn(x.shape, generator=g, dtype=F64).to(x.device) for _ in range(4)]
    zero = torch.zeros_like(x)
    lamA = [zero, zero, rnd[2] / xs, rnd[3] / ps]
    mine = stage_adjoint(S, x, p, el, F, a, b, lamA)
    ref = stage_autograd(S, x, p, kx, kp, el, a, b, lamA)
    for u, v in zip(mine, ref):
        assert rel(u, v) < 1e-11
    lamB = [rnd[0] / xs, rnd[1] / ps, rnd[2] / xs, rnd[3] / ps]
    mine = stage_adjoint(S, x, p, el, F, a, b, lamB)
    ref = stage_autograd(S, x, p, kx, kp, el, a, b, lamB)
    for u, v in zip(mine, ref):
        assert rel(u, v) < 1e-12


def test_deposit_adjoint_matches_autograd(S):
    m, lib, w, sf = S["m"], S["m"].lib, S["w"], S["sf"]
    F = fields_of(S, S["theta"])
    _, (x, p, el, _, _) = record(S, S["x0"], S["p0"], F, 5)
    n = x.shape[1]
    g = torch.Generator(device="cpu").manual_seed(5)
    nn = len(m.discretization)
    grho = torch.randn(nn, generator=g, dtype=F64).to(x.device)
    gj = torch.randn((3, nn), generator=g, dtype=F64).to(x.device)
    nodes = torch.as_tensor(w.nodes, dtype=F64, device=x.device)
    xr = x.clone().requires_grad_()
    pr = p.clone().requires_grad_()
    rho, j = R.deposit(xr, pr, S["q"], S["mass"], C_LIGHT, nodes, sf.radius, sf.exponent,
                       sf.normalizer)
    ((rho * grho).sum() + (j * gj).sum()).backward()
    v = torch.empty_like(p)
    _lib.check(lib.prt_get_velocities(n, p.data_ptr(), S["mass"].data_ptr(), C_LIGHT,
                                      v.data_ptr(), C.c_void_p(stream_handle())))
    lx = torch.zeros_like(x)
    lv = torch.zeros_like(x)
    lp = torch.zeros_like(x)
    _lib.check(lib.prt_deposit_shape_adjoint(
        m.mesh_data.handle, m.workspace, m.depositor._shape_desc(), n, x.data_ptr(),
        S["q"].data_ptr(), v.data_ptr(), el.data_ptr(), grho.data_ptr(), gj.data_ptr(),
        lx.data_ptr(), lv.data_ptr(), C.c_void_p(stream_handle())))
    _lib.check(lib.prt_velocities_adjoint(n, p.data_ptr(), S["mass"].data_ptr(), C_LIGHT,
                                          lv.data_ptr(), lp.data_ptr(),
                                          C.c_void_p(stream_handle())))
    assert rel(lx, xr.grad) < 1e-11
    assert rel(lp, pr.grad) < 1e-11


def gradients(S, traj, x0, p0, theta, fields=None):
    x0 = x0.clone().requires_grad_()
    p0 = p0.clone().requires_grad_()
    th = theta.clone().requires_grad_()
    if fields is not None:
        fields = fields.clone().requires_grad_()
    rho, j = traj(x0, p0, th, fields)
    L = S["loss"](rho, j)
    L.backward()
    return L.detach(), x0.grad, p0.grad, th.grad, (fields.grad if fields is not None else None)


def test_trajectory_gradient_matches_autograd_reference(S):
    """Full DifferentiableTrajectory (sort + 3 checkpointed segments +
    recomputation) against torch autograd through the restated forward."""
    w = S["w"]
    L, gx, gp, gth, _ = gradients(S, S["traj"], S["x0"], S["p0"], S["theta"])
    F = fields_of(S, S["theta"])
    els, _ = record(S, S["x0"], S["p0"], F, 5 * STEPS)
    assert all(bool((e >= 0).all()) for e in els)
    dev = S["x0"].device
    W = R.lagrange_weights(w.order, dev)
    inv_maps = torch.as_tensor(w.mesh.inverse_maps, dtype=F64, device=dev)
    nodes = torch.as_tensor(w.nodes, dtype=F64, device=dev)
    xr = S["x0"].clone().requires_grad_()
    pr = S["p0"].clone().requires_grad_()
    thr = S["theta"].clone().requires_grad_()
    Fr = torch.einsum("k,kcn->cn", thr, S["basis"])
    xf, pf = R.trajectory(xr, pr, Fr, S["q"], S["mass"], els, inv_maps, W, w.order, w.dt,
                          C_LIGHT)
    sf = S["sf"]
    rho, j = R.deposit(xf, pf, S["q"], S["mass"], C_LIGHT, nodes, sf.radius, sf.exponent,
                       sf.normalizer)
    Lr = S["loss"](rho, j)
    Lr.backward()
    assert abs(float(L) - float(Lr)) <= 1e-10 * abs(float(Lr))
    assert rel(gp, pr.grad) < 1e-9
    assert rel(gx, xr.grad) < 1e-9
    assert rel(gth, thr.grad) < 1e-9


def test_trajectory_gradient_central_differences(S):
    """Central differences, h = 1e-6 (relative), on 64 random directions in
    (initial momenta, Bz, focusing gradient), and 16 in initial positions."""
    traj, loss = S["traj"], S["loss"]
    x0, p0, theta = S["x0"], S["p0"], S["theta"]
    _, gx, gp, gth, _ = gradients(S, traj, x0, p0, theta)
    h = 1e-6
    pscale = float(torch.sqrt((p0 ** 2).sum(0).mean()))
    g = torch.Generator(device="cpu").manual_seed(11)

    def L(x, p, th):
        with torch.no_grad():
            return float(loss(*traj(x, p, th)))

    worst = 0.0
    for k in range(64):
        dp = torch.randn(p0.shape, generator=g, dtype=F64).to(p0.device) * pscale
        dth = torch.randn(2, generator=g, dtype=F64).to(p0.device) * theta
        fd = (L(x0, p0 + h * dp, theta + h * dth) - L(x0, p0 - h * dp, theta - h * dth)) / (2 * h)
        ad = float((gp * dp).sum() + (gth * dth).sum())
        worst = max(worst, abs(fd - ad) / abs(ad))
    assert worst < 1e-5, worst
    xscale = S["sf"].radius
    worst = 0.0
    for k in range(16):
        dx = torch.randn(x0.shape, generator=g, dtype=F64).to(x0.device) * xscale
        fd = (L(x0 + h * dx, p0, theta) - L(x0 - h * dx, p0, theta)) / (2 * h)
        ad = float((gx * dx).sum())
        worst = max(worst, abs(fd - ad) / abs(ad))
    assert worst < 1e-5, worst


def test_nodal_field_gradient_matches_basis_gradient(S):
    """dL/dtheta_k = <dL/dF, basis_k>: the atomic nodal scatter against the
    deterministic per-block basis reduction."""
    x0, p0 = S["x0"], S["p0"]
    zero = torch.zeros_like(S["basis"][0])
    _, _, gp, gth, gF = gradients(S, S["traj"], x0, p0, S["theta"], fields=zero)
    proj = torch.einsum("cn,kcn->k", gF, S["basis"])
    assert rel(proj, gth) < 1e-10
    _, _, gp2, gth2, _ = gradients(S, S["traj"], x0, p0, S["theta"])
    assert rel(gp, gp2) < 1e-13


def test_adjoint_is_deterministic(S):
    a = gradients(S, S["traj"], S["x0"], S["p0"], S["theta"])
    b = gradients(S, S["traj"], S["x0"], S["p0"], S["theta"])
    for u, v in zip(a[:4], b[:4]):
        assert torch.equal(u, v)


def test_mixed_precision_forward_gradient_close_to_fp64(S):
    """FP32 deposition in the forward (the chosen form), FP64 check run."""
    m = S["m"]
    traj32 = DifferentiableTrajectory(m, S["q"], S["mass"], S["w"].dt, STEPS,
                                      checkpoint_every=K, basis=S["basis"], precision="mixed")
    L64, _, gp64, gth64, _ = gradients(S, S["traj"], S["x0"], S["p0"], S["theta"])
    L32, _, gp32, gth32, _ = gradients(S, traj32, S["x0"], S["p0"], S["theta"])
    assert abs(float(L32) - float(L64)) <= 1e-5 * abs(float(L64))
    assert rel(gp32, gp64) < 1e-4
    assert rel(gth32, gth64) < 1e-4


def test_graph_replay_matches_eager(S):
    """The segments replayed from the captured CUDA graph give bitwise the
    gradients of eager launches."""
    traj = S["traj"]
    traj.use_graphs = False
    try:
        a = gradients(S, traj, S["x0"], S["p0"], S["theta"])
    finally:
        traj.use_graphs = True
    b = gradients(S, traj, S["x0"], S["p0"], S["theta"])
    for u, v in zip(a[:4], b[:4]):
        assert torch.equal(u, v)
