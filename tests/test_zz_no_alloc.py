"""prt_deposit_shape_noalloc: the deposition for callers that cannot allocate
device memory while they run (a fixed, pre-reserved memory budget, a
real-time loop that must not stall on an allocation). It takes its scratch
from one static device array instead of a workspace; its results must equal
those of the regular entry point, prt_deposit_shape, call after call, even
though every call reuses what the previous one left in that array.

This file is collected last on purpose (name), so that a run stopping at
the first failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyrticle_b200 import _lib, problems  # noqa: E402
from pyrticle_b200.cloud import PicMethod  # noqa: E402
from pyrticle_b200.deposition.shape import ShapeFunctionDepositor  # noqa: E402
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the parity tolerance of the FP64 plain form


def rel_l2(a, b):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def setup_method():
    w = problems.make("config0", scale=0.2)
    m = PicMethod(Discretization(w.mesh, w.order, nodes=w.nodes), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    m.depositor.set_shape_function(None, sf)
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    return w, m, s, sf


def call_noalloc(m, s, sf, x=None, q=None, v=None, el=None):
    lib = _lib.load()
    x = s.x if x is None else x
    q = s.q if q is None else q
    el = s.el if el is None else el
    v = m.velocities_device(s) if v is None else v
    nn = len(m.discretization)
    rho = torch.full((nn,), float("nan"), dtype=torch.float64, device="cuda")
    j = torch.full((3, nn), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib.prt_deposit_shape_noalloc(
        m.mesh_data.handle, _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer),
        x.shape[1], x.data_ptr(), q.data_ptr(), v.data_ptr(), el.data_ptr(), rho.data_ptr(),
        j.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc, rho, j


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    w, m, s, sf = setup_method()
    rho_ref, j_ref = m.depositor.deposit_densities_device(s)
    torch.cuda.synchronize()
    for _ in range(2):
        rc, rho, j = call_noalloc(m, s, sf)
        assert rc == _lib.PRT_OK
        assert rel_l2(rho, rho_ref) < TOL
        assert rel_l2(j, j_ref) < TOL
    # a smaller particle set next: the scratch still holds the larger call's data
    half = len(s) // 2
    x2 = s.x[:, :half].contiguous()
    q2 = s.q[:half].contiguous()
    el2 = s.el[:half].contiguous()
    v2 = m.velocities_device(s)[:, :half].contiguous()
    rc, rho, j = call_noalloc(m, s, sf, x=x2, q=q2, v=v2, el=el2)
    assert rc == _lib.PRT_OK
    # reference for the half set through the regular entry point
    nn = len(m.discretization)
    rho_h = torch.empty((nn,), dtype=torch.float64, device="cuda")
    j_h = torch.empty((3, nn), dtype=torch.float64, device="cuda")
    lib = _lib.load()
    _lib.check(lib.prt_deposit_shape(
        m.mesh_data.handle, m.workspace, _lib.DEPOSIT_PLAIN,
        _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer), None, half,
        x2.data_ptr(), q2.data_ptr(), v2.data_ptr(), el2.data_ptr(), rho_h.data_ptr(),
        j_h.data_ptr(), 0, None, C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert rel_l2(rho, rho_h) < TOL
    assert rel_l2(j, j_h) < TOL


def test_noalloc_rejects_sizes_beyond_its_capacity():
    """Too many particles for the fixed scratch: a clear error, returned
    before any pointer is used (here all pointers are NULL)."""
    w, m, s, sf = setup_method()
    lib = _lib.load()
    n = _lib.NOALLOC_SCRATCH_BYTES // 64 + 1
    rc = lib.prt_deposit_shape_noalloc(
        m.mesh_data.handle, _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer), n,
        None, None, None, None, None, None, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.PRT_ERR_CAPACITY
