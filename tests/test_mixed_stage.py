"""The mixed-precision RK stage (tensor-core Lagrange values, 3-term split
BF16 with FP32 accumulation, FP32 field sums, FP64 force/update/locate)
against the FP64 stage on the same inputs.

Bars: forces (the first stage's residual kp = dt F) within 1e-5 relative L2
of FP64 (observed ~1e-7); positions and momenta after 20 LSRK4 steps within
1e-9 relative L2; element ids equal wherever the trajectories did not cross
a face within the position error."""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from pyrticle_b200 import _lib, problems  # noqa: E402
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B, PicMethod, stream_handle  # noqa: E402
from pyrticle_b200.deposition.shape import ShapeFunctionDepositor  # noqa: E402
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

pytestmark = pytest.mark.gpu
C_LIGHT = U.VACUUM_LIGHT_SPEED()


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def setup(name, scale, cubes):
    w = problems.make(name, scale=scale, cubes=cubes)
    m = PicMethod(Discretization(w.mesh, w.order), U, ShapeFunctionDepositor(),
                  MonomialParticlePusher(), 3, 3)
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    fields = torch.as_tensor(w.fields, device="cuda")
    return w, m, s, fields


def run(m, s, fields, dt, stages, precision):
    x, p, el = s.x.clone(), s.p.clone(), s.el.clone()
    kx = torch.zeros_like(x)
    kp = torch.zeros_like(p)
    fp = m.pusher.field_pointers(fields)
    for t in range(stages):
        _lib.check(m.lib.prt_lsrk_stage(
            m.pusher.handle, m.workspace, x.shape[1], x.data_ptr(), p.data_ptr(),
            s.q.data_ptr(), s.m.data_ptr(), el.data_ptr(), kx.data_ptr(), kp.data_ptr(), fp,
            LSRK4_A[t % 5], LSRK4_B[t % 5], dt, C_LIGHT, precision,
            C.c_void_p(stream_handle())), "prt_lsrk_stage")
    m.check_status()
    return x, p, el, kx, kp


@pytest.mark.parametrize("name,scale,cubes", [
    ("config0", 0.2, (8, 8, 32)),          # order 2, focusing fields (linear)
    ("config2", 2e-4, (8, 8, 32)),         # order 3, Fourier-mode fields
])
def test_mixed_stage_forces_and_trajectories(name, scale, cubes):
    w, m, s, fields = setup(name, scale, cubes)
    *_, kp64 = run(m, s, fields, w.dt, 1, 0)
    *_, kp32 = run(m, s, fields, w.dt, 1, 1)
    assert rel(kp32, kp64) < 1e-5
    x64, p64, el64, _, _ = run(m, s, fields, w.dt, 100, 0)
    x32, p32, el32, _, _ = run(m, s, fields, w.dt, 100, 1)
    assert rel(x32, x64) < 1e-9
    assert rel(p32 - s.p, p64 - s.p) < 1e-4
    assert float((el32 == el64).float().mean()) > 0.999


def test_mixed_stage_rejects_nothing_on_empty_and_handles_dead_particles():
    w, m, s, fields = setup("config0", 0.02, (8, 8, 32))
    el = s.el.clone()
    el[::3] = -1  # removed particles are skipped
    x, p = s.x.clone(), s.p.clone()
    kx = torch.zeros_like(x)
    kp = torch.zeros_like(p)
    fp = m.pusher.field_pointers(fields)
    _lib.check(m.lib.prt_lsrk_stage(
        m.pusher.handle, m.workspace, x.shape[1], x.data_ptr(), p.data_ptr(), s.q.data_ptr(),
        s.m.data_ptr(), el.data_ptr(), kx.data_ptr(), kp.data_ptr(), fp, LSRK4_A[0],
        LSRK4_B[0], w.dt, C_LIGHT, 1, C.c_void_p(stream_handle())))
    m.check_status()
    assert torch.equal(x[:, ::3], s.x[:, ::3]) and torch.equal(p[:, ::3], s.p[:, ::3])
    assert bool((kp[:, ::3] == 0).all()) and bool((kp[:, 1::3] != 0).any())
    _lib.check(m.lib.prt_lsrk_stage(
        m.pusher.handle, m.workspace, 0, None, None, None, None, None, None, None, fp,
        0.0, 1.0, w.dt, C_LIGHT, 1, C.c_void_p(stream_handle())))
