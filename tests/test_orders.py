"""Element orders 1 and 4 through the device path (config4 runs at order 4;
the other workloads at 2 and 3): LSRK4 steps, element ids and the plain
deposition against the oracle (1e-12 relative L2, ids equal), and the
tensor-core stage (chosen form) against the FP64 stage: forces within 1e-5,
positions after 20 steps within 1e-9 relative L2.
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import pyoracle as O  # noqa: E402
from pyrticle_b200 import _lib, meshgen, problems, refelement  # noqa: E402
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B, PicMethod, stream_handle  # noqa: E402
from pyrticle_b200.deposition.shape import ShapeFunctionDepositor  # noqa: E402
from pyrticle_b200.discretization import Discretization  # noqa: E402
from pyrticle_b200.pusher import MonomialParticlePusher  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402

from conftest import rel_l2  # noqa: E402

pytestmark = pytest.mark.gpu
C_LIGHT = U.VACUUM_LIGHT_SPEED()
CM = 1e-2


def case(order, n=400, seed=3):
    mesh = meshgen.box_mesh((4, 4, 8), (0, 0, 0), (CM, CM, 2 * CM), jitter=0.15, seed=0)
    nodes = meshgen.element_nodes(mesh, order)
    rng = np.random.default_rng(seed)
    x = np.column_stack([rng.uniform(0.2 * CM, 0.8 * CM, n), rng.uniform(0.2 * CM, 0.8 * CM, n),
                         rng.uniform(0.3 * CM, 1.7 * CM, n)])
    gamma = 2.0
    pz = gamma * U.EL_MASS * C_LIGHT * (1 - 1 / gamma ** 2) ** 0.5
    p = np.column_stack([rng.normal(size=n) * 1e-2 * pz, rng.normal(size=n) * 1e-2 * pz,
                         np.full(n, pz)])
    q = np.full(n, -U.EL_CHARGE)
    m = np.full(n, U.EL_MASS)
    # smooth nodal fields, curved enough that the order matters
    X, Y, Z = (nodes[:, 0] - 0.5 * CM) / CM, (nodes[:, 1] - 0.5 * CM) / CM, nodes[:, 2] / CM
    fields = np.zeros((6, len(nodes)))
    fields[0] = -1e6 * CM * X * (1 + 0.3 * np.sin(2.1 * Z))
    fields[1] = -1e6 * CM * Y * (1 + 0.3 * np.cos(1.7 * Z))
    fields[2] = 2e4 * np.sin(3.0 * X * Y + Z)
    fields[5] = 0.1 * (1 + 0.2 * X ** 2 - 0.1 * Y ** 3)
    return mesh, nodes, x, p, q, m, fields


@pytest.mark.parametrize("order", [1, 4])
def test_order_parity_with_oracle(order):
    mesh, nodes, x, p, q, m, fields = case(order)
    dt = problems.stable_dt(mesh)
    meth = PicMethod(Discretization(mesh, order, nodes=nodes), U, ShapeFunctionDepositor(),
                     MonomialParticlePusher(), 3, 3)
    sf = PolynomialShapeFunction(0.3 * CM, 3, 2)
    meth.depositor.set_shape_function(None, sf)
    s = meth.make_state()
    meth.add_particles_from_arrays(s, x, p, q, m)
    steps = 10
    meth.step(s, torch.as_tensor(fields, device="cuda"), dt, steps=steps, deposit=False)

    om = O.OracleMesh(mesh, nodes, meshgen.element_bins(mesh))
    ex = refelement.node_tuples(order)
    pu = O.OraclePusher(ex, refelement.monomial_vandermonde(refelement.unit_nodes(order), ex))
    el0 = O.find_containing_elements(om, x)
    r = O.lsrk_steps(pu, om, x, p, q, m, el0, list(fields), LSRK4_A, LSRK4_B, dt, C_LIGHT, steps)
    idx = np.argsort(r["ids"])
    assert np.array_equal(s.containing_elements, r["el"][idx])
    assert rel_l2(s.positions, r["x"][idx]) < 1e-12
    assert rel_l2(s.momenta, r["p"][idx]) < 1e-12

    rho, j = meth.deposit_densities(s)
    ro, jo, _, _ = O.deposit_shape(om, 0, sf, s.positions, s.charges, meth.velocities(s),
                                   s.containing_elements)
    assert rel_l2(rho, ro) < 1e-12 and rel_l2(j, jo.T) < 1e-12
    assert np.count_nonzero(ro) > 0


@pytest.mark.parametrize("order", [1, 4])
def test_tensor_core_stage_at_order(order):
    mesh, nodes, x, p, q, m, fields = case(order, n=2000, seed=5)
    dt = problems.stable_dt(mesh)
    meth = PicMethod(Discretization(mesh, order, nodes=nodes), U, ShapeFunctionDepositor(),
                     MonomialParticlePusher(), 3, 3)
    s = meth.make_state()
    meth.add_particles_from_arrays(s, x, p, q, m)
    f = torch.as_tensor(fields, device="cuda")
    fp = meth.pusher.field_pointers(f)

    def run(stages, precision):
        xx, pp, el = s.x.clone(), s.p.clone(), s.el.clone()
        kx = torch.zeros_like(xx)
        kp = torch.zeros_like(pp)
        for t in range(stages):
            _lib.check(meth.lib.prt_lsrk_stage(
                meth.pusher.handle, meth.workspace, xx.shape[1], xx.data_ptr(), pp.data_ptr(),
                s.q.data_ptr(), s.m.data_ptr(), el.data_ptr(), kx.data_ptr(), kp.data_ptr(), fp,
                LSRK4_A[t % 5], LSRK4_B[t % 5], dt, C_LIGHT, precision,
                C.c_void_p(stream_handle())), "prt_lsrk_stage")
        meth.check_status()
        return xx, pp, el, kp

    kp64 = run(1, 0)[3]
    kp32 = run(1, 1)[3]
    ef = float(torch.linalg.norm(kp32 - kp64) / torch.linalg.norm(kp64))
    assert 0 < ef < 1e-5, ef
    x64, _, el64, _ = run(100, 0)
    x32, _, el32, _ = run(100, 1)
    assert float(torch.linalg.norm(x32 - x64) / torch.linalg.norm(x64)) < 1e-9
    assert float((el32 == el64).float().mean()) > 0.999
