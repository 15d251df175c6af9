"""Two ranks on CPU (gloo, 127.0.0.1): the sharded particle step — each rank
pushes its own particles and deposits them, then one all-reduce of rho and j —
gives the single-process result. The per-rank compute here is the oracle
(CPU); on GPUs it is libprt, with the same sharding and collectives
(bench.py, pyrticle_b200.sharding)."""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from pyrticle_b200.sharding import allreduce_densities, max_over_ranks, shard_slice  # noqa: E402


def test_shard_slices_partition_the_particles():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            covered = []
            for r in range(world):
                sl = shard_slice(n, r, world)
                covered.extend(range(sl.start, sl.stop))
            assert covered == list(range(n))
    with pytest.raises(ValueError):
        shard_slice(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from oracle import pyoracle as O
        from pyrticle_b200 import meshgen, problems, refelement
        from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
        from pyrticle_b200.tools import PolynomialShapeFunction
        from pyrticle_b200.units import SIUnitsWithNaturalConstants as U
        w = problems.make("config0", scale=0.02)
        om = O.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
        ex = refelement.node_tuples(w.order)
        pu = O.OraclePusher(ex, refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex))
        c = U.VACUUM_LIGHT_SPEED()
        sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
        sl = shard_slice(w.particle_count, rank, world)
        x, p, q, m = w.positions[sl], w.momenta[sl], w.charges[sl], w.masses[sl]
        el = O.find_containing_elements(om, x)
        r = O.lsrk_steps(pu, om, x, p, q, m, el, w.fields, LSRK4_A, LSRK4_B, w.dt, c, 3)
        rho, j, _, _ = O.deposit_shape(om, 0, sf, r["x"], r["q"], O.velocities(r["p"], r["m"], c),
                                       r["el"])
        trho = torch.as_tensor(rho)
        tj = torch.as_tensor(np.ascontiguousarray(j.T))
        allreduce_densities(trho, tj)
        slowest = max_over_ranks(float(rank + 1), "cpu")
        if rank == 0:
            out.put((trho.numpy(), tj.numpy(), slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_single_process_step():
    from oracle import pyoracle as O
    from pyrticle_b200 import meshgen, problems, refelement
    from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
    from pyrticle_b200.tools import PolynomialShapeFunction
    from pyrticle_b200.units import SIUnitsWithNaturalConstants as U
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run_rank, args=(r, 2, port, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    rho2, j2, slowest = out.get(timeout=180)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    assert slowest == 2.0
    w = problems.make("config0", scale=0.02)
    om = O.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
    ex = refelement.node_tuples(w.order)
    pu = O.OraclePusher(ex, refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex))
    c = U.VACUUM_LIGHT_SPEED()
    el = O.find_containing_elements(om, w.positions)
    r = O.lsrk_steps(pu, om, w.positions, w.momenta, w.charges, w.masses, el, w.fields, LSRK4_A,
                     LSRK4_B, w.dt, c, 3)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    rho, j, _, _ = O.deposit_shape(om, 0, sf, r["x"], r["q"], O.velocities(r["p"], r["m"], c),
                                   r["el"])
    assert np.linalg.norm(rho2 - rho) <= 1e-12 * np.linalg.norm(rho)
    assert np.linalg.norm(j2 - j.T) <= 1e-12 * np.linalg.norm(j)


# ---- the exact sharded deposition protocol (sharding.exact_deposit_protocol)
#
# The GPU steps (prt_deposit_shape_charges / _sums / _combine) are stood in
# for by the same integer arithmetic in numpy: weights F = round(65525
# max(1 - r^2/a^2, 0)^2), charges and currents as balanced base-256 digits
# scaled by the global maxima, digit sums F @ digits, and the combination.
# The protocol's collectives (max, then exact sum) run on gloo ranks.

def _digits(X, nd):
    out = []
    for _ in range(nd):
        d = ((X + 128) & 255) - 128
        out.append(d)
        X = (X - d) >> 8
    return out


def _exact_steps(pts, x, q, v, a):
    import torch
    d2 = ((pts[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    F = np.rint(65525.0 * np.maximum(1 - d2 / a ** 2, 0) ** 2).astype(np.int64)
    cols = [q, q * v[:, 0], q * v[:, 1], q * v[:, 2]]

    def exps(gmax):
        return [(46 if i == 0 else 22) - (np.frexp(m)[1] if m > 0 else 46 if i == 0 else 22)
                for i, m in enumerate(gmax.tolist())]

    def charges():
        return torch.tensor([np.abs(c).max() if len(c) else 0.0 for c in cols],
                            dtype=torch.float64)

    def sums(gmax):
        E = exps(gmax)
        T = np.zeros((16, len(pts)))
        k = 0
        for i, c in enumerate(cols):
            for dgt in _digits(np.rint(np.ldexp(c, E[i])).astype(np.int64), 6 if i == 0 else 3):
                T[k] = (F @ dgt).astype(np.float64)
                k += 1
        return torch.as_tensor(T)

    def combine(gmax, T):
        E = exps(gmax)
        T = T.numpy()
        r = T[5]
        for i in range(4, -1, -1):
            r = r * 256.0 + T[i]
        out = [np.ldexp(r, -E[0])]
        for d in range(3):
            b = 6 + 3 * d
            out.append(np.ldexp((T[b + 2] * 256.0 + T[b + 1]) * 256.0 + T[b], -E[1 + d]))
        return out

    return charges, sums, combine


def _exact_case():
    rng = np.random.default_rng(11)
    pts = rng.uniform(0, 1, (200, 3))
    x = rng.uniform(0, 1, (3000, 3))
    q = -rng.uniform(0.5, 1.5, 3000) * 1.6e-19
    v = rng.normal(size=(3000, 3)) * 1e7
    return pts, x, q, v, 0.2


def _run_exact_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from pyrticle_b200.sharding import exact_deposit_protocol
        pts, x, q, v, a = _exact_case()
        sl = shard_slice(len(x), rank, world)
        charges, sums, combine = _exact_steps(pts, x[sl], q[sl], v[sl], a)
        res = exact_deposit_protocol(
            charges, sums, combine,
            lambda t: dist.all_reduce(t, op=dist.ReduceOp.MAX),
            lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM))
        if rank == 0:
            out.put([np.asarray(r) for r in res])
    finally:
        dist.destroy_process_group()


def test_exact_protocol_is_bitwise_independent_of_the_rank_count():
    from pyrticle_b200.sharding import exact_deposit_protocol
    pts, x, q, v, a = _exact_case()
    one = exact_deposit_protocol(*_exact_steps(pts, x, q, v, a), lambda t: None, lambda t: None)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run_exact_rank, args=(r, 2, port, out)) for r in range(2)]
    for pr in procs:
        pr.start()
    two = out.get(timeout=180)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for r1, r2 in zip(one, two):
        assert np.array_equal(r1, r2)
    # and the integer weights reproduce the FP64 sum to their rounding
    d2 = ((pts[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    S = 65525.0 * np.maximum(1 - d2 / a ** 2, 0) ** 2
    ref = S @ q
    assert np.linalg.norm(one[0] - ref) <= 1e-5 * np.linalg.norm(ref)
