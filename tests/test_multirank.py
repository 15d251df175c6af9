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
