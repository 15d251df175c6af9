"""Particle sharding over ranks (one process per GPU, torch.distributed).

The particle side of a PIC step partitions by particle: every rank pushes its
own particles and deposits them onto the full node vectors; the only exchange
is the sum of the per-rank rho and j (one all-reduce each), after which every
rank holds the global densities (the reference is single-process; its
deposition is a sum over particles, dep_target.hpp:203-273, so any partition
of the particles gives the same sum up to the order of the additions).
"""

from __future__ import annotations


def shard_slice(n: int, rank: int, world: int) -> slice:
    """Contiguous block of particles [start, stop) owned by `rank`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def allreduce_densities(rho, j, group=None):
    """Sum rho [Nn] and j [3, Nn] over the ranks, in place (either may be
    None). Every rank must call it, in the same order, once per deposition."""
    import torch.distributed as dist
    for t in (rho, j):
        if t is not None:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return rho, j


def max_over_ranks(value: float, device, group=None) -> float:
    """The largest of the ranks' values (a time, for the slowest rank)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def exact_deposit_protocol(charges, sums, combine, allreduce_max, allreduce_sum):
    """The collectives of the sharded chosen-form deposition, in order.

    ``charges()`` returns this rank's four charge maxima (|c|, |c vx|,
    |c vy|, |c vz|), ``allreduce_max`` makes them global in place;
    ``sums(global_max)`` returns this rank's digit sums per node position,
    integers held in FP64, which ``allreduce_sum`` adds in place (exactly:
    integers below 2^53 add without rounding in any order);
    ``combine(global_max, sums)`` returns (rho, j). Every rank calls it with
    the same sequence of collectives, so the result is bitwise the same for
    any number of ranks and any split of the particles."""
    gmax = charges()
    allreduce_max(gmax)
    partial = sums(gmax)
    allreduce_sum(partial)
    return combine(gmax, partial)


def deposit_densities_exact(method, state, group=None, rho=True, j=True):
    """rho [Nn] and j [3, Nn] of the particles of every rank (each rank
    passes its own ``state``), through the tensor-core deposition split
    around two collectives (prt_deposit_shape_charges / _sums / _combine).
    With torch.distributed not initialised it is the single-process
    deposition. The method's depositor decides plain or normalising mode."""
    import ctypes as C

    import torch
    import torch.distributed as dist

    from . import _lib

    dep = method.depositor
    lib = method.lib
    dev = state.x.device
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    sf = dep.shape_function
    desc = _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer)
    iw = getattr(dep, "integral_weights", None)
    npos = C.c_int64()
    _lib.check(lib.prt_mesh_position_count(method.mesh_data.handle, C.byref(npos)),
               "prt_mesh_position_count")
    n = len(state)
    v = method.velocities_device(state)
    multi = dist.is_available() and dist.is_initialized()

    def charges():
        mx = torch.zeros(4, dtype=torch.float64, device=dev)
        if n:
            _lib.check(lib.prt_deposit_shape_charges(
                method.mesh_data.handle, method.workspace, dep.mode, desc,
                _lib.ptr(iw) if iw is not None else None, n, state.x.data_ptr(),
                state.q.data_ptr(), v.data_ptr(), state.el.data_ptr(), mx.data_ptr(), None,
                stream), "prt_deposit_shape_charges")
        return mx

    def sums(gmax):
        out = torch.zeros((16, npos.value), dtype=torch.float64, device=dev)
        if n:
            _lib.check(lib.prt_deposit_shape_sums(
                method.mesh_data.handle, method.workspace, desc, n, gmax.data_ptr(),
                out.data_ptr(), stream), "prt_deposit_shape_sums")
        return out

    def combine(gmax, partial):
        r, jj = dep._outputs(state)
        _lib.check(lib.prt_deposit_shape_combine(
            method.mesh_data.handle, method.workspace, desc, gmax.data_ptr(),
            partial.data_ptr(), r.data_ptr() if rho else None, jj.data_ptr() if j else None,
            stream), "prt_deposit_shape_combine")
        method.check_status()
        return r, jj

    def ar(op):
        def f(t):
            if multi:
                dist.all_reduce(t, op=op, group=group)
        return f

    return exact_deposit_protocol(charges, sums, combine, ar(dist.ReduceOp.MAX if multi else None),
                                  ar(dist.ReduceOp.SUM if multi else None))
