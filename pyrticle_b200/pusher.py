"""Particle pushers (the reference's ``pyrticle/pusher.py``)."""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .refelement import monomial_vandermonde


class EmptyPusherState:
    pass


class Pusher:
    def initialize(self, method):
        self.method = method

    def make_state(self, state):
        return EmptyPusherState()

    def advance_state(self, state):
        return state.pusher_state

    def upkeep(self, state):
        pass

    def add_instrumentation(self, mgr, observer):
        """Log constant: the pusher's class (pusher.py:54-57)."""
        if hasattr(mgr, "set_constant"):
            mgr.set_constant("pusher", self.__class__.__name__)

    def note_move(self, state, orig, dest, size):
        pass

    def note_change_size(self, state, count):
        pass


class MonomialParticlePusher(Pusher):
    """Field interpolation with a monomial basis and the Lorentz force
    (pusher.py:86-114, push_monomial.hpp)."""

    def initialize(self, method):
        Pusher.initialize(self, method)
        lib = _lib.load()
        ldis = method.discretization.element_groups[0].local_discretization
        self.exponents = np.ascontiguousarray(ldis.node_tuples(), dtype=np.uint32)
        self.vandermonde = np.ascontiguousarray(
            monomial_vandermonde(ldis.unit_nodes(), ldis.node_tuples()))
        h = C.c_void_p()
        _lib.check(lib.prt_monomial_pusher_create(
            method.mesh_data.handle, len(self.exponents),
            _lib.ptr(self.exponents, C.c_uint32), _lib.ptr(self.vandermonde), C.byref(h)),
            "prt_monomial_pusher_create")
        self.handle = h
        self.lib = lib

    def __del__(self):
        if getattr(self, "handle", None) is not None and _lib._lib is not None:
            _lib._lib.prt_monomial_pusher_destroy(self.handle)
            self.handle = None

    def lsrk_stage(self, state, fptrs, kx, kp, a, b, dt, c, precision=0):
        """One fused low-storage RK stage of the whole store (prt_lsrk_stage)."""
        m = self.method
        _lib.check(self.lib.prt_lsrk_stage(
            self.handle, m.workspace, len(state), state.x.data_ptr(), state.p.data_ptr(),
            state.q.data_ptr(), state.m.data_ptr(), state.el.data_ptr(), kx.data_ptr(),
            kp.data_ptr(), fptrs, a, b, dt, c, precision,
            C.c_void_p(torch.cuda.current_stream().cuda_stream)), "prt_lsrk_stage")

    def field_pointers(self, fields):
        """Pointer array for six device field components (None = zero)."""
        arr = (C.c_void_p * 6)()
        if fields is None:
            return arr
        comps = list(fields) if not isinstance(fields, torch.Tensor) else [fields[k] for k in range(6)]
        self._keep = []
        for k, f in enumerate(comps):
            if f is None:
                arr[k] = None
                continue
            if not isinstance(f, torch.Tensor):
                f = torch.as_tensor(np.ascontiguousarray(f, dtype=np.float64),
                                    device=self.method.dev)
            f = f.contiguous()
            assert f.dtype == torch.float64 and f.is_cuda
            self._keep.append(f)
            arr[k] = f.data_ptr()
        return arr

    def forces_device(self, state, velocities, *field_args, vis=False):
        n = len(state)
        out = torch.empty_like(state.x)
        visbuf = torch.empty((4, 3, n), dtype=torch.float64, device=state.x.device) if vis else None
        fptrs = self.field_pointers(field_args if field_args else None)
        _lib.check(self.lib.prt_forces(
            self.handle, n, state.x.data_ptr(), state.el.data_ptr(), state.q.data_ptr(),
            velocities.data_ptr(), fptrs, out.data_ptr(),
            visbuf.data_ptr() if vis else None,
            C.c_void_p(torch.cuda.current_stream().cuda_stream)), "prt_forces")
        return out, visbuf

    def forces(self, state, velocities, *field_args):
        """Host [n, 3] forces in id order; ``velocities`` as returned by
        PicMethod.velocities. Field components may be None (ZeroVector)."""
        from .cloud import to_store_from_id
        order = state.id_order()
        vdev = to_store_from_id(velocities, order, state.x.device)
        vis = "verbose_vis" in self.method.debug
        out, visbuf = self.forces_device(state, vdev, *field_args, vis=vis)
        if vis:
            for k, name in enumerate(("pt_e", "pt_b", "el_force", "mag_force")):
                state.vis_listener.store_particle_vis_vector(
                    name, visbuf[k][:, order].T.contiguous().cpu().numpy())
        return out[:, order].T.contiguous().cpu().numpy()


class AveragePusherState:
    """Normalisation statistics of the last force evaluation
    (push_average.hpp:330-340)."""

    def __init__(self):
        from .tools import StatsGatherer
        self.e_normalization_stats = StatsGatherer()
        self.b_normalization_stats = StatsGatherer()


class AverageParticlePusher(MonomialParticlePusher):
    """Forces from the fields averaged over the depositor's shape, weighted by
    the integration weights (pusher.py:167-207, push_average.hpp): q <E> +
    v x (q <B>). Uses the method's depositor's shape function; the field
    pointer handling and stage plumbing come from the monomial pusher."""

    def initialize(self, method):
        MonomialParticlePusher.initialize(self, method)
        ldis = method.discretization.element_groups[0].local_discretization
        # w = M 1 (push_average.hpp:343-350)
        self.integral_weights = np.ascontiguousarray(ldis.mass_matrix().sum(axis=1))

    def make_state(self, state):
        return AveragePusherState()

    def _shape_desc(self):
        sf = self.method.depositor.shape_function
        if sf is None:
            raise RuntimeError("shape function never set")
        return _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer)

    def forces_device(self, state, velocities, *field_args, vis=False, stats=True):
        m = self.method
        n = len(state)
        out = torch.empty_like(state.x)
        visbuf = torch.empty((14, n), dtype=torch.float64, device=state.x.device) if vis else None
        scales = torch.empty((n,), dtype=torch.float64, device=state.x.device) if stats else None
        fptrs = self.field_pointers(field_args if field_args else None)
        _lib.check(self.lib.prt_average_forces(
            m.mesh_data.handle, m.workspace, self._shape_desc(),
            _lib.ptr(self.integral_weights), n, state.x.data_ptr(), state.q.data_ptr(),
            velocities.data_ptr(), state.el.data_ptr(), fptrs, out.data_ptr(),
            visbuf.data_ptr() if vis else None, scales.data_ptr() if stats else None,
            C.c_void_p(torch.cuda.current_stream().cuda_stream)), "prt_average_forces")
        if stats and state.pusher_state is not None and n:
            sc = scales[scales != 0].cpu().numpy()
            for st in (state.pusher_state.e_normalization_stats,
                       state.pusher_state.b_normalization_stats):
                st.reset()
                if len(sc):
                    st.add_moments(len(sc), float(sc.sum()), float((sc * sc).sum()),
                                   float(sc.min()), float(sc.max()))
        m.check_status()
        return out, visbuf

    def forces(self, state, velocities, *field_args):
        """Host [n, 3] forces in id order; with ``verbose_vis`` the vectors
        el_force, mag_force, pt_e, pt_b, pt_e_stddev, pt_b_stddev
        (push_average.hpp:409-418) go to the state's vis listener."""
        from .cloud import to_store_from_id
        order = state.id_order()
        vdev = to_store_from_id(velocities, order, state.x.device)
        vis = "verbose_vis" in self.method.debug
        out, visbuf = self.forces_device(state, vdev, *field_args, vis=vis)
        if vis:
            rows = {"pt_e": visbuf[0:3], "pt_b": visbuf[3:6], "el_force": visbuf[8:11],
                    "mag_force": visbuf[11:14]}
            for name, t in rows.items():
                state.vis_listener.store_particle_vis_vector(
                    name, t[:, order].T.contiguous().cpu().numpy())
            state.vis_listener.store_particle_vis_vector(
                "pt_e_stddev", visbuf[6][order].cpu().numpy())
            state.vis_listener.store_particle_vis_vector(
                "pt_b_stddev", visbuf[7][order].cpu().numpy())
        return out[:, order].T.contiguous().cpu().numpy()

    def lsrk_stage(self, state, fptrs, kx, kp, a, b, dt, c, precision=0):
        """Velocities, averaged forces, then the RK update with relocation."""
        m = self.method
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        n = len(state)
        v = torch.empty_like(state.p)
        _lib.check(self.lib.prt_get_velocities(n, state.p.data_ptr(), state.m.data_ptr(), c,
                                               v.data_ptr(), stream), "prt_get_velocities")
        f = torch.empty_like(state.x)
        _lib.check(self.lib.prt_average_forces(
            m.mesh_data.handle, m.workspace, self._shape_desc(),
            _lib.ptr(self.integral_weights), n, state.x.data_ptr(), state.q.data_ptr(),
            v.data_ptr(), state.el.data_ptr(), fptrs, f.data_ptr(), None, None, stream),
            "prt_average_forces")
        _lib.check(self.lib.prt_lsrk_update(
            m.mesh_data.handle, m.workspace, n, state.x.data_ptr(), state.p.data_ptr(),
            state.m.data_ptr(), state.el.data_ptr(), kx.data_ptr(), kp.data_ptr(),
            f.data_ptr(), a, b, dt, c, stream), "prt_lsrk_update")
