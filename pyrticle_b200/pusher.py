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
