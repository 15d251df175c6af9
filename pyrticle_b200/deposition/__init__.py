"""Depositors (the reference's ``pyrticle/deposition/__init__.py``)."""

from __future__ import annotations

import ctypes as C

import torch

from .. import _lib


class Depositor:
    """Base of the depositors: shape-function bookkeeping and the
    rho / j entry points (deposition/__init__.py:30-143)."""

    def __init__(self):
        self.log_constants = {}
        self.shape_function = None

    def initialize(self, method):
        self.method = method
        self.lib = _lib.load()
        self.shape_function = None

    def set_shape_function(self, state, sf):
        self.shape_function = sf

    def add_instrumentation(self, mgr, observer):
        """Log constants: the depositor's class and its parameters
        (deposition/__init__.py:41-45)."""
        if hasattr(mgr, "set_constant"):
            mgr.set_constant("depositor", self.__class__.__name__)
            for key, value in self.log_constants.items():
                mgr.set_constant(key, value)

    def deposit_hook(self):
        if self.shape_function is None:
            raise RuntimeError("shape function never set")

    def make_state(self, state):
        return None

    def note_move(self, state, orig, dest, size):
        pass

    def note_change_size(self, state, count):
        pass

    def upkeep(self, state):
        pass

    def rhs(self, state):
        return 0

    def advance_state(self, state, rhs):
        return state.depositor_state

    # host-array entry points with the reference's names and layouts:
    # rho [Nn]; j [Nn, 3] (the backend layout, dep_target.hpp:234-255)
    def deposit_densites(self, state, velocities=None):
        rho, j = self.deposit_densities_device(state)
        return rho.cpu().numpy(), j.T.contiguous().cpu().numpy()

    deposit_densities = deposit_densites

    def deposit_j(self, state, velocities=None):
        return self.deposit_densities_device(state)[1].T.contiguous().cpu().numpy()

    def deposit_rho(self, state):
        return self.deposit_densities_device(state)[0].cpu().numpy()

    def _outputs(self, state):
        nn = len(self.method.discretization)
        dev = state.x.device
        return (torch.empty((nn,), dtype=torch.float64, device=dev),
                torch.empty((3, nn), dtype=torch.float64, device=dev))

    @staticmethod
    def _stream():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
