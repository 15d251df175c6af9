"""Shape-function depositors (the reference's ``deposition/shape.py``,
``dep_shape.hpp`` and ``dep_normshape.hpp``)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib
from ..tools import StatsGatherer
from . import Depositor


class NormalizationStats:
    """Per-state statistics of the normalising depositor (dep_normshape.hpp:42-47)."""

    def __init__(self):
        self.normalization_stats = StatsGatherer()
        self.el_per_particle_stats = StatsGatherer()


PRECISIONS = {"fp64": 0, "mixed": 1, "mixed_simt": 2}


class ShapeFunctionDepositor(Depositor):
    """rho[n] = sum_p q_p S(x_n - x_p), j = sum_p q_p v_p S (dep_shape.hpp).

    ``precision="fp64"`` is the plain form. ``"mixed"`` is the chosen form:
    on the tensor cores, the shape weights from a split-FP16 product rounded
    to 23-bit integers and summed exactly against charges scaled to integers
    below 2^46 (currents below 2^22), combined into FP64 per node; the
    normalising integral
    is summed exactly from the same weights, so the normalised depositor's
    deposited charge equals the particles' charge to FP64 rounding.
    ``"mixed_simt"`` evaluates the weights and sums them in FP32 per batch of
    32 particles on the CUDA cores, combining the batches into FP64."""

    name = "Shape"
    mode = _lib.DEPOSIT_PLAIN

    def __init__(self, precision="fp64"):
        Depositor.__init__(self)
        if precision not in PRECISIONS:
            raise ValueError("precision must be 'fp64', 'mixed' or 'mixed_simt'")
        self.precision = precision

    def set_shape_function(self, state, sf):
        Depositor.set_shape_function(self, state, sf)

    def _shape_desc(self):
        sf = self.shape_function
        return _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer)

    def deposit_densities_device(self, state, rho=True, j=True, precision=None):
        precision = PRECISIONS[precision or self.precision]
        self.deposit_hook()
        m = self.method
        r, jj = self._outputs(state)
        v = m.velocities_device(state) if j else None
        stats = _lib.DepositStats()
        iw = getattr(self, "integral_weights", None)
        _lib.check(self.lib.prt_deposit_shape(
            m.mesh_data.handle, m.workspace, self.mode, self._shape_desc(),
            _lib.ptr(iw) if iw is not None else None, len(state),
            state.x.data_ptr(), state.q.data_ptr(),
            v.data_ptr() if v is not None else None, state.el.data_ptr(),
            r.data_ptr() if rho else None, jj.data_ptr() if j else None, precision,
            C.byref(stats) if self.mode == _lib.DEPOSIT_NORMALIZED else None,
            self._stream()), "prt_deposit_shape")
        if self.mode == _lib.DEPOSIT_NORMALIZED:
            self._note_stats(state, stats)
        return r, jj

    def _note_stats(self, state, stats):
        pass


class NormalizedShapeFunctionDepositor(ShapeFunctionDepositor):
    """Deposits q_p S / (sum_e |J_e| sum_i w_i S_i) per particle so that each
    particle's deposited charge is exactly q_p (dep_normshape.hpp:125-199)."""

    name = "NormShape"
    mode = _lib.DEPOSIT_NORMALIZED

    def initialize(self, method):
        ShapeFunctionDepositor.initialize(self, method)
        ldis = method.discretization.element_groups[0].local_discretization
        # w = M 1 (dep_normshape.hpp:214-222)
        self.integral_weights = np.ascontiguousarray(ldis.mass_matrix().sum(axis=1))

    def make_state(self, state):
        return NormalizationStats()

    def _note_stats(self, state, s):
        ds = state.depositor_state
        if ds is None:
            return
        ds.normalization_stats.add_moments(s.norm_count, s.norm_sum, s.norm_sum_sq,
                                           s.norm_min, s.norm_max)
        ds.el_per_particle_stats.add_moments(s.el_count, s.el_sum, s.el_sum_sq, s.el_min,
                                             s.el_max)
        self.method.check_status()
