"""Beam diagnostics of the device particle store (the reference's
``_internal.kinetic_energies``, ``total_charge``, ``particle_momentum``,
``rms_beam_size``, ``rms_beam_emittance``, ``rms_energy_spread``,
``particle_current``; diagnostics.hpp:38-180).

One fused libprt reduction (``prt_beam_moments``) yields all the sums; each
function applies the reference's formula to them. Removed particles
(element PRT_INVALID_ELEMENT, not yet compacted) are excluded, as the
reference has already dropped them from its store.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from .cloud import stream_handle

BM = _lib.BM


def _csqrt(v):
    """C's sqrt: NaN for a negative argument (a rounding-level negative
    variance of a degenerate beam gives NaN, as in the reference)."""
    return math.sqrt(v) if v >= 0 else float("nan")


def beam_moments(state, vacuum_c, beam_axis=2, ke_shift=0.0) -> np.ndarray:
    """The PRT_BEAM_MOMENTS sums of prt_beam_moments (host array)."""
    m = state.method
    out = np.zeros(_lib.BEAM_MOMENTS)
    n = len(state)
    _lib.check(m.lib.prt_beam_moments(
        m.workspace, n, state.x.data_ptr() if n else None, state.p.data_ptr() if n else None,
        state.q.data_ptr() if n else None, state.m.data_ptr() if n else None,
        state.el.data_ptr() if n else None, float(vacuum_c), int(beam_axis), float(ke_shift),
        _lib.ptr(out), C.c_void_p(stream_handle())), "prt_beam_moments")
    return out


def kinetic_energies_device(state, vacuum_c) -> torch.Tensor:
    n = len(state)
    out = torch.zeros((n,), dtype=torch.float64, device=state.x.device)
    if n:
        _lib.check(state.method.lib.prt_kinetic_energies(
            n, state.p.data_ptr(), state.m.data_ptr(), state.el.data_ptr(), float(vacuum_c),
            out.data_ptr(), C.c_void_p(stream_handle())), "prt_kinetic_energies")
    return out


def kinetic_energies(state, vacuum_c) -> np.ndarray:
    """Per particle (gamma - 1) m c^2, ascending particle-id order."""
    return kinetic_energies_device(state, vacuum_c)[state.id_order()].cpu().numpy()


def total_charge(state) -> float:
    return float(beam_moments(state, 1.0)[BM["charge"]])


def particle_momentum(state) -> np.ndarray:
    return beam_moments(state, 1.0)[BM["p"]:BM["p"] + 3].copy()


def rms_beam_size(state, axis) -> float:
    s = beam_moments(state, 1.0)
    n = s[BM["count"]]
    return 0.0 if n == 0 else math.sqrt(s[BM["x2"] + axis] / n)


def rms_beam_emittance(state, axis, beam_axis) -> float:
    s = beam_moments(state, 1.0, beam_axis)
    n = s[BM["count"]]
    if n == 0:
        return 0.0
    mx = s[BM["x"] + axis] / n
    mxp = s[BM["xp"] + axis] / n
    mx2 = s[BM["x2"] + axis] / n
    mxp2 = s[BM["xp2"] + axis] / n
    mxxp = s[BM["xxp"] + axis] / n
    # diagnostics.hpp:120-130, term for term
    return _csqrt(mx2 * mxp2 - mx ** 2 * mxp2 - mx2 * mxp ** 2
                  - (mxxp ** 2 - 2 * mxxp * mx * mxp))


def rms_energy_spread(state, vacuum_c) -> float:
    """Standard deviation of the kinetic energies (tools.hpp:303-322). The
    squares are summed about the mean from a first pass, so the result keeps
    its digits where the reference's <KE^2> - <KE>^2 cancels (a gamma = 2
    beam with a 1e-3 momentum spread loses ~12 digits that way)."""
    s = beam_moments(state, vacuum_c)
    n = s[BM["count"]]
    if n == 0:
        return 0.0
    mean = s[BM["ke"]] / n
    s2 = beam_moments(state, vacuum_c, ke_shift=mean)
    return _csqrt(s2[BM["ke2"]] / n - (s2[BM["ke"]] / n - mean) ** 2)


def particle_current(state, velocities, length, vacuum_c=None) -> np.ndarray:
    """sum_p q_p v_p / length. The velocities are the state's own
    (PicMethod.velocities(state), as the reference's only caller passes), so
    they are formed on the device from the momenta; `velocities` is accepted
    for the reference's signature."""
    c = vacuum_c if vacuum_c is not None else state.method.units.VACUUM_LIGHT_SPEED()
    s = beam_moments(state, c)
    return s[BM["qv"]:BM["qv"] + 3] / length
