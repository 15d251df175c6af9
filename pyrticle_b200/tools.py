"""Shape functions, statistics and warnings (``tools.hpp``, ``tools.cpp``,
``pyrticle/tools.py`` of the reference)."""

from __future__ import annotations

import math
import warnings

import numpy as np


def sphere_area(dims: float) -> float:
    """Surface area of the unit sphere in ``dims`` dimensions (tools.cpp:35-38)."""
    return 2 * math.pi ** (dims / 2) / math.gamma(dims / 2)


def _beta(a: float, b: float) -> float:
    return math.exp(math.lgamma(a) + math.lgamma(b) - math.lgamma(a + b))


class PolynomialShapeFunction:
    """S(r) = N (a - r^2/a)^alpha for r <= a, else 0 (tools.hpp:514-556).

    The normaliser ``N = 2 / (|S^{n-1}| a^{n+alpha} B(n/2, alpha+1))``
    (tools.cpp:43-58) makes S integrate to one over R^n.
    """

    def __init__(self, radius: float = 1.0, dimensions: int = 1, alpha: float = 2.0):
        self.radius = float(radius)
        self.dimensions = int(dimensions)
        self.exponent = float(alpha)
        n = float(dimensions)
        self.normalizer = 2 / (sphere_area(n) * self.radius ** (n + alpha)
                               * _beta(n / 2, alpha + 1))

    @property
    def alpha(self) -> float:
        return self.exponent

    def __call__(self, r) -> float:
        r = np.asarray(r, dtype=np.float64)
        r2 = float(np.dot(r, r))
        if r2 > self.radius ** 2:
            return 0.0
        t = self.radius - r2 / self.radius
        return self.normalizer * t ** self.exponent

    def evaluate(self, r: np.ndarray) -> np.ndarray:
        """Vectorised over the last axis of ``r``."""
        r2 = np.sum(np.asarray(r) ** 2, axis=-1)
        t = np.maximum(self.radius - r2 / self.radius, 0.0)
        out = self.normalizer * t ** self.exponent
        out[r2 > self.radius ** 2] = 0.0
        return out

    @staticmethod
    def name() -> str:
        return "polynomial"


class CInfinityShapeFunction:
    """S(r) = N exp(-1 / (r^2/a^2 - 1)^2) for r <= a, else 0 (tools.hpp:561-591),
    with N = 1 / (|S^{n-1}| a^n I), I = int_0^1 s^(n-1) exp(-1/(1 - s^2)^2) ds
    by 50-point Gauss-Legendre on [0, 1] (tools.cpp:63-72, tools.py:268-283).
    Host evaluation only: the deposition kernels use the polynomial shape,
    as the reference's compiled depositors do."""

    def __init__(self, radius: float = 1.0, dimensions: int = 1):
        self.radius = float(radius)
        self.dimensions = int(dimensions)
        x, w = np.polynomial.legendre.leggauss(50)
        s = 0.5 * (x + 1)
        integral = float(0.5 * np.sum(w * s ** (dimensions - 1)
                                      * np.exp(-1 / (1 - s ** 2) ** 2)))
        self.normalizer = 1 / (sphere_area(float(dimensions)) * self.radius ** dimensions
                               * integral)

    def __call__(self, r) -> float:
        r = np.asarray(r, dtype=np.float64)
        r2 = float(np.dot(r, r))
        if r2 >= self.radius ** 2:  # exp(-1/0) = 0 at the radius itself
            return 0.0
        t = r2 / self.radius ** 2 - 1
        return self.normalizer * math.exp(-1 / (t * t))

    def evaluate(self, r: np.ndarray) -> np.ndarray:
        """Vectorised over the last axis of ``r``."""
        r2 = np.sum(np.asarray(r) ** 2, axis=-1)
        inside = r2 < self.radius ** 2
        t = np.where(inside, r2 / self.radius ** 2 - 1, -1.0)
        return np.where(inside, self.normalizer * np.exp(-1 / (t * t)), 0.0)

    @staticmethod
    def name() -> str:
        return "c_infinity"


class StatsGatherer:
    """Welford mean/variance with min and max (tools.hpp:340-417)."""

    def __init__(self):
        self.reset()

    def reset(self):
        self._count = 0
        self._mean = 0.0
        self._m2 = 0.0
        self._min = None
        self._max = None

    def add(self, x: float) -> None:
        x = float(x)
        if self._count == 0 or x < self._min:
            self._min = x
        if self._count == 0 or x > self._max:
            self._max = x
        self._count += 1
        delta = x - self._mean
        self._mean += delta / self._count
        self._m2 += delta * (x - self._mean)

    def add_moments(self, count, total, total_sq, lo, hi) -> None:
        """Merge a block summarised by count / sum / sum of squares / min / max."""
        count = int(count)
        if count == 0:
            return
        mean_b = total / count
        m2_b = max(total_sq - count * mean_b * mean_b, 0.0)
        n = self._count + count
        delta = mean_b - self._mean
        self._m2 += m2_b + delta * delta * self._count * count / n
        self._mean += delta * count / n
        self._min = lo if self._min is None else min(self._min, lo)
        self._max = hi if self._max is None else max(self._max, hi)
        self._count = n

    def count(self) -> int:
        return self._count

    def minimum(self):
        return self._min

    def maximum(self):
        return self._max

    def mean(self) -> float:
        if self._count == 0:
            raise RuntimeError("attempted to take empty mean")
        return self._mean

    def variance_sample(self) -> float:
        if self._count < 2:
            raise RuntimeError("sample too small for sample variance")
        return self._m2 / (self._count - 1)

    def standard_deviation_sample(self) -> float:
        return math.sqrt(self.variance_sample())

    def variance(self) -> float:
        if self._count == 0:
            raise RuntimeError("attempted to take empty variance")
        return self._m2 / self._count

    def standard_deviation(self) -> float:
        return math.sqrt(self.variance())


class WarningForwarder:
    """Routes core warnings to Python's ``warnings`` (pyrticle/tools.py:31-46)."""

    def note_warning(self, message, filename="libprt", lineno=0):
        warnings.warn_explicit(message, UserWarning, filename, lineno)


class WarningIgnorer:
    def note_warning(self, message, filename="libprt", lineno=0):
        pass


warning_forwarder = WarningForwarder()


# particle-number shifts -------------------------------------------------------
class NumberShiftMultiplexer:
    """Fans particle-number shifts out to its subscribers (the reference's
    tools.py:52-73): note_change_size(new_size), note_move(orig, dest, size)
    (particles [orig, orig + size) now live at [dest, dest + size)) and
    note_reset(start, size). Subscribers are held weakly."""

    def __init__(self, name=None):
        import weakref
        self.subscribers = weakref.WeakKeyDictionary()
        self.name = name

    def subscribe(self, subscriber):
        self.subscribers[subscriber] = None

    def note_change_size(self, new_size):
        for s in list(self.subscribers.keys()):
            s.note_change_size(new_size)

    def note_move(self, orig, dest, size):
        for s in list(self.subscribers.keys()):
            s.note_move(orig, dest, size)

    def note_reset(self, start, size):
        for s in list(self.subscribers.keys()):
            s.note_reset(start, size)


class StatePassingNumberShiftMultiplexer(NumberShiftMultiplexer):
    """Also notifies subscribers that take the particle state as their first
    argument (depositors and pushers; tools.py:78-103)."""

    def __init__(self, state):
        import weakref
        NumberShiftMultiplexer.__init__(self)
        self.subscribers_with_state = weakref.WeakKeyDictionary()
        self.state = state

    def subscribe_with_state(self, subscriber):
        self.subscribers_with_state[subscriber] = None

    def note_change_size(self, new_size):
        NumberShiftMultiplexer.note_change_size(self, new_size)
        for s in list(self.subscribers_with_state.keys()):
            s.note_change_size(self.state, new_size)

    def note_move(self, orig, dest, size):
        NumberShiftMultiplexer.note_move(self, orig, dest, size)
        for s in list(self.subscribers_with_state.keys()):
            s.note_move(self.state, orig, dest, size)

    def note_reset(self, start, size):
        NumberShiftMultiplexer.note_reset(self, start, size)
        for s in list(self.subscribers_with_state.keys()):
            s.note_reset(self.state, start, size)


def compaction_moves(alive):
    """The note_move calls that turn a store into its survivors, keeping their
    order: runs of surviving particles, (orig, dest, size) with dest <= orig,
    to be applied in the order given. `alive`: boolean sequence."""
    moves = []
    dest = 0
    i = 0
    n = len(alive)
    while i < n:
        if not alive[i]:
            i += 1
            continue
        j = i
        while j < n and alive[j]:
            j += 1
        if dest != i:
            moves.append((i, dest, j - i))
        dest += j - i
        i = j
    return moves


class NumberShiftableVector:
    """A per-particle host vector (rows = particle numbers) kept in step with
    the particle-number shifts of its signaller (tools.py:106-177), so that
    RK stage vectors survive particles being removed in mid-step. Adds and
    scales like its vector; `unwrap` returns the plain vector."""

    def __init__(self, vector, signaller):
        self.vector = vector
        self.signaller = signaller
        signaller.subscribe(self)

    @staticmethod
    def unwrap(instance):
        return instance.vector if isinstance(instance, NumberShiftableVector) else instance

    def __len__(self):
        return len(self.vector)

    def __add__(self, other):
        return NumberShiftableVector(self.vector + self.unwrap(other), self.signaller)

    __radd__ = __add__

    def __iadd__(self, other):
        self.vector += self.unwrap(other)
        return self

    def __mul__(self, other):
        return NumberShiftableVector(self.vector * self.unwrap(other), self.signaller)

    __rmul__ = __mul__

    def note_change_size(self, new_size):
        old = len(self.vector)
        if new_size > old:
            grown = np.zeros((new_size,) + tuple(self.vector.shape[1:]), dtype=self.vector.dtype)
            grown[:old] = self.vector
            self.vector = grown
        elif new_size < old:
            self.vector = self.vector[:new_size]

    def note_move(self, orig, dest, size):
        self.vector[dest:dest + size] = self.vector[orig:orig + size].copy()

    def note_reset(self, start, size):
        self.vector[start:start + size] = 0
