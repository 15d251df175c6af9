"""Seeded synthetic PIC workloads (meshes, particles, static nodal fields).

Five workloads, all in SI units (metres), as the reference works in SI
(``units.py:80-89``):

* ``config0`` -- 1x1x4 cm box, 8x8x32 cubes x 6 jittered tets, order 2,
  10,000 electrons in an r < 0.25 cm beam, uniform Bz = 0.1 T plus a linear
  focusing field E_r = -1e6 V/m^2 * r, shape radius 0.1 cm, 200 steps.
* ``config1`` -- 32x32x128 cubes, order 3, 4M electrons, static Bz plus 8
  seeded Fourier modes of E and B, 128x128x512 brick grid, 100 steps.
* ``config2`` -- config1's mesh and fields, 16M electrons, shape radius 0.08 cm.
* ``config3`` -- 16x16x64 cubes, order 3, 1M electrons, 100 steps, the
  focusing fields of config0 (gradients with respect to Bz and the focusing
  gradient are the differentiable set-up's parameters).
* ``config4`` -- 64x64x128 cubes, order 4, 64M electrons in a Gaussian bunch.

``scale`` shrinks the particle count (and, through ``cubes``, the mesh) for
tests; the physics set-up stays the same.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import meshgen, refelement
from .units import SIUnitsWithNaturalConstants as U

CM = 1e-2


@dataclasses.dataclass
class Workload:
    name: str
    mesh: meshgen.Mesh
    order: int
    positions: np.ndarray     # [N, 3]
    momenta: np.ndarray       # [N, 3]
    charges: np.ndarray       # [N]
    masses: np.ndarray        # [N]
    fields: np.ndarray        # [6, Nn]: ex, ey, ez, bx, by, bz at the nodes
    shape_radius: float
    dt: float
    steps: int
    brick_dims: tuple | None = None
    nodes: np.ndarray | None = None
    # fields = sum_k theta[k] * field_basis[k] where the workload defines a
    # basis (the differentiable set-ups): [K, 6, Nn] and [K]
    field_basis: np.ndarray | None = None
    theta: np.ndarray | None = None

    @property
    def particle_count(self) -> int:
        return len(self.positions)


def _beam(n, rng, radius, zlo, zhi, gamma, axis_xy, transverse_rel=1e-3):
    u = rng.random(n)
    th = rng.random(n) * 2 * math.pi
    r = radius * np.sqrt(u)
    x = np.empty((n, 3))
    x[:, 0] = axis_xy[0] + r * np.cos(th)
    x[:, 1] = axis_xy[1] + r * np.sin(th)
    x[:, 2] = rng.uniform(zlo, zhi, n)
    m = U.EL_MASS
    c = U.VACUUM_LIGHT_SPEED()
    beta = math.sqrt(1 - 1 / gamma ** 2)
    pz = gamma * m * c * beta
    p = np.zeros((n, 3))
    p[:, 2] = pz
    p[:, 0] = rng.normal(0, transverse_rel * pz, n)
    p[:, 1] = rng.normal(0, transverse_rel * pz, n)
    return x, p


def _bunch(n, rng, sigma_r, sigma_z, center, gamma, lo, hi, transverse_rel=1e-3):
    x = np.empty((n, 3))
    x[:, 0] = rng.normal(center[0], sigma_r, n)
    x[:, 1] = rng.normal(center[1], sigma_r, n)
    x[:, 2] = rng.normal(center[2], sigma_z, n)
    pad = 1e-3 * (hi - lo)
    np.clip(x, lo + pad, hi - pad, out=x)
    m = U.EL_MASS
    c = U.VACUUM_LIGHT_SPEED()
    beta = math.sqrt(1 - 1 / gamma ** 2)
    pz = gamma * m * c * beta
    p = np.zeros((n, 3))
    p[:, 2] = pz
    p[:, 0] = rng.normal(0, transverse_rel * pz, n)
    p[:, 1] = rng.normal(0, transverse_rel * pz, n)
    return x, p


def focusing_fields(nodes, axis_xy, bz=0.1, grad=1e6):
    """Uniform Bz and E_r = -grad * r about the beam axis, at the nodes."""
    f = np.zeros((6, len(nodes)))
    f[0] = -grad * (nodes[:, 0] - axis_xy[0])
    f[1] = -grad * (nodes[:, 1] - axis_xy[1])
    f[5] = bz
    return f


def focusing_basis(nodes, axis_xy):
    """Basis of the focusing set-up: unit uniform Bz, unit focusing gradient
    (``focusing_fields(bz, grad) = bz * basis[0] + grad * basis[1]``)."""
    return np.stack([focusing_fields(nodes, axis_xy, bz=1.0, grad=0.0),
                     focusing_fields(nodes, axis_xy, bz=0.0, grad=1.0)])


def fourier_fields(nodes, rng, bz=0.1, modes=8, amp=1e4, lam=(0.2 * CM, 2 * CM)):
    """Static Bz plus ``modes`` seeded plane-wave modes of E and of B.

    Each mode: amplitude N(0, amp) [V/m] (B modes carry amplitude/c tesla),
    wavelength U[lam], random unit direction k and random polarisation
    perpendicular to k, random phase.
    """
    c = U.VACUUM_LIGHT_SPEED()
    f = np.zeros((6, len(nodes)))
    f[5] = bz
    for which in (0, 1):
        for _ in range(modes):
            a = rng.normal(0, amp)
            wl = rng.uniform(*lam)
            k = rng.normal(size=3)
            k /= np.linalg.norm(k)
            pol = np.cross(k, rng.normal(size=3))
            pol /= np.linalg.norm(pol)
            ph = rng.uniform(0, 2 * math.pi)
            phase = 2 * math.pi / wl * (nodes @ k) + ph
            s = a * (1.0 if which == 0 else 1.0 / c)
            wave = s * np.cos(phase)
            for d in range(3):
                f[3 * which + d] += pol[d] * wave
    return f


def stable_dt(mesh, courant=0.3):
    return courant * float(mesh.inradii().min()) / U.VACUUM_LIGHT_SPEED()


def make(name: str, scale: float = 1.0, cubes=None, steps=None, seed=1,
         zslab=None) -> Workload:
    """Build a named workload; ``scale`` multiplies the particle count.

    ``zslab=(rank, world)`` (beam workloads): the rank's share of a beam of
    ``world`` times the particles, i.e. the particles of the world-times-larger
    beam whose z falls in the rank's slab of the beam's z range (the beam is
    uniform in z, so each slab holds the same count). Elements are numbered
    with z slowest, so this is the rank's contiguous block of the
    element-sorted global particle order."""
    lo = np.zeros(3)
    hi = np.array([1 * CM, 1 * CM, 4 * CM])
    axis_xy = (0.5 * CM, 0.5 * CM)
    if name == "config0":
        cubes = cubes or (8, 8, 32)
        order, n, a, nsteps = 2, 10_000, 0.1 * CM, 200
    elif name == "config1":
        cubes = cubes or (32, 32, 128)
        order, n, a, nsteps = 3, 4_000_000, 0.1 * CM, 100
    elif name == "config2":
        cubes = cubes or (32, 32, 128)
        order, n, a, nsteps = 3, 16_000_000, 0.08 * CM, 100
    elif name == "config3":
        cubes = cubes or (16, 16, 64)
        order, n, a, nsteps = 3, 1_000_000, 0.1 * CM, 100
    elif name == "config4":
        cubes = cubes or (64, 64, 128)
        order, n, a, nsteps = 4, 64_000_000, 0.05 * CM, 50
    else:
        raise ValueError(f"unknown workload {name!r}")
    n = max(1, int(round(n * scale)))
    mesh = meshgen.box_mesh(cubes, lo, hi, jitter=0.15, seed=0)
    nodes = meshgen.element_nodes(mesh, order)
    rng = np.random.default_rng(seed)
    if name == "config4":
        x, p = _bunch(n, rng, 0.1 * CM, 0.05 * CM, (0.5 * CM, 0.5 * CM, 2 * CM), 5.0,
                      lo, hi)
    else:
        zlo, zhi = 0.5 * CM, 3.5 * CM
        if zslab is not None:
            r, nr = zslab
            zlo, zhi = zlo + (zhi - zlo) * r / nr, zlo + (zhi - zlo) * (r + 1) / nr
        x, p = _beam(n, rng, 0.25 * CM, zlo, zhi, 2.0, axis_xy)
    basis = theta = None
    if name in ("config0", "config3"):
        basis = focusing_basis(nodes, axis_xy)
        theta = np.array([0.1, 1e6])
        fields = focusing_fields(nodes, axis_xy)
    else:
        fields = fourier_fields(nodes, np.random.default_rng(2))
    q = np.full(n, -U.EL_CHARGE)
    m = np.full(n, U.EL_MASS)
    brick = (128, 128, 512) if name in ("config1",) else None
    return Workload(name=name, mesh=mesh, order=order, positions=x, momenta=p,
                    charges=q, masses=m, fields=fields, shape_radius=a,
                    dt=stable_dt(mesh), steps=steps or nsteps, brick_dims=brick,
                    nodes=nodes, field_basis=basis, theta=theta)


def node_count(order: int) -> int:
    return refelement.node_count(order)
