"""FP64 PyTorch restatement of the differentiable particle step (test
infrastructure only).

The reference gradient for the hand-written adjoint kernels: the same
forward as libprt's stage and deposition kernels, written with plain torch
ops so that torch.autograd differentiates it independently. The containing
element of every stage is an input (taken from a recorded forward run); the
derivative holds it fixed, as the adjoint kernels do. Small cases only
(dense particle x node pairs for the deposition).
"""

import numpy as np
import torch

from pyrticle_b200 import refelement
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B

F64 = torch.float64


def lagrange_weights(order, dev):
    """W[i][j]: Lagrange value i = sum_j W[i][j] monomial_j (canonical order)."""
    ex = refelement.node_tuples(order)
    V = refelement.monomial_vandermonde(refelement.unit_nodes(order), ex)
    return torch.as_tensor(np.linalg.inv(V).T.copy(), dtype=F64, device=dev)


def monomials(r, order):
    """[n, Np] monomials r0^a r1^b r2^c, canonical order (a fastest)."""
    cols = [r[:, 0] ** a * r[:, 1] ** b * r[:, 2] ** c
            for (a, b, c) in refelement.node_tuples(order)]
    return torch.stack(cols, dim=1)


def velocity(p, m, c):
    """v = c p / sqrt(m^2 c^2 + |p|^2); p [3, n]."""
    s = torch.sqrt(m * m * c * c + (p * p).sum(0))
    return c * p / s


def stage(x, p, kx, kp, el, q, m, F, inv_maps, W, order, a, b, dt, c):
    """One low-storage RK stage; x, p, kx, kp [3, n]; el [n] long (>= 0)."""
    NP = W.shape[0]
    M = inv_maps[el]
    r = torch.einsum("nij,jn->ni", M[:, :9].reshape(-1, 3, 3), x) + M[:, 9:]
    ell = monomials(r, order) @ W.T                       # [n, NP]
    idx = el[:, None] * NP + torch.arange(NP, device=x.device)
    Fn = F[:, idx]                                        # [6, n, NP]
    EB = (Fn * ell[None]).sum(-1)                         # [6, n]
    v = velocity(p, m, c)
    force = q * (EB[:3] + torch.linalg.cross(v, EB[3:], dim=0))
    kx = a * kx + dt * v
    kp = a * kp + dt * force
    return x + b * kx, p + b * kp, kx, kp


def trajectory(x0, p0, F, q, m, elements, inv_maps, W, order, dt, c):
    """len(elements) stages from (x0, p0); elements[t] the stage-t elements."""
    x, p = x0, p0
    kx = torch.zeros_like(x0)
    kp = torch.zeros_like(p0)
    for t, el in enumerate(elements):
        a, b = LSRK4_A[t % 5], LSRK4_B[t % 5]
        x, p, kx, kp = stage(x, p, kx, kp, el, q, m, F, inv_maps, W, order, a, b, dt, c)
    return x, p


def deposit(x, p, q, m, c, nodes, radius, alpha, normalizer):
    """rho [Nn], j [3, Nn] of the plain shape depositor (no periodic images)."""
    v = velocity(p, m, c)
    rho = []
    j = []
    for k0 in range(0, nodes.shape[0], 4096):
        nd = nodes[k0:k0 + 4096]
        d2 = ((nd[:, None, :] - x.T[None, :, :]) ** 2).sum(-1)   # [chunk, n]
        t = torch.clamp(radius - d2 / radius, min=0.0) ** alpha * normalizer
        rho.append(t @ q)
        j.append((t @ (q * v).T).T)
    return torch.cat(rho), torch.cat(j, dim=1)
