"""CPU restatement of the averaging pusher's forces (test infrastructure
only): push_average.hpp:26-420 driven by the shape depositor's element walk
(dep_shape.hpp:128-149, element_finder.hpp:203-294), on a non-periodic mesh.

For each particle, the elements the face walk reaches; for each of their
nodes rho_i = q S(x_i - x_p) (zero beyond the radius); the E and B
averaging targets accumulate |J_e| w_i rho_i F_i and |J_e| w_i rho_i; the
forces are scale * qE_acc and scale * (v x qB_acc) with scale = q / (the
reconstructed charge)."""

import numpy as np

from oracle import pyoracle as O


def average_forces(om, shape, integral_weights, x, q, v, el, fields):
    """fields: [6, Nn]; returns (forces [n, 3], pt_e [n, 3], pt_b [n, 3])."""
    mesh = om.mesh
    np_ = om.np
    nodes = om.nodes
    a = shape.radius
    n = len(x)
    forces = np.zeros((n, 3))
    pt_e = np.zeros((n, 3))
    pt_b = np.zeros((n, 3))
    for p in range(n):
        qe = np.zeros(3)
        qb = np.zeros(3)
        charge = 0.0
        for e in O.walk_elements(om, x[p], int(el[p]), a):
            jac = mesh.jacobians[e]
            sl = slice(e * np_, (e + 1) * np_)
            r2 = ((nodes[sl] - x[p]) ** 2).sum(axis=1)
            rt = np.where(r2 <= a * a, a - r2 / a, 0.0)
            rho = q[p] * shape.normalizer * rt ** shape.exponent
            wr = rho * integral_weights
            qe += jac * (fields[0:3, sl] @ wr)
            qb += jac * (fields[3:6, sl] @ wr)
            charge += jac * wr.sum()
        if charge == 0:
            continue
        scale = q[p] / charge
        pt_e[p] = qe / charge
        pt_b[p] = qb / charge
        forces[p] = scale * qe + scale * np.cross(v[p], qb)
    return forces, pt_e, pt_b
