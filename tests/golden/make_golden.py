"""Regenerates the committed golden fixtures from the CPU oracle.

Run: ``python tests/golden/make_golden.py``. The fixture freezes the
oracle's output (element ids, counters, trajectories, rho, j) on a small
seeded config0 case so that the oracle itself, and the GPU path through the
parity tests, are checked against fixed numbers on any machine.
"""

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle as O  # noqa: E402
from pyrticle_b200 import meshgen, problems, refelement  # noqa: E402
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B  # noqa: E402
from pyrticle_b200.tools import PolynomialShapeFunction  # noqa: E402
from pyrticle_b200.units import SIUnitsWithNaturalConstants as U  # noqa: E402


def main():
    scale, steps = 0.05, 20
    w = problems.make("config0", scale=scale)
    om = O.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
    el0 = O.find_containing_elements(om, w.positions)
    ex = refelement.node_tuples(w.order)
    V = refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex)
    pu = O.OraclePusher(ex, V)
    c = U.VACUUM_LIGHT_SPEED()
    r = O.lsrk_steps(pu, om, w.positions, w.momenta, w.charges, w.masses, el0,
                     list(w.fields), LSRK4_A, LSRK4_B, w.dt, c, steps)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    v = O.velocities(r["p"], r["m"], c)
    rho, j, _, _ = O.deposit_shape(om, 0, sf, r["x"], r["q"], v, r["el"])
    ctr = r["counters"]
    np.savez_compressed(
        Path(__file__).parent / "config0_small.npz",
        scale=scale, steps=steps, x0=w.positions, el0=el0, x=r["x"], p=r["p"], el=r["el"],
        ids=r["ids"], rho=rho, j=j,
        counters=np.array([ctr.find_same, ctr.find_by_neighbor, ctr.find_by_vertex,
                           ctr.find_global], dtype=np.uint64))
    print("wrote config0_small.npz:", len(r["x"]), "particles,", steps, "steps")


if __name__ == "__main__":
    main()
