"""Particle files: checkpoints of the device store and VTK particle output
(the reference's cloud.py:606-671 visualisation, as files; Silo needs pylo,
which this package does not use).

* ``save_checkpoint`` / ``load_checkpoint``: the store's positions, momenta,
  charges, masses, containing elements (alive = element != invalid) and
  particle ids in a NumPy ``.npz`` file, in ascending id order, so a run can
  resume in another process.
* ``write_vtk`` / ``write_particles_vtk``: legacy-format VTK polydata
  (ASCII), one vertex per particle with point data (charge, mass, momentum,
  velocity and any per-particle visualisation vectors).
"""

from __future__ import annotations

import numpy as np

from . import _lib

CHECKPOINT_VERSION = 1


def save_checkpoint(state, path):
    el = state.containing_elements
    np.savez(path, version=CHECKPOINT_VERSION, positions=state.positions,
             momenta=state.momenta, charges=state.charges, masses=state.masses,
             elements=el, alive=el != _lib.INVALID_ELEMENT, ids=state.particle_ids,
             next_id=state.next_id)


def load_checkpoint(method, path):
    """A new PicState of `method` holding the checkpoint's particles (the
    removed ones dropped)."""
    import torch
    from .cloud import F64, PicState
    with np.load(path) as f:
        if int(f["version"]) != CHECKPOINT_VERSION:
            raise ValueError("unknown checkpoint version %d" % int(f["version"]))
        alive = f["alive"]
        ids = f["ids"][alive]
        dev = method.dev
        x = torch.as_tensor(np.ascontiguousarray(f["positions"][alive].T), dtype=F64,
                            device=dev).contiguous()
        p = torch.as_tensor(np.ascontiguousarray(f["momenta"][alive].T), dtype=F64,
                            device=dev).contiguous()
        q = torch.as_tensor(f["charges"][alive], dtype=F64, device=dev)
        m = torch.as_tensor(f["masses"][alive], dtype=F64, device=dev)
        el = torch.as_tensor(f["elements"][alive].view(np.int32), device=dev)
        tid = torch.as_tensor(ids, dtype=torch.int64, device=dev)
        state = PicState(method, x=x, p=p, q=q, m=m, el=el, ids=tid)
        state.next_id = max(int(f["next_id"]), state.next_id)
    state.particle_number_shift_signaller.subscribe_with_state(method.depositor)
    state.particle_number_shift_signaller.subscribe_with_state(method.pusher)
    state.particle_number_shift_signaller.note_change_size(len(state))
    return state


def write_vtk(path, positions, point_data=None, title="pyrticle_b200 particles"):
    """Legacy VTK polydata: `positions` [N, 3]; `point_data` name -> [N] or
    [N, 3] arrays."""
    x = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    n = len(x)
    lines = ["# vtk DataFile Version 3.0", title, "ASCII", "DATASET POLYDATA",
             "POINTS %d double" % n]
    lines += ["%.17g %.17g %.17g" % tuple(r) for r in x]
    lines.append("VERTICES %d %d" % (n, 2 * n))
    lines += ["1 %d" % i for i in range(n)]
    if point_data:
        lines.append("POINT_DATA %d" % n)
        for name, val in point_data.items():
            a = np.asarray(val, dtype=np.float64)
            if a.ndim == 1:
                lines += ["SCALARS %s double 1" % name, "LOOKUP_TABLE default"]
                lines += ["%.17g" % v for v in a]
            else:
                a = a.reshape(n, -1)
                if a.shape[1] != 3:
                    raise ValueError("point data %r: 1 or 3 components per particle" % name)
                lines.append("VECTORS %s double" % name)
                lines += ["%.17g %.17g %.17g" % tuple(r) for r in a]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_particles_vtk(method, state, path, vis_listener=None):
    """The reference's particle output (charge, mass, momentum, velocity and
    the visualisation listener's per-particle vectors), ascending id order."""
    data = {"charge": state.charges, "mass": state.masses, "momentum": state.momenta,
            "velocity": method.velocities(state)}
    if vis_listener is not None:
        for name, val in vis_listener.particle_vis_map.items():
            data[name] = val
    write_vtk(path, state.positions, data)


def read_vtk_points(path):
    """Positions and point data of a file written by write_vtk (for checks)."""
    with open(path) as fh:
        tok = fh.read().split("\n")
    i = tok.index(next(t for t in tok if t.startswith("POINTS")))
    n = int(tok[i].split()[1])
    pos = np.array([[float(v) for v in tok[i + 1 + k].split()] for k in range(n)])
    data = {}
    j = i + 1 + n
    while j < len(tok):
        t = tok[j].split()
        if t and t[0] == "SCALARS":
            data[t[1]] = np.array([float(tok[j + 2 + k]) for k in range(n)])
            j += 2 + n
        elif t and t[0] == "VECTORS":
            data[t[1]] = np.array([[float(v) for v in tok[j + 1 + k].split()] for k in range(n)])
            j += 1 + n
        else:
            j += 1
    return pos, data
