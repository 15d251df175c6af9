"""Host-side set-up logic (no GPU): reference element, meshes, stats,
grid-depositor remap matrices, LSRK4 coefficients."""

import math

import numpy as np
import pytest

from pyrticle_b200 import meshgen, problems, refelement
from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
from pyrticle_b200.deposition.grid import (BrickInfo, basis_reduction_matrices,
                                           find_points_in_elements)
from pyrticle_b200.tools import StatsGatherer


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_nodes_edges_are_gauss_lobatto(order):
    n = refelement.unit_nodes(order)
    assert len(n) == refelement.node_count(order)
    e = np.sort(n[(np.abs(n[:, 1] + 1) < 1e-12) & (np.abs(n[:, 2] + 1) < 1e-12)][:, 0])
    assert np.allclose(e, refelement.gauss_lobatto_nodes(order), atol=1e-14)
    assert (n >= -1 - 1e-12).all() and (n.sum(axis=1) <= -1 + 1e-12).all()


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_orthonormal_mass_matrix_matches_exact_integrals(order):
    M = refelement.mass_matrix(order)
    w = refelement.integration_weights(order)
    assert np.allclose(M.sum(axis=1), w, atol=1e-13)
    assert w.sum() == pytest.approx(4 / 3, rel=1e-14)


def test_variance_like_the_reference():
    """test_pyrticle.py:13-35 (Welford variance with a 1e9 offset)."""
    for entire in (False, True):
        data = [4, 7, 13, 16]
        want = np.var(data, ddof=0 if entire else 1)
        for d in (data, [1e9 + x for x in data]):
            sg = StatsGatherer()
            for x in d:
                sg.add(x)
            got = sg.variance() if entire else sg.variance_sample()
            assert abs(got - want) < 1e-15 * max(1, want) * (1e9 if d[0] > 1e8 else 1)


def test_stats_merge_equals_sequential():
    rng = np.random.default_rng(0)
    x = rng.normal(size=1000)
    a, b = StatsGatherer(), StatsGatherer()
    for v in x:
        a.add(v)
    b.add_moments(len(x), x.sum(), (x * x).sum(), x.min(), x.max())
    assert b.mean() == pytest.approx(a.mean(), rel=1e-12)
    assert b.variance() == pytest.approx(a.variance(), rel=1e-10)


def test_lsrk4_is_fourth_order():
    """The 2N-storage scheme integrates y' = y to 4th order."""
    def run(nsteps):
        y, k, dt = 1.0, 0.0, 1.0 / nsteps
        for _ in range(nsteps):
            for a, b in zip(LSRK4_A, LSRK4_B):
                k = a * k + dt * y
                y = y + b * k
        return abs(y - math.e)
    e1, e2 = run(10), run(20)
    assert 14 < e1 / e2 < 18


def test_box_mesh_tables_consistent():
    m = meshgen.box_mesh((4, 3, 5), jitter=0.15, seed=4)
    assert m.jacobians.sum() * 4 / 3 == pytest.approx(0.01 * 0.01 * 0.04, rel=1e-12)
    for e in range(0, m.element_count, 7):
        for f in range(4):
            nb = m.face_neighbors[e, f]
            if nb == meshgen.INVALID_ELEMENT:
                continue
            g = list(m.face_neighbors[nb]).index(e)
            assert np.allclose(m.face_normals[e, f], -m.face_normals[nb, g])
    # inverse maps take vertices to the reference vertices
    p = m.points[m.elements[0]]
    A = m.inverse_maps[0, :9].reshape(3, 3)
    ref = (A @ p.T).T + m.inverse_maps[0, 9:]
    assert np.allclose(ref, [[-1, -1, -1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], atol=1e-12)


def test_grid_remap_reproduces_kept_polynomials():
    """I_e (w f(grid)) = f(nodes) for f in the span of the kept modes (grid.py:217-273)."""
    mesh = meshgen.box_mesh((3, 3, 6), jitter=0.1, seed=2)
    order = 2
    brk = BrickInfo(0, 0, np.array([0.01, 0.01, 0.04]) / [12, 12, 48], [0, 0, 0], [12, 12, 48])
    starts, gidx, pts, w = find_points_in_elements(mesh, [brk], 0.12)
    mats, mstarts, kept = basis_reduction_matrices(mesh, order, starts, pts, w)
    nodes = meshgen.element_nodes(mesh, order).reshape(mesh.element_count, -1, 3)
    Np = refelement.node_count(order)
    for e in range(0, mesh.element_count, 5):
        P = starts[e + 1] - starts[e]
        I = mats[mstarts[e]:mstarts[e + 1]].reshape(Np, P, order="F")
        # constants are always kept
        f = np.ones(P)
        assert np.allclose(I @ (w[starts[e]:starts[e + 1]] * f), np.ones(Np), atol=1e-10)
        assert 1 <= kept[e] <= min(Np, P)


def test_workload_generators_are_seeded():
    a = problems.make("config0", scale=0.01)
    b = problems.make("config0", scale=0.01)
    assert np.array_equal(a.positions, b.positions) and np.array_equal(a.fields, b.fields)
    r = np.hypot(a.positions[:, 0] - 0.005, a.positions[:, 1] - 0.005)
    assert r.max() < 0.0025


def test_number_shift_multiplexers():
    """Fan-out of particle-number shifts (tools.py:52-103 of the reference)
    and the moves of an order-keeping compaction."""
    from pyrticle_b200.tools import (NumberShiftMultiplexer, StatePassingNumberShiftMultiplexer,
                                     compaction_moves)

    class Rec:
        def __init__(self):
            self.calls = []

        def note_change_size(self, *a):
            self.calls.append(("size",) + a)

        def note_move(self, *a):
            self.calls.append(("move",) + a)

        def note_reset(self, *a):
            self.calls.append(("reset",) + a)

    state = object()
    sig = StatePassingNumberShiftMultiplexer(state)
    plain, with_state = Rec(), Rec()
    sig.subscribe(plain)
    sig.subscribe_with_state(with_state)
    sig.note_move(5, 2, 3)
    sig.note_change_size(7)
    sig.note_reset(0, 4)
    assert plain.calls == [("move", 5, 2, 3), ("size", 7), ("reset", 0, 4)]
    assert with_state.calls == [("move", state, 5, 2, 3), ("size", state, 7),
                                ("reset", state, 0, 4)]
    m = NumberShiftMultiplexer()
    r = Rec()
    m.subscribe(r)
    del r  # held weakly
    m.note_change_size(3)
    assert len(m.subscribers) == 0

    rng = np.random.default_rng(4)
    for n in (0, 1, 7, 100):
        alive = rng.random(n) < 0.6
        vals = list(range(n))
        for orig, dest, size in compaction_moves(alive.tolist()):
            assert dest <= orig
            vals[dest:dest + size] = vals[orig:orig + size]
        kept = int(alive.sum())
        assert vals[:kept] == [i for i in range(n) if alive[i]]


def test_number_shiftable_vector():
    """RK stage vectors follow particle removals (tools.py:106-177)."""
    from pyrticle_b200.tools import NumberShiftableVector, StatePassingNumberShiftMultiplexer
    sig = StatePassingNumberShiftMultiplexer(object())
    v = NumberShiftableVector(np.arange(12.0).reshape(6, 2), sig)
    w = 2 * v + v
    assert isinstance(w, NumberShiftableVector)
    assert np.array_equal(w.vector, 3 * np.arange(12.0).reshape(6, 2))
    # particles 1 and 4 removed: runs [2, 4) -> 1, [5, 6) -> 3
    sig.note_move(2, 1, 2)
    sig.note_move(5, 3, 1)
    sig.note_change_size(4)
    keep = [0, 2, 3, 5]
    assert np.array_equal(v.vector, np.arange(12.0).reshape(6, 2)[keep])
    assert np.array_equal(w.vector, 3 * np.arange(12.0).reshape(6, 2)[keep])
    sig.note_change_size(5)
    assert np.array_equal(v.vector[4], [0, 0])
    assert NumberShiftableVector.unwrap(v) is v.vector and NumberShiftableVector.unwrap(3) == 3


def test_derived_quantities_cache():
    """get_derived_quantities_from_cache (cloud.py:141-154) without the
    reference's always-true count: all cached, none cached (one joint
    computation), some cached (the missing ones alone)."""
    from pyrticle_b200.cloud import PicState

    class S:
        def __init__(self):
            self.derived_quantity_cache = {}

    s = S()
    calls = []

    def g(name, val):
        def f():
            calls.append(name)
            s.derived_quantity_cache[name] = val
            return val
        return f

    get = PicState.get_derived_quantities_from_cache
    names = ("a", "b")
    r = get(s, names, (g("a", 1), g("b", 2)), all_getter=lambda: (calls.append("all") or (1, 2)))
    assert r == (1, 2) and calls == ["all"] and s.derived_quantity_cache == {"a": 1, "b": 2}
    del s.derived_quantity_cache["b"]
    calls.clear()
    assert get(s, names, (g("a", 1), g("b", 2)), all_getter=None) == (1, 2)
    assert calls == ["b"]
    calls.clear()
    assert get(s, names, (g("a", 1), g("b", 2))) == (1, 2) and calls == []


def test_find_counter_log_quantity():
    from pyrticle_b200.log import FindCounter

    class M:
        find_same_counter = 5

    m = M()
    q = FindCounter(m, "find_same_counter", "n_find_same", "d")
    m.find_same_counter = 12
    assert q() == 7
    assert q() == 0


def test_continuity_groups():
    """average_groups (grid.py:143-183): on a non-periodic mesh every group
    is a set of coincident nodes, and every node shared by two elements is in
    one; on a z-periodic mesh the groups also join the nodes of the two
    periodic faces."""
    from pyrticle_b200 import meshgen
    from pyrticle_b200.deposition.grid import average_groups
    for periodic in ((False, False, False), (False, False, True)):
        mesh = meshgen.box_mesh((3, 3, 4), (0, 0, 0), (0.01, 0.01, 0.02), periodic=periodic)
        nodes = meshgen.element_nodes(mesh, 2)
        starts, members = average_groups(mesh, nodes, 10)
        assert np.all(np.diff(starts.astype(np.int64)) >= 2)
        assert len(np.unique(members)) == len(members)
        key = np.round(nodes / 1e-9).astype(np.int64)
        _, inv, counts = np.unique(key, axis=0, return_inverse=True, return_counts=True)
        shared = counts[inv.ravel()] >= 2
        grouped = np.zeros(len(nodes), dtype=bool)
        grouped[members] = True
        assert np.array_equal(grouped[shared], np.ones(shared.sum(), dtype=bool))
        z = nodes[:, 2]
        for g in range(len(starts) - 1):
            mem = members[starts[g]:starts[g + 1]]
            assert np.all(np.diff(mem.astype(np.int64)) > 0)      # ascending
            p = nodes[mem]
            if periodic[2]:
                p = p.copy()
                p[:, 2] = np.where(np.isclose(p[:, 2], 0.02), 0.0, p[:, 2])
            assert np.ptp(p, axis=0).max() < 1e-12
        if periodic[2]:
            joined = sum(1 for g in range(len(starts) - 1)
                         if np.isclose(z[members[starts[g]:starts[g + 1]]], 0.0).any()
                         and np.isclose(z[members[starts[g]:starts[g + 1]]], 0.02).any())
            assert joined > 0  # groups span the periodic seam
