"""PIC method and particle state (the reference's ``pyrticle/cloud.py``).

``PicMethod`` keeps the reference's constructor and method names
(cloud.py:316-603): ``make_state``, ``add_particles``, ``velocities``,
``deposit_rho``, ``deposit_j``, ``deposit_densities``, ``advance_state``,
``upkeep``, plus the find-path counters. The particle store lives on the GPU
(torch tensors used only as device buffers); every computation goes through
libprt's C ABI. Host-facing accessors return numpy arrays in ascending
particle-id order, so results do not depend on the device store's internal
(element-sorted) order.

``PicMethod.step`` is the device-resident fast path: whole low-storage RK
steps (5 fused stages each) followed by one rho/j deposition, without host
round trips.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .meshdata import MeshData
from .tools import (NumberShiftableVector, StatePassingNumberShiftMultiplexer,
                    compaction_moves)

# Carpenter & Kennedy (1994), 5-stage 4th-order 2N-storage Runge-Kutta: the
# LSRK4 stepper the reference drives its particles with (driver.py:53,108).
LSRK4_A = (0.0,
           -567301805773.0 / 1357537059087.0,
           -2404267990393.0 / 2016746695238.0,
           -3550918686646.0 / 2091501179385.0,
           -1275806237668.0 / 842570457699.0)
LSRK4_B = (1432997174477.0 / 9575080441755.0,
           5161836677717.0 / 13612068292357.0,
           1720146321549.0 / 2090206949498.0,
           3134564353537.0 / 4481467310338.0,
           2277821191437.0 / 14882151754819.0)
LSRK4_C = (0.0,
           1432997174477.0 / 9575080441755.0,
           2526269341429.0 / 6820363962896.0,
           2006345519317.0 / 3224310063776.0,
           2802321613138.0 / 2924317926251.0)

F64 = torch.float64


def device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("pyrticle_b200 needs a CUDA device (sm_100a); none is available")
    return torch.device("cuda", torch.cuda.current_device())


def stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def to_store(arr, order_ids, dev) -> torch.Tensor:
    """Host [n, 3] (id order) -> device [3, n] (store order)."""
    a = torch.as_tensor(np.ascontiguousarray(arr, dtype=np.float64), device=dev)
    return a[order_ids].T.contiguous()


class MapStorageVisualizationListener:
    """Keeps the per-particle visualisation vectors (cloud.py:86-92)."""

    def __init__(self):
        self.mesh_vis_map = {}
        self.particle_vis_map = {}

    def store_particle_vis_vector(self, name, vec):
        self.particle_vis_map[name] = vec

    def store_mesh_vis_vector(self, name, vec):
        self.mesh_vis_map[name] = vec

    def clear(self):
        self.mesh_vis_map.clear()
        self.particle_vis_map.clear()


class ParticleStateView:
    """Host view with the attribute names of the reference's ParticleState3d3v."""

    xdim = 3
    vdim = 3

    def __init__(self, state: "PicState"):
        self._state = state

    @property
    def particle_count(self) -> int:
        return len(self._state)

    @property
    def positions(self):
        return self._state.positions

    @property
    def momenta(self):
        return self._state.momenta

    @property
    def charges(self):
        return self._state.charges

    @property
    def masses(self):
        return self._state.masses

    @property
    def containing_elements(self):
        return self._state.containing_elements


class PicState:
    """Device particle store: x, p [3, n]; q, m [n]; elements [n] (uint32 bit
    pattern in int32, PRT_INVALID_ELEMENT = -1 marks a removed particle);
    stable ids [n]; LSRK residuals kx, kp [3, n]."""

    def __init__(self, method, x=None, p=None, q=None, m=None, el=None, ids=None,
                 depositor_state=None, pusher_state=None, vis_listener=None, pnss=None):
        self.method = method
        # particle numbers are ranks in ascending id order (the host views'
        # order); kills shift them (cloud.py:75-84)
        self.particle_number_shift_signaller = (
            StatePassingNumberShiftMultiplexer(self) if pnss is None else pnss)
        dev = device()
        if x is None:
            x = torch.empty((3, 0), dtype=F64, device=dev)
            p = torch.empty((3, 0), dtype=F64, device=dev)
            q = torch.empty((0,), dtype=F64, device=dev)
            m = torch.empty((0,), dtype=F64, device=dev)
            el = torch.empty((0,), dtype=torch.int32, device=dev)
            ids = torch.empty((0,), dtype=torch.int64, device=dev)
        self.x, self.p, self.q, self.m, self.el, self.ids = x, p, q, m, el, ids
        self.kx = None
        self.kp = None
        self.next_id = int(ids.max().item()) + 1 if ids.numel() else 0
        self.derived_quantity_cache = {}
        self.depositor_state = (method.depositor.make_state(self)
                                if depositor_state is None else depositor_state)
        self.pusher_state = (method.pusher.make_state(self)
                             if pusher_state is None else pusher_state)
        self.vis_listener = vis_listener or MapStorageVisualizationListener()
        self.particle_state = ParticleStateView(self)

    def __len__(self) -> int:
        return int(self.x.shape[1])

    # --- host views, ascending id order ----------------------------------
    def id_order(self) -> torch.Tensor:
        return torch.argsort(self.ids)

    def _host3(self, t) -> np.ndarray:
        return t[:, self.id_order()].T.contiguous().cpu().numpy()

    @property
    def positions(self) -> np.ndarray:
        return self._host3(self.x)

    @property
    def momenta(self) -> np.ndarray:
        return self._host3(self.p)

    @property
    def charges(self) -> np.ndarray:
        return self.q[self.id_order()].cpu().numpy()

    @property
    def masses(self) -> np.ndarray:
        return self.m[self.id_order()].cpu().numpy()

    @property
    def containing_elements(self) -> np.ndarray:
        return self.el[self.id_order()].cpu().numpy().view(np.uint32)

    @property
    def particle_ids(self) -> np.ndarray:
        return self.ids[self.id_order()].cpu().numpy()

    def residuals(self):
        if self.kx is None or self.kx.shape != self.x.shape:
            self.kx = torch.zeros_like(self.x)
            self.kp = torch.zeros_like(self.p)
        return self.kx, self.kp

    def clear(self):
        self.__init__(self.method, depositor_state=self.depositor_state,
                      pusher_state=self.pusher_state, vis_listener=self.vis_listener,
                      pnss=self.particle_number_shift_signaller)
        self.derived_quantity_cache.clear()
        self.particle_number_shift_signaller.note_change_size(0)

    def resize(self, newsize):
        """Capacity hint (cloud.py:114-124): the device store grows as particles
        are added, so only a size below the particle count is an error."""
        if newsize < len(self):
            raise ValueError("cannot resize below the particle count (%d)" % len(self))

    # --- derived quantity cache (cloud.py:133-154) -------------------------
    def get_derived_quantity_from_cache(self, name, getter):
        try:
            return self.derived_quantity_cache[name]
        except KeyError:
            self.derived_quantity_cache[name] = value = getter()
            return value

    def get_derived_quantities_from_cache(self, names, getters, all_getter=None):
        """Cached values of several quantities; `all_getter` computes all of
        them at once when none is cached, else each missing one comes from its
        getter (which stores it)."""
        cached = tuple(self.derived_quantity_cache.get(name) for name in names)
        cached_number = sum(1 for v in cached if v is not None)
        if cached_number == len(names):
            return cached
        if cached_number == 0 and all_getter is not None:
            values = all_getter()
            for name, value in zip(names, values):
                self.derived_quantity_cache[name] = value
            return tuple(values)
        return tuple(c if c is not None else g() for c, g in zip(cached, getters))


class PicMethod:
    """Particle side of a PIC method on one GPU.

    @arg debug: set of strings; ``verbose_vis`` stores pt_e, pt_b, el_force
      and mag_force per particle in ``state.vis_listener`` (cloud.py:317-333).
    """

    def __init__(self, discr, units, depositor, pusher, dimensions_pos,
                 dimensions_velocity, debug=frozenset()):
        if (dimensions_pos, dimensions_velocity) != (3, 3):
            raise ValueError("only the 3d3v particle state is supported")
        self.units = units
        self.discretization = discr
        self.debug = set(debug)
        self.depositor = depositor
        self.pusher = pusher
        self.dimensions_mesh = discr.dimensions
        self.dimensions_pos = dimensions_pos
        self.dimensions_velocity = dimensions_velocity
        self.lib = _lib.load()
        self.dev = device()
        self.mesh_data = MeshData(discr.dimensions)
        self.mesh_data.fill_from_hedge(discr)
        ws = C.c_void_p()
        _lib.check(self.lib.prt_workspace_create(C.byref(ws)), "prt_workspace_create")
        self.workspace = ws
        self.depositor.initialize(self)
        self.pusher.initialize(self)
        self.find_same_counter = 0
        self.find_by_neighbor_counter = 0
        self.find_by_vertex_counter = 0
        self.find_global_counter = 0

    def __del__(self):
        if getattr(self, "workspace", None) is not None and _lib._lib is not None:
            _lib._lib.prt_workspace_destroy(self.workspace)
            self.workspace = None

    def get_dimensionality_suffix(self) -> str:
        return "%dd%dv" % (self.dimensions_pos, self.dimensions_velocity)

    def get_shape_function_class(self):
        """The shape function the deposition kernels evaluate (cloud.py:391-404):
        the polynomial one."""
        from .tools import PolynomialShapeFunction
        return PolynomialShapeFunction

    def set_ignore_core_warnings(self, ignore):
        """Forward (False) or drop (True) the library's warnings (cloud.py:406-413)."""
        from . import tools
        tools.warning_forwarder = tools.WarningIgnorer() if ignore else tools.WarningForwarder()

    def add_instrumentation(self, mgr, observer):
        """Log quantities of the element finder and of the depositor and pusher
        (cloud.py:415-423): the four find counters, as events per tick."""
        from .log import FindCounter
        for attr, name, desc in (
                ("find_same_counter", "n_find_same", "#Particles found in same element"),
                ("find_by_neighbor_counter", "n_find_neighbor",
                 "#Particles found through neighbor"),
                ("find_by_vertex_counter", "n_find_by_vertex",
                 "#Particles found by vertex"),
                ("find_global_counter", "n_find_global", "#Particles found by global search")):
            mgr.add_quantity(FindCounter(self, attr, name, desc))
        for part in (self.depositor, self.pusher):
            if hasattr(part, "add_instrumentation"):
                part.add_instrumentation(mgr, observer)

    def make_state(self) -> PicState:
        state = PicState(self)
        state.particle_number_shift_signaller.subscribe_with_state(self.depositor)
        state.particle_number_shift_signaller.subscribe_with_state(self.pusher)
        return state

    # --- status ------------------------------------------------------------
    def check_status(self, clear=True):
        """Raise on a device error recorded since the last check; forward
        warnings (the reference's WARN -> warnings.warn path)."""
        err = C.c_int32()
        eidx = C.c_int64()
        warn = C.c_int32()
        widx = C.c_int64()
        _lib.check(self.lib.prt_workspace_status(self.workspace, C.c_void_p(stream_handle()),
                                                 C.byref(err), C.byref(eidx), C.byref(warn),
                                                 C.byref(widx), int(clear)))
        if warn.value == _lib.PRT_WARN_ZERO_MASS:
            from .tools import warning_forwarder
            warning_forwarder.note_warning(
                "deposited particle mass is zero (particle %d)" % widx.value)
        elif warn.value == _lib.PRT_WARN_ZERO_AVERAGE:
            from .tools import warning_forwarder
            warning_forwarder.note_warning(
                "average pusher: particle %d had zero reconstructed charge" % widx.value)
        if err.value:
            raise RuntimeError("%s (particle %d)" % (_lib.ERRORS.get(err.value, err.value),
                                                     eidx.value))

    def transfer_find_counters(self):
        ctr = _lib.FindCounters()
        _lib.check(self.lib.prt_workspace_counters(self.workspace, C.c_void_p(stream_handle()),
                                                   C.byref(ctr), 1))
        self.find_same_counter += ctr.find_same
        self.find_by_neighbor_counter += ctr.find_by_neighbor
        self.find_by_vertex_counter += ctr.find_by_vertex
        self.find_global_counter += ctr.find_global
        return ctr

    # --- particles -------------------------------------------------------------
    def find_containing_elements_device(self, x: torch.Tensor) -> torch.Tensor:
        n = x.shape[1]
        el = torch.empty((n,), dtype=torch.int32, device=self.dev)
        _lib.check(self.lib.prt_find_containing_elements(
            self.mesh_data.handle, n, x.data_ptr(), el.data_ptr(),
            C.c_void_p(stream_handle())), "prt_find_containing_elements")
        return el

    def add_particles(self, state, iterable, maxcount=None):
        """Add particles from tuples (position, velocity, charge, mass)
        (cloud.py:441-490); particles outside the mesh are skipped."""
        pos, vel, ch, ms = [], [], [], []
        for item in iterable:
            if maxcount is not None:
                if maxcount == 0:
                    break
                maxcount -= 1
            x, v, q, m = item
            assert len(x) == self.dimensions_pos
            assert len(v) == self.dimensions_velocity
            pos.append(np.asarray(x, dtype=np.float64))
            vel.append(np.asarray(v, dtype=np.float64))
            ch.append(float(q))
            ms.append(float(m))
        if not pos:
            return
        vel = np.array(vel)
        ms = np.array(ms)
        gamma = np.array([self.units.gamma_from_v(v) for v in vel])
        mom = (ms * gamma)[:, None] * vel
        self.add_particles_from_arrays(state, np.array(pos), mom, np.array(ch), ms)

    def add_particles_from_arrays(self, state, positions, momenta, charges, masses):
        """Vectorised add: host or device arrays, positions/momenta [n, 3]."""
        dev = self.dev
        x = torch.as_tensor(np.ascontiguousarray(positions), dtype=F64, device=dev).T.contiguous()
        p = torch.as_tensor(np.ascontiguousarray(momenta), dtype=F64, device=dev).T.contiguous()
        q = torch.as_tensor(np.ascontiguousarray(charges), dtype=F64, device=dev).contiguous()
        m = torch.as_tensor(np.ascontiguousarray(masses), dtype=F64, device=dev).contiguous()
        el = self.find_containing_elements_device(x)
        ok = el != -1
        nbad = int((~ok).sum().item())
        if nbad:
            print("%d particles not in a valid element" % nbad)
            x, p, q, m, el = x[:, ok].contiguous(), p[:, ok].contiguous(), q[ok], m[ok], el[ok]
        n = x.shape[1]
        ids = torch.arange(state.next_id, state.next_id + n, dtype=torch.int64, device=dev)
        state.next_id += n
        state.x = torch.cat([state.x, x], dim=1).contiguous()
        state.p = torch.cat([state.p, p], dim=1).contiguous()
        state.q = torch.cat([state.q, q]).contiguous()
        state.m = torch.cat([state.m, m]).contiguous()
        state.el = torch.cat([state.el, el]).contiguous()
        state.ids = torch.cat([state.ids, ids]).contiguous()
        state.kx = state.kp = None
        self.check_containment(state)
        state.particle_number_shift_signaller.note_change_size(len(state))
        state.derived_quantity_cache.clear()

    def check_containment(self, state):
        assert bool((state.el != -1).all().item())

    def upkeep(self, state):
        self.depositor.upkeep(state)
        self.pusher.upkeep(state)
        state.vis_listener.clear()

    def compact(self, state) -> int:
        """Drop removed particles (element PRT_INVALID_ELEMENT), keeping the
        survivors' relative order; returns how many were dropped."""
        alive = state.el != -1
        dead = int((~alive).sum().item())
        if dead:
            # the shifts of the particle numbers (ranks in id order)
            order = state.id_order()
            moves = compaction_moves(alive[order].cpu().numpy().tolist())
            state.x = state.x[:, alive].contiguous()
            state.p = state.p[:, alive].contiguous()
            state.q = state.q[alive].contiguous()
            state.m = state.m[alive].contiguous()
            state.el = state.el[alive].contiguous()
            state.ids = state.ids[alive].contiguous()
            if state.kx is not None:
                state.kx = state.kx[:, alive].contiguous()
                state.kp = state.kp[:, alive].contiguous()
            state.derived_quantity_cache.clear()
            sig = state.particle_number_shift_signaller
            for orig, dest, size in moves:
                sig.note_move(orig, dest, size)
            sig.note_change_size(len(state))
        return dead

    # --- kinematics --------------------------------------------------------
    def velocities_device(self, state) -> torch.Tensor:
        def getter():
            v = torch.empty_like(state.p)
            _lib.check(self.lib.prt_get_velocities(
                len(state), state.p.data_ptr(), state.m.data_ptr(),
                self.units.VACUUM_LIGHT_SPEED(), v.data_ptr(),
                C.c_void_p(stream_handle())), "prt_get_velocities")
            return v
        return state.get_derived_quantity_from_cache("velocities_device", getter)

    def velocities(self, state) -> np.ndarray:
        """Host [n, 3], id order (cloud.py:425-432)."""
        return state._host3(self.velocities_device(state))

    def mean_beta(self, state):
        if len(state):
            return np.average(self.velocities(state), axis=0) / self.units.VACUUM_LIGHT_SPEED()
        return np.zeros((self.dimensions_velocity,))

    # --- deposition ----------------------------------------------------------
    def deposit_densities_device(self, state):
        return state.get_derived_quantity_from_cache(
            "rho_j_device", lambda: self.depositor.deposit_densities_device(state))

    def deposit_densities(self, state):
        """(rho [Nn], j [3, Nn]) as host arrays (cloud.py:513-526)."""
        rho, j = self.deposit_densities_device(state)
        return rho.cpu().numpy(), j.cpu().numpy()

    def deposit_j(self, state):
        return self.deposit_densities(state)[1]

    def deposit_rho(self, state):
        return self.deposit_densities(state)[0]

    # --- time advance ------------------------------------------------------------
    def advance_state(self, state, dx, dp, ddep=None):
        """New state with x += dx, p += dp, then relocated; particles lost at
        the boundary are removed (cloud.py:554-603). dx, dp: [n, 3] host arrays
        in id order (what ``velocities`` and the pusher's ``forces`` return) or
        [3, n] device tensors in store order."""
        order = state.id_order()
        if isinstance(dx, torch.Tensor):
            dxd, dpd = dx, dp
        else:
            dxd = to_store_from_id(dx, order, self.dev)
            dpd = to_store_from_id(dp, order, self.dev)
        x = (state.x + dxd).contiguous()
        p = (state.p + dpd).contiguous()
        new = PicState(self, x=x, p=p, q=state.q, m=state.m, el=state.el.clone(),
                       ids=state.ids, depositor_state=self.depositor.advance_state(state, ddep),
                       pusher_state=self.pusher.advance_state(state),
                       vis_listener=state.vis_listener,
                       pnss=state.particle_number_shift_signaller)
        new.next_id = state.next_id
        _lib.check(self.lib.prt_update_containing_elements(
            self.mesh_data.handle, self.workspace, len(new), new.x.data_ptr(),
            new.p.data_ptr(), new.el.data_ptr(), C.c_void_p(stream_handle())),
            "prt_update_containing_elements")
        self.check_status()
        self.transfer_find_counters()
        self.compact(new)
        return new

    def step(self, state, fields, dt, steps=1, deposit=True, sort_every=1,
             check=True, precision=0):
        """Device fast path: ``steps`` LSRK4 steps (5 fused stages each) with
        one rho/j deposition after each step. ``fields`` is a [6, Nn] device
        tensor (ex, ey, ez, bx, by, bz) or a sequence of six [Nn] tensors or
        None. Returns the last (rho, j) device tensors (or None)."""
        fptrs = self.pusher.field_pointers(fields)
        kx, kp = state.residuals()
        c = self.units.VACUUM_LIGHT_SPEED()
        s = C.c_void_p(stream_handle())
        out = None
        for step in range(steps):
            if sort_every and step % sort_every == 0:
                # at a step boundary the residuals are dead (the first stage's
                # a = 0 overwrites them), so they are not permuted
                self.sort_by_element(state, residuals=False)
                kx, kp = state.kx, state.kp
            for a, b in zip(LSRK4_A, LSRK4_B):
                self.pusher.lsrk_stage(state, fptrs, kx, kp, a, b, dt, c, precision)
            state.derived_quantity_cache.clear()
            if deposit:
                out = self.deposit_densities_device(state)
        if check:
            self.check_status()
        return out

    def sort_by_element(self, state, residuals=True):
        """Sort the store by containing element; `residuals=False` leaves the
        LSRK residuals unpermuted (valid only at a step boundary)."""
        kx, kp = state.residuals()
        _lib.check(self.lib.prt_sort_by_element(
            self.workspace, len(state), state.el.data_ptr(), state.x.data_ptr(),
            state.p.data_ptr(), state.q.data_ptr(), state.m.data_ptr(),
            kx.data_ptr() if residuals else None, kp.data_ptr() if residuals else None,
            state.ids.data_ptr(), C.c_void_p(stream_handle())),
            "prt_sort_by_element")
        state.derived_quantity_cache.clear()


def to_store_from_id(arr, order, dev) -> torch.Tensor:
    """Host [n, 3] in ascending-id order -> device [3, n] in store order."""
    a = torch.as_tensor(np.ascontiguousarray(arr, dtype=np.float64), device=dev)
    out = torch.empty((3, a.shape[0]), dtype=F64, device=dev)
    out[:, order] = a.T
    return out.contiguous()


class TimesteppablePicState:
    """Adapter letting an RK stepper advance a PicState (cloud.py:159-188)."""

    def __init__(self, method, state):
        self.method = method
        self.state = state

    def __mul__(self, factor):
        if factor != 1:
            raise NotImplementedError("cannot multiply PIC state by anything but unity.")
        return self

    __rmul__ = __mul__

    def __add__(self, update):
        if isinstance(update, (int, float)) and update == 0:
            return self
        dx, dp, ddep = update
        dx = NumberShiftableVector.unwrap(dx)
        dp = NumberShiftableVector.unwrap(dp)
        if isinstance(dx, (int, float)) and dx == 0:
            dx = np.zeros((len(self.state), 3))
        if isinstance(dp, (int, float)) and dp == 0:
            dp = np.zeros((len(self.state), 3))
        return TimesteppablePicState(self.method,
                                     self.method.advance_state(self.state, dx, dp, ddep))

    __radd__ = __add__


def _obj_array(items):
    out = np.empty(len(items), dtype=object)
    for k, v in enumerate(items):
        out[k] = v
    return out


class FieldToParticleRhsCalculator:
    """The particles' momentum right-hand side from the fields (cloud.py:238-290):
    the pusher's forces at the particles as a number-shiftable vector, in the
    (dx, dp, ddep) layout of a TimesteppablePicState update.

    ``maxwell_op`` supplies ``split_eh(fields) -> (e, h)``, ``get_eh_subset()``
    (six flags: which of ex, ey, ez, hx, hy, hz the field vector carries) and
    ``mu`` (B = mu H); absent components are zero."""

    def __init__(self, method, maxwell_op):
        self.method = method
        self.maxwell_op = maxwell_op

    def __call__(self, t, fields_f, state_f):
        fields = fields_f()
        state = state_f()
        e, h = self.maxwell_op.split_eh(fields)
        subset = list(self.maxwell_op.get_eh_subset())
        e_arg, b_arg = [], []
        idx = 0
        for use in subset[0:3]:
            e_arg.append(e[idx] if use else None)
            idx += 1 if use else 0
        idx = 0
        for use in subset[3:6]:
            b_arg.append(self.maxwell_op.mu * h[idx] if use else None)
            idx += 1 if use else 0
        velocities = self.method.velocities(state)
        forces = self.method.pusher.forces(state, velocities, *(e_arg + b_arg))
        return _obj_array([0, NumberShiftableVector(
            forces, signaller=state.particle_number_shift_signaller), 0])


class ParticleRhsCalculator:
    """The particles' position right-hand side (cloud.py:293-311): their
    velocities as a number-shiftable vector, plus the depositor's rhs."""

    def __init__(self, method, maxwell_op=None):
        self.method = method
        self.maxwell_op = maxwell_op

    def __call__(self, t, fields_f, state_f):
        state = state_f()
        velocities = self.method.velocities(state)
        return _obj_array([NumberShiftableVector(
            velocities, signaller=state.particle_number_shift_signaller), 0,
            self.method.depositor.rhs(state)])


# shape bandwidth --------------------------------------------------------------
def guess_shape_bandwidth(method, state, exponent):
    """Shape radius from the mesh (cloud.py:680-686): the mesh data's
    advisable particle radius."""
    method.depositor.set_shape_function(state, method.get_shape_function_class()(
        method.mesh_data.advisable_particle_radius(), method.mesh_data.dimensions, exponent))


def optimize_shape_bandwidth(method, state, analytic_rho, exponent):
    """Shape radius that best reproduces `analytic_rho` (cloud.py:691-824):
    50 radii from 2^-4 to 2^2 times the advisable one (log-spaced), each
    deposition's L1 error against `analytic_rho`; the largest radius at a
    local minimum of the error is set (a warning when even the best relative
    L1 error exceeds 0.1). Returns (chosen radius, tried radii, L1 errors)."""
    discr = method.discretization
    adv = method.mesh_data.advisable_particle_radius()
    radii = [adv * 2 ** i for i in np.linspace(-4, 2, 50)]
    cls = method.get_shape_function_class()

    def set_radius(r):
        method.depositor.set_shape_function(state, cls(r, method.mesh_data.dimensions, exponent))

    tried, errors = [], []
    for radius in radii:
        try:
            method.set_ignore_core_warnings(True)
            set_radius(radius)
            state.derived_quantity_cache.clear()
            rec_rho = method.deposit_rho(state)
        except RuntimeError as exc:
            if "particle mass is zero" in str(exc):
                continue
            raise
        finally:
            method.set_ignore_core_warnings(False)
        tried.append(radius)
        errors.append(discr.integral(np.abs(rec_rho - analytic_rho)))
    best = int(np.argmin(errors))
    rel = abs(errors[best] / discr.integral(analytic_rho))
    if rel > 0.1:
        import warnings
        warnings.warn("Charge density is very poorly resolved (rel L1 error=%g)" % rel)
    minima = [i for i in range(1, len(errors) - 1)
              if errors[i] < errors[i - 1] and errors[i] < errors[i + 1]]
    chosen = tried[max(minima)] if minima else tried[best]
    set_radius(chosen)
    state.derived_quantity_cache.clear()
    return chosen, tried, errors
