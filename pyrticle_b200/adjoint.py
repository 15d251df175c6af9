"""Differentiable particle trajectories (reverse mode, hand-written adjoints).

``DifferentiableTrajectory`` runs ``steps`` LSRK4 steps of the particle side
of a PIC step from initial positions and momenta, then deposits rho and j
from the final state, as one ``torch.autograd.Function``: gradients of any
loss of (rho, j) with respect to the initial positions and momenta, to the
coefficients theta of the fields along fixed basis fields, and to the nodal
field values.

Fields: ``F = fields + sum_k theta[k] * basis[k]`` ([6, Nn] each: ex, ey,
ez, bx, by, bz at the nodes). The forward keeps a checkpoint of the particle
state (x, p, element, order) every ``checkpoint_every`` steps; the backward
walks the segments in reverse, recomputes each from its checkpoint while
recording every stage's input state (``prt_lsrk_stage_record``: bitwise the
forward's arithmetic), then runs the stage adjoints in reverse
(``prt_lsrk_stage_adjoint``). The last segment is recorded by the forward
itself, so the backward starts with its stage adjoints. The deposition adjoint
(``prt_deposit_shape_adjoint``) and the velocity adjoint start the chain.
Every derivative is computed by libprt's CUDA kernels; torch tensors are the
device buffers and the autograd boundary.

Particles are sorted by element at each checkpoint (the element-sorted order
keeps the field gathers coherent); adjoints are carried across segments by
the particle order stored with each checkpoint. The launches of a segment
(recomputation and stage adjoints) are captured once into a CUDA graph and
replayed for the other segments of the same length.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from .cloud import LSRK4_A, LSRK4_B, stream_handle
from .deposition.shape import PRECISIONS

F64 = torch.float64


def _ptrs(tensors):
    arr = (C.c_void_p * len(tensors))()
    for k, t in enumerate(tensors):
        arr[k] = None if t is None else t.data_ptr()
    return arr


def _arg_key(a):
    """A hashable value of a launch argument (pointer arrays as tuples)."""
    if isinstance(a, C.Array):
        return tuple(a)
    if isinstance(a, C.c_void_p):
        return a.value
    return a


def _field_components(f):
    """Six component tensors of a [6, Nn] field, None where identically zero."""
    return [f[k] if bool(torch.any(f[k] != 0)) else None for k in range(6)]


def monomial_coefficients(method, comps):
    """Per-element monomial coefficients ([Nn] -> [E * Np]) of nodal field
    components (None stays None), the form the stage adjoint reads."""
    out = [None if c is None else torch.empty_like(c) for c in comps]
    _lib.check(method.lib.prt_fields_to_monomial(
        method.pusher.handle, len(comps), _ptrs(comps), _ptrs(out),
        C.c_void_p(stream_handle())), "prt_fields_to_monomial")
    return out


class DifferentiableTrajectory:
    """Differentiable ``steps`` LSRK4 steps + final rho/j deposition.

    @arg method: a PicMethod whose depositor is a (plain) ShapeFunctionDepositor
      with its shape function set.
    @arg charges, masses: [n] device tensors (not differentiated).
    @arg basis: optional [K, 6, Nn] device tensor of basis fields (K <= 4).
    @arg precision: deposition precision of the forward ("fp64" or "mixed");
      the trajectory and every adjoint run in FP64.
    """

    def __init__(self, method, charges, masses, dt, steps, checkpoint_every=10,
                 basis=None, precision="fp64"):
        dep = method.depositor
        if dep.mode != _lib.DEPOSIT_PLAIN:
            raise NotImplementedError("the deposition adjoint covers the plain shape depositor")
        if dep.shape_function is None:
            raise RuntimeError("shape function never set")
        if basis is not None and basis.shape[0] > _lib.MAX_FIELD_BASIS:
            raise ValueError("at most %d basis fields" % _lib.MAX_FIELD_BASIS)
        self.method = method
        self.lib = method.lib
        self.q = charges.contiguous()
        self.m = masses.contiguous()
        self.dt = float(dt)
        self.steps = int(steps)
        self.K = max(1, int(checkpoint_every))
        self.basis = basis.contiguous() if basis is not None else None
        self.precision = PRECISIONS[precision]
        self.c = method.units.VACUUM_LIGHT_SPEED()
        self.nn = len(method.discretization)
        # replay each segment's recomputation and adjoint launches from a
        # CUDA graph captured on the first full segment; the graphs are kept
        # across backward calls, keyed by every launch argument they hold
        # (the caching allocator hands a repeated call the same buffers, so
        # the capture happens once)
        self.use_graphs = True
        self._graphs = {}
        # when True, backward_run records CUDA events between its phases
        # (launching every segment eagerly) and leaves the elapsed
        # milliseconds per phase in self.phase_ms
        self.time_phases = False
        self.phase_ms = {}

    def __call__(self, x0, p0, theta=None, fields=None):
        dev = x0.device
        if theta is None:
            theta = torch.zeros((0 if self.basis is None else self.basis.shape[0],),
                                dtype=F64, device=dev)
        if fields is None:
            fields = torch.zeros((6, self.nn), dtype=F64, device=dev)
        return _TrajectoryFunction.apply(x0, p0, theta, fields, self)

    # ------------------------------------------------------------ pieces
    def combined_fields(self, theta, fields):
        F = fields.detach().clone()
        if self.basis is not None and theta.numel():
            F += torch.einsum("k,kcn->cn", theta.detach().to(F.device), self.basis)
        return F.contiguous()

    def _stage(self, F, x, p, q, m, el, kx, kp, a, b):
        _lib.check(self.lib.prt_lsrk_stage(
            self.method.pusher.handle, self.method.workspace, x.shape[1], x.data_ptr(),
            p.data_ptr(), q.data_ptr(), m.data_ptr(), el.data_ptr(), kx.data_ptr(),
            kp.data_ptr(), F, a, b, self.dt, self.c, 0, C.c_void_p(stream_handle())),
            "prt_lsrk_stage")

    def _sort(self, el, x, p, q, m, kx, kp, order):
        _lib.check(self.lib.prt_sort_by_element(
            self.method.workspace, x.shape[1], el.data_ptr(), x.data_ptr(), p.data_ptr(),
            q.data_ptr(), m.data_ptr(), kx.data_ptr(), kp.data_ptr(), order.data_ptr(),
            C.c_void_p(stream_handle())), "prt_sort_by_element")

    def _velocities(self, p, m):
        v = torch.empty_like(p)
        _lib.check(self.lib.prt_get_velocities(p.shape[1], p.data_ptr(), m.data_ptr(), self.c,
                                               v.data_ptr(), C.c_void_p(stream_handle())),
                   "prt_get_velocities")
        return v

    def forward_run(self, x0, p0, F):
        """Forward pass; returns (rho, j, saved) with the checkpoints."""
        meth = self.method
        n = x0.shape[1]
        dev = x0.device
        Fp = _ptrs(_field_components(F))
        x = x0.detach().clone().contiguous()
        p = p0.detach().clone().contiguous()
        q = self.q.clone()
        m = self.m.clone()
        el = meth.find_containing_elements_device(x)
        order = torch.arange(n, dtype=torch.int64, device=dev)
        kx = torch.zeros_like(x)
        kp = torch.zeros_like(p)
        checkpoints = []
        # the last segment runs recorded (prt_lsrk_stage_record, bitwise the
        # in-place stage): its tape spares the backward that recomputation
        last = ((self.steps - 1) // self.K) * self.K if self.steps else 0
        Tmax = 5 * min(self.K, self.steps) if self.steps else 0
        tape = None
        t = 0
        cs = C.c_void_p(stream_handle())
        for step in range(self.steps):
            if step % self.K == 0:
                self._sort(el, x, p, q, m, kx, kp, order)
                checkpoints.append((x.clone(), p.clone(), el.clone(), order.clone()))
                if step == last:
                    tape = (torch.empty((Tmax + 1, 3, n), dtype=F64, device=dev),
                            torch.empty((Tmax + 1, 3, n), dtype=F64, device=dev),
                            torch.empty((Tmax + 1, n), dtype=torch.int32, device=dev))
                    tape[0][0].copy_(x)
                    tape[1][0].copy_(p)
                    tape[2][0].copy_(el)
            if tape is None:
                for a, b in zip(LSRK4_A, LSRK4_B):
                    self._stage(Fp, x, p, q, m, el, kx, kp, a, b)
                continue
            tx, tp, te = tape
            for a, b in zip(LSRK4_A, LSRK4_B):
                _lib.check(self.lib.prt_lsrk_stage_record(
                    meth.pusher.handle, meth.workspace, n, tx[t].data_ptr(), tp[t].data_ptr(),
                    te[t].data_ptr(), tx[t + 1].data_ptr(), tp[t + 1].data_ptr(),
                    te[t + 1].data_ptr(), q.data_ptr(), m.data_ptr(), kx.data_ptr(),
                    kp.data_ptr(), Fp, a, b, self.dt, self.c, cs), "prt_lsrk_stage_record")
                t += 1
        if tape is not None:
            x = tape[0][t].clone()
            p = tape[1][t].clone()
            el = tape[2][t].clone()
        if not checkpoints:  # zero steps: the initial state is the final one
            self._sort(el, x, p, q, m, kx, kp, order)
            checkpoints.append((x.clone(), p.clone(), el.clone(), order.clone()))
        meth.check_status()
        v = self._velocities(p, m)
        rho = torch.empty((self.nn,), dtype=F64, device=dev)
        j = torch.empty((3, self.nn), dtype=F64, device=dev)
        dep = meth.depositor
        _lib.check(self.lib.prt_deposit_shape(
            meth.mesh_data.handle, meth.workspace, _lib.DEPOSIT_PLAIN, dep._shape_desc(), None,
            n, x.data_ptr(), q.data_ptr(), v.data_ptr(), el.data_ptr(), rho.data_ptr(),
            j.data_ptr(), self.precision, None, C.c_void_p(stream_handle())),
            "prt_deposit_shape")
        saved = dict(final=(x, p, el, q, m, order, v), checkpoints=checkpoints, tape=tape)
        return rho, j, saved

    def _mark(self, marks, name):
        if self.time_phases:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            marks.append((name, ev))

    def backward_run(self, saved, F, grho, gj, want_fields, want_theta):
        meth = self.method
        lib = self.lib
        s = C.c_void_p(stream_handle())
        marks = []
        self._mark(marks, "start")
        x, p, el, q, m, order, v = saved["final"]
        n = x.shape[1]
        dev = x.device
        lam_x = torch.zeros_like(x)
        lam_p = torch.zeros_like(p)
        lam_v = torch.zeros_like(p)
        grho = grho.contiguous() if grho is not None else None
        gj = gj.contiguous() if gj is not None else None
        _lib.check(lib.prt_deposit_shape_adjoint(
            meth.mesh_data.handle, meth.workspace, meth.depositor._shape_desc(), n,
            x.data_ptr(), q.data_ptr(), v.data_ptr(), el.data_ptr(),
            grho.data_ptr() if grho is not None else None,
            gj.data_ptr() if gj is not None else None, lam_x.data_ptr(), lam_v.data_ptr(), s),
            "prt_deposit_shape_adjoint")
        _lib.check(lib.prt_velocities_adjoint(n, p.data_ptr(), m.data_ptr(), self.c,
                                              lam_v.data_ptr(), lam_p.data_ptr(), s),
                   "prt_velocities_adjoint")
        self._mark(marks, "deposit_adjoint")
        lam_kx = torch.zeros_like(x)
        lam_kp = torch.zeros_like(p)
        comps = _field_components(F)
        Fp = _ptrs(comps)
        fcoef = monomial_coefficients(meth, comps)  # kept alive: Cp points into it
        Cp = _ptrs(fcoef)
        nb = self.basis.shape[0] if (self.basis is not None and want_theta) else 0
        grad_theta = torch.zeros((max(nb, 1),), dtype=F64, device=dev)
        if nb:
            bcomps = []
            for k in range(nb):
                bcomps += _field_components(self.basis[k])
            bcoef = monomial_coefficients(meth, bcomps)  # kept alive: Bp points into it
            Bp = _ptrs(bcoef)
        else:
            Bp = None
        grad_fields = torch.zeros((6, self.nn), dtype=F64, device=dev) if want_fields else None
        Gp = _ptrs([grad_fields[k] for k in range(6)]) if want_fields else None

        cps = saved["checkpoints"]
        cur_order = order
        Tmax = 5 * min(self.K, self.steps) if self.steps else 0
        fwd_tape = saved.get("tape")
        if fwd_tape is not None:
            tx, tp, te = fwd_tape  # holds the last segment's stages already
        else:
            tx = torch.empty((Tmax + 1, 3, n), dtype=F64, device=dev)
            tp = torch.empty((Tmax + 1, 3, n), dtype=F64, device=dev)
            te = torch.empty((Tmax + 1, n), dtype=torch.int32, device=dev)
        kx = torch.empty_like(x)
        kp = torch.empty_like(p)
        qs = torch.empty_like(self.q)
        ms = torch.empty_like(self.m)
        gth_ptr = grad_theta.data_ptr() if nb else None
        ptr = lambda t: t.data_ptr()  # noqa: E731
        # launch arguments of every stage of a segment, built once
        rec_args = [(meth.pusher.handle, meth.workspace, n, ptr(tx[t]), ptr(tp[t]), ptr(te[t]),
                     ptr(tx[t + 1]), ptr(tp[t + 1]), ptr(te[t + 1]), ptr(qs), ptr(ms), ptr(kx),
                     ptr(kp), Fp, LSRK4_A[t % 5], LSRK4_B[t % 5], self.dt, self.c)
                    for t in range(Tmax)]
        adj_args = [(meth.pusher.handle, meth.workspace, n, ptr(tx[t]), ptr(tp[t]), ptr(te[t]),
                     ptr(qs), ptr(ms), ptr(lam_x), ptr(lam_p), ptr(lam_kx), ptr(lam_kp), Cp,
                     LSRK4_A[t % 5], LSRK4_B[t % 5], self.dt, self.c, Gp, nb, Bp, gth_ptr)
                    for t in range(Tmax)]

        def segment(T):
            """Recompute T stages from tape slot 0, recording their inputs,
            then run the T stage adjoints in reverse, on the current stream
            (the capture stream while a graph is being captured)."""
            cs = C.c_void_p(stream_handle())
            kx.zero_()
            kp.zero_()
            for t in range(T):
                _lib.check(lib.prt_lsrk_stage_record(*rec_args[t], cs), "prt_lsrk_stage_record")
            self._mark(marks, "recompute")
            for t in reversed(range(T)):
                _lib.check(lib.prt_lsrk_stage_adjoint(*adj_args[t], cs),
                           "prt_lsrk_stage_adjoint")
            self._mark(marks, "stage_adjoint")

        graphs = self._graphs
        self._mark(marks, "setup")
        for seg in reversed(range(len(cps))):
            xs, ps, els, order_s = cps[seg]
            if cur_order is not order_s:
                # carry the adjoints from the later segment's particle order
                inv = torch.empty_like(cur_order)
                inv[cur_order] = torch.arange(n, dtype=torch.int64, device=dev)
                idx = inv[order_s]
                lam_x.copy_(lam_x[:, idx])
                lam_p.copy_(lam_p[:, idx])
                lam_kx.zero_()  # the first stage's a = 0 clears them at step boundaries
                lam_kp.zero_()
            cur_order = order_s
            T = 5 * min(self.K, self.steps - seg * self.K)
            if T == 0:
                continue
            torch.index_select(self.q, 0, order_s, out=qs)
            torch.index_select(self.m, 0, order_s, out=ms)
            if fwd_tape is not None and seg == len(cps) - 1:
                # recorded by the forward: the stage adjoints only
                self._mark(marks, "carry")
                cs = C.c_void_p(stream_handle())
                for t in reversed(range(T)):
                    _lib.check(lib.prt_lsrk_stage_adjoint(*adj_args[t], cs),
                               "prt_lsrk_stage_adjoint")
                self._mark(marks, "stage_adjoint")
                continue
            tx[0].copy_(xs)
            tp[0].copy_(ps)
            te[0].copy_(els)
            self._mark(marks, "carry")
            if not self.use_graphs or self.time_phases or seg == len(cps) - 1:
                segment(T)  # eager (the first one also sizes libprt's scratch)
                continue
            key = (T, tuple(tuple(_arg_key(a) for a in args) for args in rec_args[:T]),
                   tuple(tuple(_arg_key(a) for a in args) for args in adj_args[:T]))
            g = graphs.get(key)
            if g is None:
                if len(graphs) >= 8:
                    graphs.clear()
                # captured on a side stream with capture_begin/capture_end:
                # the torch.cuda.graph context would also empty the caching
                # allocator, making every later allocation a cudaMalloc
                g = torch.cuda.CUDAGraph()
                side = torch.cuda.Stream()
                side.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(side):
                    g.capture_begin()
                    try:
                        segment(T)
                    finally:
                        g.capture_end()
                torch.cuda.current_stream().wait_stream(side)
                graphs[key] = g
            g.replay()
        meth.check_status()
        inv = torch.empty_like(cur_order)
        inv[cur_order] = torch.arange(n, dtype=torch.int64, device=dev)
        gx0 = lam_x[:, inv].contiguous()
        gp0 = lam_p[:, inv].contiguous()
        self._mark(marks, "carry")
        if self.time_phases:
            torch.cuda.synchronize()
            self.phase_ms = {}
            for (_, e0), (name, e1) in zip(marks[:-1], marks[1:]):
                self.phase_ms[name] = self.phase_ms.get(name, 0.0) + e0.elapsed_time(e1)
        return gx0, gp0, (grad_theta[:nb] if nb else None), grad_fields


class _TrajectoryFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, p0, theta, fields, traj):
        F = traj.combined_fields(theta, fields)
        rho, j, saved = traj.forward_run(x0, p0, F)
        ctx.traj = traj
        ctx.saved = saved
        ctx.F = F
        ctx.theta_shape = theta.shape
        ctx.theta_device = theta.device
        return rho, j

    @staticmethod
    def backward(ctx, grho, gj):
        traj = ctx.traj
        want_fields = ctx.needs_input_grad[3]
        want_theta = ctx.needs_input_grad[2]
        gx0, gp0, gth, gf = traj.backward_run(ctx.saved, ctx.F, grho, gj, want_fields,
                                              want_theta)
        gtheta = None
        if want_theta:
            gtheta = (gth if gth is not None
                      else torch.zeros(ctx.theta_shape, dtype=F64)).to(ctx.theta_device)
        ctx.saved = None
        return gx0, gp0, gtheta, gf, None
