"""Benchmark: particle-steps/s of the particle side of a PIC step on B200.

One step = 5 fused LSRK4 stages (velocity, monomial interpolation, Lorentz
force, RK update, element relocation) + one deposition of rho and j onto the
DG nodes (+ the element sort of the store). Default workload: config2 --
32x32x128 cubes x 6 jittered tets (786,432 tets), order 3 (Np = 20,
15.7M nodes), 16M electrons in an r < 0.25 cm beam, shape-function
deposition with radius 0.08 cm, static Bz + 8 seeded Fourier modes of E and
B; FP64 plain form. Inputs are far larger than L2 (3.5 GB of particle state
moved per stage), so no L2 flush is needed between steps.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
With N > 1 (torchrun), every rank advances its own 16M particles (weak
scaling) and rho/j are summed across ranks with one NCCL all-reduce per step.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--depositor", default="normalized", choices=["normalized", "plain"],
                    help="NormalizedShapeFunctionDepositor (the chosen form's deposition, "
                         "default) or ShapeFunctionDepositor")
    ap.add_argument("--adjoint-scale", type=float, default=1.0,
                    help="particle-count scale of the differentiable workload (1M electrons)")
    ap.add_argument("--adjoint-config4", type=float, default=None, metavar="SCALE",
                    help="only the config4 adjoint (50 steps, checkpoint every 5) at this "
                         "particle-count scale of its 64M; prints its own JSON line")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_method(w, torch, normalized=False):
    from pyrticle_b200.cloud import PicMethod
    from pyrticle_b200.deposition.shape import (NormalizedShapeFunctionDepositor,
                                                ShapeFunctionDepositor)
    from pyrticle_b200.discretization import Discretization
    from pyrticle_b200.pusher import MonomialParticlePusher
    from pyrticle_b200.tools import PolynomialShapeFunction
    from pyrticle_b200.units import SIUnitsWithNaturalConstants as U
    discr = Discretization(w.mesh, w.order, nodes=w.nodes)
    dep = NormalizedShapeFunctionDepositor() if normalized else ShapeFunctionDepositor()
    m = PicMethod(discr, U, dep, MonomialParticlePusher(), 3, 3)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    m.depositor.set_shape_function(None, sf)
    return m, sf


def count_pairs(m, state, sf):
    """Exact (particle, position) and (particle, node) pair counts inside the
    radius, the pairs the FP64 kernel evaluates after its culls, and the
    pairs the tensor-core kernel evaluates per pass (candidates x 128 tile
    rows); two extra deposition calls."""
    from pyrticle_b200 import _lib
    import torch
    nn = len(m.discretization)
    rho = torch.empty((nn,), dtype=torch.float64, device="cuda")
    out = []
    for prec in (0, 1):
        st = _lib.DepositStats()
        _lib.check(m.lib.prt_deposit_shape(
            m.mesh_data.handle, m.workspace, _lib.DEPOSIT_PLAIN,
            _lib.ShapeFunctionDesc(sf.radius, sf.exponent, sf.normalizer), None, len(state),
            state.x.data_ptr(), state.q.data_ptr(), None, state.el.data_ptr(), rho.data_ptr(),
            None, prec, C.byref(st), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        out.append(st)
    return (int(out[0].pair_count), int(out[0].node_pair_count), int(out[0].evaluated_pairs),
            int(out[1].evaluated_pairs))


def timing_read(m, cat, reset=True):
    from pyrticle_b200 import _lib
    ms = C.c_double()
    k = C.c_int64()
    _lib.check(m.lib.prt_workspace_timing_read(m.workspace, cat, C.byref(ms), C.byref(k),
                                               int(reset)))
    return ms.value, k.value


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# dominant kernels on the config2 workload at full size (16M particles), from
# one-pass ncu captures of `python bench.py --steps 1 --warmup 1 --no-e2e
# --no-adjoint --no-cpu-baseline` (summarised in
# profiles/dram_traffic_config2_16M.md); reported only for that workload.
MEASURED_TRAFFIC = {
    "config2": {
        "tc_deposit_kernel<0, 0>": 1486009600 + 119841792,
        "tc_deposit_kernel<1, 1>": 1075521536 + 520001792,
        "deposit_groups_kernel<1, 1, 2>": 166834674176 + 130093312,
        "lsrk_stage_mixed_kernel<3>": 2012872448 + 1545450240,
    }
}


def measured_traffic(args, kernel):
    if args.scale != 1.0:
        return None
    return MEASURED_TRAFFIC.get(args.workload, {}).get(kernel)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_peak_tflops(torch):
    """FP64 peak measured here: cuBLAS DGEMM 8192^3, best of 5 (CUDA events)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e9
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def fp32_peak_tflops(torch):
    """FP32 CUDA-core peak measured here: cuBLAS SGEMM 8192^3 with TF32 off."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, dtype=torch.float32, device="cuda")
        b = torch.randn(n, n, dtype=torch.float32, device="cuda")
        for _ in range(2):
            torch.matmul(a, b)
        best = 1e9
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b)
            e1.record()
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def form_accuracy(m, s, fields, dt, torch, steps=5):
    """Errors of the chosen form against the plain FP64 form on the same
    state: one deposition (rho, j), the first stage's residual kp = dt F
    (forces), and positions / momentum changes after `steps` steps."""
    from pyrticle_b200 import _lib
    from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))  # noqa: E731
    r64, j64 = m.depositor.deposit_densities_device(s, precision="fp64")
    r32, j32 = m.depositor.deposit_densities_device(s, precision="mixed")
    out = {"rho_rel_l2": rel(r32, r64), "j_rel_l2": rel(j32, j64)}
    del r64, j64, r32, j32
    fp = m.pusher.field_pointers(fields)
    c = m.units.VACUUM_LIGHT_SPEED()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run(prec, stages):
        x, p, el = s.x.clone(), s.p.clone(), s.el.clone()
        kx = torch.zeros_like(x)
        kp = torch.zeros_like(p)
        for t in range(stages):
            _lib.check(m.lib.prt_lsrk_stage(
                m.pusher.handle, m.workspace, x.shape[1], x.data_ptr(), p.data_ptr(),
                s.q.data_ptr(), s.m.data_ptr(), el.data_ptr(), kx.data_ptr(), kp.data_ptr(), fp,
                LSRK4_A[t % 5], LSRK4_B[t % 5], dt, c, prec, stream))
        return x, p, el, kp

    kp64 = run(0, 1)[3]
    kp32 = run(1, 1)[3]
    out["force_rel_l2"] = rel(kp32, kp64)
    del kp64, kp32
    x64, p64, el64, _ = run(0, 5 * steps)
    x32, p32, el32, _ = run(1, 5 * steps)
    out[f"x_rel_l2_after_{steps}_steps"] = rel(x32, x64)
    out[f"dp_rel_l2_after_{steps}_steps"] = rel(p32 - s.p, p64 - s.p)
    out["elements_equal_fraction"] = float((el32 == el64).float().mean())
    del x64, p64, el64, x32, p32, el32
    m.check_status()
    out["normalized_total_charge_rel_error"] = normalized_charge(m, s, torch)
    return out


def normalized_charge(m, s, torch):
    """|sum_e |J_e| sum_i w_i rho_i - sum_p q_p| / |sum_p q_p| of the
    normalising depositor on the same state: FP64 (the form the normalised
    depositor keeps in the chosen configuration) and FP32 weights."""
    from pyrticle_b200.deposition.shape import NormalizedShapeFunctionDepositor
    dep = NormalizedShapeFunctionDepositor()
    dep.initialize(m)
    dep.set_shape_function(None, m.depositor.shape_function)
    iw = torch.as_tensor(dep.integral_weights, device=s.x.device)
    jac = torch.as_tensor(m.discretization.mesh.jacobians, device=s.x.device)
    qsum = float(s.q.sum())
    out = {}
    for prec in ("fp64", "mixed"):
        rho, _ = dep.deposit_densities_device(s, j=False, precision=prec)
        total = float(((rho.view(-1, iw.shape[0]) @ iw) * jac).sum())
        out[prec] = abs(total - qsum) / abs(qsum)
        del rho
    return out


def cpu_baseline(w, target_seconds, threads=0, steps=1, seed=7):
    """The oracle's multi-core path on a bounded random sample of the
    workload's particles (full mesh and fields): particle-steps/s."""
    from oracle import pyoracle as O
    from pyrticle_b200 import meshgen, refelement
    from pyrticle_b200.cloud import LSRK4_A, LSRK4_B
    from pyrticle_b200.tools import PolynomialShapeFunction
    from pyrticle_b200.units import SIUnitsWithNaturalConstants as U
    om = O.OracleMesh(w.mesh, w.nodes, meshgen.element_bins(w.mesh))
    ex = refelement.node_tuples(w.order)
    pu = O.OraclePusher(ex, refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex),
                        parallel=True)
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    c = U.VACUUM_LIGHT_SPEED()
    rng = np.random.default_rng(seed)
    threads = threads or O.max_threads()

    def sample(n):
        idx = np.sort(rng.choice(w.particle_count, size=n, replace=False))
        x = w.positions[idx]
        return idx, x, O.find_containing_elements(om, x, linear=False)

    def run(n):
        idx, x, el = sample(n)
        t0 = time.perf_counter()
        r = O.pic_steps_parallel(pu, om, x, w.momenta[idx], w.charges[idx], w.masses[idx], el,
                                 list(w.fields), LSRK4_A, LSRK4_B, w.dt, c, steps, sf,
                                 threads=threads)
        dt = time.perf_counter() - t0
        assert r["rc"] == 0
        return dt

    # two sizes: the per-particle (marginal) cost excludes the fixed cost of
    # a deposition over the full node set, which a full-size run amortises
    n1 = 2000
    t1 = run(n1)
    n2 = int(max(4 * n1, min(w.particle_count, 2 * n1 * target_seconds / max(t1, 1e-9))))
    t2 = run(n2)
    marginal = (t2 - t1) / (n2 - n1)
    out = {"value": steps / marginal if marginal > 0 else n2 * steps / t2, "unit": METRIC,
           "cores": threads, "kind": "port",
           "value_including_fixed_cost": n2 * steps / t2,
           "sample": f"{n1} and {n2} random particles of the workload x {steps} step(s) on the "
                     f"full mesh/fields, oracle OpenMP build ({t1:.1f} s, {t2:.1f} s); value = "
                     f"1 / per-particle cost from the two sizes"}
    # one core: the reference's serial algorithms (oracle serial build)
    pu1 = O.OraclePusher(ex, refelement.monomial_vandermonde(refelement.unit_nodes(w.order), ex))
    ts = []
    for n in (n1 // 4, n1):
        idx, x, el = sample(n)
        t0 = time.perf_counter()
        r = O.lsrk_steps(pu1, om, x, w.momenta[idx], w.charges[idx], w.masses[idx], el,
                         list(w.fields), LSRK4_A, LSRK4_B, w.dt, c, steps)
        O.deposit_shape(om, 0, sf, r["x"], r["q"], O.velocities(r["p"], r["m"], c), r["el"])
        ts.append((n, time.perf_counter() - t0))
    (na, ta), (nb, tb) = ts
    m1 = (tb - ta) / (nb - na)
    out["one_core"] = {"value": steps / m1 if m1 > 0 else nb * steps / tb, "unit": METRIC,
                       "cores": 1, "kind": "port",
                       "sample": f"{na} and {nb} particles x {steps} step(s), oracle serial "
                                 f"build ({ta:.1f} s, {tb:.1f} s)"}
    return out


def run_reference(args):
    """The reference's CPU algorithms (restated in the oracle; the reference
    itself cannot be built here) on the host cores, bounded sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from pyrticle_b200 import problems
    w = problems.make(args.workload, scale=args.scale)
    from oracle import pyoracle as O
    threads = O.max_threads()
    # one pilot to size the per-step sample to ~target seconds
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    base = cpu_baseline(w, per_step, threads=threads)
    n_per_step = int(base["value"] * per_step)
    times = []
    for k in range(args.warmup + args.steps):
        b = cpu_baseline(w, per_step, threads=threads, seed=100 + k)
        if k >= args.warmup:
            times.append(b["value"])
    value = float(np.mean(times))
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "particles_per_step_sample": n_per_step},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                             "sample": base["sample"]},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def adjoint_bench(torch, scale, hbm_gbs, reps=3, checkpoint_every=10):
    """Differentiable workload (16x16x64 cubes, order 3, 1M electrons, 100
    LSRK4 steps, checkpoint every 10): forward (push + final deposition) and
    backward (deposition adjoint + recomputation + stage adjoints) times of
    one autograd call, loss sum over nodes of (j - j_target)^2 with j_target
    from a run with 5% higher Bz; gradients with respect to the initial
    momenta and the (Bz, focusing gradient) scalars. The chosen form (FP32
    deposition in the forward, its own target) against the FP64 check run."""
    from pyrticle_b200 import _lib, problems
    from pyrticle_b200.adjoint import DifferentiableTrajectory
    w = problems.make("config3", scale=scale)
    m, sf = build_method(w, torch)
    dev = torch.device("cuda")
    f64 = torch.float64
    basis = torch.as_tensor(w.field_basis, dtype=f64, device=dev).contiguous()
    theta = torch.as_tensor(w.theta, dtype=f64, device=dev)
    q = torch.as_tensor(w.charges, dtype=f64, device=dev)
    mass = torch.as_tensor(w.masses, dtype=f64, device=dev)
    x0 = torch.as_tensor(w.positions.T.copy(), dtype=f64, device=dev).contiguous()
    p0 = torch.as_tensor(w.momenta.T.copy(), dtype=f64, device=dev).contiguous()
    trajs = {form: DifferentiableTrajectory(m, q, mass, w.dt, w.steps, checkpoint_every,
                                            basis=basis, precision=form)
             for form in ("mixed", "fp64")}
    # targets from the same form (a run with 5% higher Bz)
    j_t = {}
    with torch.no_grad():
        for form, traj in trajs.items():
            _, j_t[form] = traj(x0, p0, theta * torch.tensor([1.05, 1.0], dtype=f64, device=dev))

    def run(traj, target):
        p = p0.clone().requires_grad_()
        th = theta.clone().requires_grad_()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        rho, j = traj(x0, p, th)
        L = ((j - target) ** 2).sum()
        e[1].record()
        L.backward()
        e[2].record()
        torch.cuda.synchronize()
        return (e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), p.grad, th.grad,
                float(L.detach()))

    out = {}
    for form in ("mixed", "fp64"):
        run(trajs[form], j_t[form])  # warm-up
        f = b = 0.0
        for _ in range(reps):
            fm, bm, gp, gth, L = run(trajs[form], j_t[form])
            f += fm
            b += bm
        # one more call with per-kernel events and the backward's phases
        _lib.check(m.lib.prt_workspace_timing(m.workspace, 1))
        for cat in (_lib.TIME_LSRK_STAGE, _lib.TIME_STAGE_ADJOINT, _lib.TIME_DEPOSIT_ADJOINT):
            timing_read(m, cat, reset=True)
        trajs[form].time_phases = True
        run(trajs[form], j_t[form])
        trajs[form].time_phases = False
        _lib.check(m.lib.prt_workspace_timing(m.workspace, 0))
        adj_ms, adj_n = timing_read(m, _lib.TIME_STAGE_ADJOINT)
        dep_ms, dep_n = timing_read(m, _lib.TIME_DEPOSIT_ADJOINT)
        n = len(w.positions)
        # per adjoint stage: read x, p (48 B), element (4), q, m (16), four
        # adjoints (96); write four adjoints (96)
        adj_gbs = 260.0 * n / (adj_ms / max(adj_n, 1) * 1e-3) / 1e9
        out[form] = {"forward_ms": f / reps, "backward_ms": b / reps,
                     "ratio_backward_over_forward": b / f, "loss": L,
                     "grad_p0": gp, "grad_theta": gth,
                     "stage_adjoint_kernel_ms": adj_ms / max(adj_n, 1),
                     "stage_adjoint_gbs": adj_gbs, "stage_adjoint_frac_hbm": adj_gbs / hbm_gbs,
                     "deposit_adjoint_ms": dep_ms / max(dep_n, 1),
                     "backward_phases_ms": dict(trajs[form].phase_ms)}
    g32, g64 = out["mixed"].pop("grad_p0"), out["fp64"].pop("grad_p0")
    t32, t64 = out["mixed"].pop("grad_theta"), out["fp64"].pop("grad_theta")

    # the mixed-vs-FP64 gradient gap split: the loss above differences two
    # nearby currents (j - j_target is a small part of j), which amplifies
    # the forward's FP32 deposition error by |j| / |j - j_target|; the same
    # gradients for the well-conditioned loss sum j^2 show the FP32 error
    # itself
    def grads_sq(traj):
        p = p0.clone().requires_grad_()
        th = theta.clone().requires_grad_()
        _, j = traj(x0, p, th)
        (j ** 2).sum().backward()
        return p.grad, th.grad

    with torch.no_grad():
        j64 = trajs["fp64"](x0, p0, theta)[1]
        j32 = trajs["mixed"](x0, p0, theta)[1]
    kappa = float(torch.linalg.norm(j64) / torch.linalg.norm(j64 - j_t["fp64"]))
    sq32, sqt32 = grads_sq(trajs["mixed"])
    sq64, sqt64 = grads_sq(trajs["fp64"])

    # central differences of the FP64 run, h = 1e-6 relative, on 64 random
    # directions in (initial momenta, Bz, focusing gradient), for the
    # well-conditioned loss: with the target loss, j - j_target is ~1e-7 of
    # j, so a 1e-6 step is already beyond the range where the loss is
    # quadratic in it and the differences measure its curvature instead
    def loss_sq(p, th):
        with torch.no_grad():
            return float((trajs["fp64"](x0, p, th)[1] ** 2).sum())

    h = 1e-6
    pscale = float(torch.sqrt((p0 ** 2).sum(0).mean()))
    gen = torch.Generator(device="cpu").manual_seed(11)
    fd_worst = 0.0
    t0 = time.perf_counter()
    for _ in range(64):
        dp = torch.randn(p0.shape, generator=gen, dtype=f64).to(dev) * pscale
        dth = torch.randn(2, generator=gen, dtype=f64).to(dev) * theta
        fd = (loss_sq(p0 + h * dp, theta + h * dth) -
              loss_sq(p0 - h * dp, theta - h * dth)) / (2 * h)
        ad = float((sq64 * dp).sum() + (sqt64 * dth).sum())
        fd_worst = max(fd_worst, abs(fd - ad) / abs(ad))
    fd_s = time.perf_counter() - t0
    return {"workload": f"config3: {w.mesh.element_count} tets order {w.order}, "
                        f"{len(w.positions)} electrons, {w.steps} LSRK4 steps, checkpoint "
                        f"every {checkpoint_every} steps with recomputation",
            "chosen_form": out["mixed"], "fp64_check_run": out["fp64"],
            "grad_p0_rel_l2_mixed_vs_fp64": float(torch.linalg.norm(g32 - g64) /
                                                  torch.linalg.norm(g64)),
            "grad_theta_mixed": [float(v) for v in t32],
            "grad_theta_fp64": [float(v) for v in t64],
            "loss_rel_diff_mixed_vs_fp64": abs(out["mixed"]["loss"] - out["fp64"]["loss"]) /
                                           abs(out["fp64"]["loss"]),
            "central_differences": {
                "form": "fp64", "loss": "sum of j^2", "directions": 64, "h_relative": h,
                "worst_rel_diff_vs_adjoint": fd_worst, "seconds": fd_s},
            "gradient_gap_split": {
                "j_rel_l2_mixed_vs_fp64": float(torch.linalg.norm(j32 - j64) /
                                                torch.linalg.norm(j64)),
                "loss_condition_j_over_j_minus_target": kappa,
                "predicted_gap": kappa * float(torch.linalg.norm(j32 - j64) /
                                               torch.linalg.norm(j64)),
                "well_conditioned_loss": "sum of j^2",
                "grad_p0_rel_l2_mixed_vs_fp64": float(torch.linalg.norm(sq32 - sq64) /
                                                      torch.linalg.norm(sq64)),
                "grad_theta_rel_l2_mixed_vs_fp64": float(torch.linalg.norm(sqt32 - sqt64) /
                                                         torch.linalg.norm(sqt64))}}


def grid_bench(args, torch):
    """config1: GridDepositor (shape weights on one 128 x 128 x 512 brick's
    points, then the FP64 remap to the DG nodes), 4M particles, order 3,
    radius 0.1 cm. Times the host set-up, and K steps of the FP64 form and of
    the chosen (mixed) form: tensor-core stages and the tensor-core grid
    deposition. One GPU only."""
    from pyrticle_b200 import problems
    from pyrticle_b200.cloud import PicMethod
    from pyrticle_b200.deposition.grid import GridDepositor
    from pyrticle_b200.deposition.grid_base import SingleBrickGenerator
    from pyrticle_b200.discretization import Discretization
    from pyrticle_b200.pusher import MonomialParticlePusher
    from pyrticle_b200.tools import PolynomialShapeFunction
    from pyrticle_b200.units import SIUnitsWithNaturalConstants as U
    w = problems.make("config1", scale=args.scale)
    discr = Discretization(w.mesh, w.order, nodes=w.nodes)
    t0 = time.perf_counter()
    dep = GridDepositor(SingleBrickGenerator(dims=w.brick_dims))
    m = PicMethod(discr, U, dep, MonomialParticlePusher(), 3, 3)
    setup_s = time.perf_counter() - t0
    sf = PolynomialShapeFunction(w.shape_radius, 3, 2)
    m.depositor.set_shape_function(None, sf)
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    fields = torch.as_tensor(w.fields, device="cuda")
    n = len(s)

    def one_step(prec):
        dep.precision = "mixed" if prec == 1 else "fp64"
        try:
            return m.step(s, fields, w.dt, steps=1, check=False, precision=prec)
        finally:
            dep.precision = "fp64"

    for prec in (0, 1):
        for _ in range(args.warmup):
            one_step(prec)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()

    def timed(prec):
        _lib_check = m.lib.prt_workspace_timing
        _lib_check(m.workspace, 1)
        for cat in range(7):
            timing_read(m, cat, reset=True)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        e[0].record()
        for _ in range(args.steps):
            one_step(prec)
        e[1].record()
        torch.cuda.synchronize()
        _lib_check(m.workspace, 0)
        kernel = {name: timing_read(m, cat)[0] / args.steps for cat, name in
                  ((0, "deposit_grid"), (1, "deposit_stage"), (2, "lsrk_stage"), (3, "sort"))}
        return e[0].elapsed_time(e[1]), kernel

    ms64, k64 = timed(0)
    ms, k = timed(1)
    clk = clocks.stop()
    m.check_status()
    # the chosen form's grid densities against FP64 on the same state
    dep.precision = "mixed"
    gr32, gj32 = dep.deposit_grid_densities_device(s)
    dep.precision = "fp64"
    gr, gj = dep.deposit_grid_densities_device(s)
    acc = {"grid_rho_rel_l2": float(torch.linalg.norm(gr32 - gr) / torch.linalg.norm(gr)),
           "grid_j_rel_l2": float(torch.linalg.norm(gj32 - gj) / torch.linalg.norm(gj))}
    # the remap alone (rho and the three j components), CUDA events
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e[0].record()
    dep.remap_grid_to_mesh_device(gr)
    dep.remap_grid_to_mesh_device(gj)
    e[1].record()
    torch.cuda.synchronize()
    remap_ms = e[0].elapsed_time(e[1])
    # algorithmic work of the grid deposition: 15 flops per (particle, grid
    # point) pair within the radius, the points of a radius ball
    cell = float(np.prod(np.asarray(dep.bricks[0].stepwidths)))
    pairs = n * (4.0 / 3.0 * np.pi * sf.radius ** 3) / cell
    fp64 = fp64_peak_tflops(torch)
    achieved64 = 15.0 * pairs / (k64["deposit_grid"] * 1e-3) / 1e12
    peaks, src = measured_peaks()
    bf16 = float(peaks.get("bf16_tflops", 1590.0))
    # the chosen form's grid deposition: 80 dense-FP16-equivalent tensor flops
    # per evaluated pair; counted here over the pairs within the radius only
    # (a lower bound of the executed work)
    achieved = 80.0 * pairs / (k["deposit_grid"] * 1e-3) / 1e12
    value = n * args.steps / (ms * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16/i8 tensor + f32 + f64 (mixed: tensor-core grid deposition with "
                     "split-FP16 scores and 23-bit integer weights summed exactly on the int8 "
                     "tensor cores, FP64 per-point combine and remap; split-BF16 tensor-core "
                     "Lagrange values; FP64 state/force/locate)",
            "data": "synthetic (seeded mesh, particles and fields of the workload)",
            "config": {"workload": f"config1: {w.mesh.element_count} tets order {w.order}, "
                                   f"{n} particles, GridDepositor on one "
                                   f"{'x'.join(str(d) for d in w.brick_dims)} brick, shape "
                                   f"radius {sf.radius * 100:g} cm",
                       "particles_per_gpu": n, "grid_points": dep.grid_node_count,
                       "l2": "inputs larger than L2", "parallelism": "1 GPU"},
            "clocks": clk, "e2e": None,
            "grid_setup_s": setup_s,
            "kernel_ms_per_step": k, "remap_ms_per_deposition": remap_ms,
            "accuracy_mixed_vs_fp64": acc,
            "speedup_mixed_vs_fp64": ms64 / ms,
            "fp64": {"value": n * args.steps / (ms64 * 1e-3), "ms_per_step": ms64 / args.steps,
                     "kernel_ms_per_step": k64,
                     "roofline": {"bound": "fp64", "kernel": "deposit_grid_kernel (FP64)",
                                  "achieved": achieved64, "peak": fp64, "unit": "TFLOP/s",
                                  "frac": achieved64 / fp64, "traffic": None,
                                  "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                                  "algorithmic": f"15 flops x {pairs:.4g} (particle, grid point) "
                                                 "pairs within the radius per deposition"}},
            "roofline": {"bound": "tensor",
                         "kernel": "tc_deposit_kernel (grid points, chosen form)",
                         "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                         "frac": achieved / bf16, "traffic": None,
                         "peak_source": ("MEASURED_PEAKS.json bf16_tflops" if src == "measured"
                                         else "fallback 1,590 TFLOP/s"),
                         "algorithmic": f"80 dense-FP16-equivalent tensor flops x {pairs:.4g} "
                                        "(particle, grid point) pairs within the radius (a lower "
                                        "bound: the kernel evaluates more pairs)"}}
    print(json.dumps(line), flush=True)


def adjoint_config4(torch, scale):
    """config4's differentiable run: the 3,145,728-tet order-4 mesh, a Gaussian
    bunch of 64M x scale electrons, 50 LSRK4 steps forward (chosen form:
    mixed final deposition) and the adjoint with a checkpoint every 5 steps;
    loss sum of j^2 (the workload has no field parameters). Reports the times
    and the device memory in use after the forward and at the end of the
    backward (cudaMemGetInfo: libprt's workspace and tapes included)."""
    from pyrticle_b200 import problems
    from pyrticle_b200.adjoint import DifferentiableTrajectory
    w = problems.make("config4", scale=scale)
    m, sf = build_method(w, torch)
    dev = torch.device("cuda")
    f64 = torch.float64
    q = torch.as_tensor(w.charges, dtype=f64, device=dev)
    mass = torch.as_tensor(w.masses, dtype=f64, device=dev)
    x0 = torch.as_tensor(w.positions.T.copy(), dtype=f64, device=dev).contiguous()
    p0 = torch.as_tensor(w.momenta.T.copy(), dtype=f64, device=dev).contiguous()
    fields = torch.as_tensor(w.fields, dtype=f64, device=dev).contiguous()
    traj = DifferentiableTrajectory(m, q, mass, w.dt, w.steps, 5, precision="mixed")
    total = torch.cuda.mem_get_info()[1]

    def used():
        free, tot = torch.cuda.mem_get_info()
        return tot - free

    out = {}
    for rep in range(2):  # the first call sizes the buffers and captures the graphs
        p = p0.clone().requires_grad_()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        e[0].record()
        _, j = traj(x0, p, None, fields)
        L = (j ** 2).sum()
        e[1].record()
        torch.cuda.synchronize()
        after_forward = used()
        L.backward()
        e[2].record()
        torch.cuda.synchronize()
        out = {"forward_ms": e[0].elapsed_time(e[1]), "backward_ms": e[1].elapsed_time(e[2]),
               "device_bytes_after_forward": after_forward,
               "device_bytes_end_of_backward": used()}
        del p, j, L
    out["ratio_backward_over_forward"] = out["backward_ms"] / out["forward_ms"]
    line = {"metric": "adjoint backward / forward", "workload":
            f"config4: {w.mesh.element_count} tets order {w.order}, {len(w.positions)} "
            f"electrons ({scale:g} x 64M), {w.steps} LSRK4 steps, checkpoint every 5 steps "
            "with recomputation, loss sum j^2, chosen form (mixed final deposition)",
            "device_bytes_total": total, **out}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    if args.workload == "config1":
        grid_bench(args, torch)
        return
    if args.adjoint_config4 is not None:
        adjoint_config4(torch, args.adjoint_config4)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from pyrticle_b200 import _lib, problems
    from pyrticle_b200.sharding import (allreduce_densities, deposit_densities_exact,
                                        max_over_ranks)

    # weak scaling: every rank holds the particles of its slab of a beam
    # world times larger (its contiguous block of the element-sorted order)
    w = problems.make(args.workload, scale=args.scale, seed=1 + rank,
                      zslab=(rank, world) if world > 1 and args.workload != "config4" else None)
    m, sf = build_method(w, torch, normalized=args.depositor == "normalized")
    s = m.make_state()
    m.add_particles_from_arrays(s, w.positions, w.momenta, w.charges, w.masses)
    fields = torch.as_tensor(w.fields, device="cuda")
    n = len(s)
    nn = len(m.discretization)

    prec = {"fp64": 0, "mixed": 1}

    def one_step(form):
        """One step of the given form: 5 fused RK stages + the deposition.
        With several ranks the chosen form deposits through the exact sharded
        protocol (charge maxima all-reduced, integer digit sums all-reduced:
        bitwise the same for any rank count); the FP64 form all-reduces rho
        and j."""
        m.depositor.precision = form
        try:
            if world > 1 and form == "mixed":
                m.step(s, fields, w.dt, steps=1, deposit=False, check=False, precision=prec[form])
                return deposit_densities_exact(m, s)
            rho, j = m.step(s, fields, w.dt, steps=1, check=False, precision=prec[form])
        finally:
            m.depositor.precision = "fp64"
        if world > 1:
            allreduce_densities(rho, j)
        return rho, j

    for form in ("fp64", "mixed"):
        for _ in range(args.warmup):
            one_step(form)
    torch.cuda.synchronize()
    pairs, node_pairs, evaluated, evaluated_tc = count_pairs(m, s, sf)
    accuracy = form_accuracy(m, s, fields, w.dt, torch)

    clocks = ClockSampler(local)
    clocks.start()

    def timed(form):
        """K timed steps of one form (device events, max over ranks) with the
        per-category kernel times."""
        _lib.check(m.lib.prt_workspace_timing(m.workspace, 1))
        for cat in range(7):
            timing_read(m, cat, reset=True)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            one_step(form)
        e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        _lib.check(m.lib.prt_workspace_timing(m.workspace, 0))
        t = e0.elapsed_time(e1)
        if world > 1:
            t = max_over_ranks(t, "cuda")
        kernel = {name: timing_read(m, cat) for cat, name in
                  ((0, "deposit_gather"), (1, "deposit_stage"), (2, "lsrk_stage"), (3, "sort"),
                   (6, "deposit_normalize"))}
        return float(t), kernel

    ms64, kernel64 = timed("fp64")
    ms, kernel = timed("mixed")
    clk = clocks.stop()
    m.check_status()
    value = world * n * args.steps / (ms * 1e-3)
    value64 = world * n * args.steps / (ms64 * 1e-3)

    # ---- end to end: host buffers through the same API (chosen form) ----
    # Every step copies its particle state in from pinned host memory and its
    # rho, j out to pinned host memory. The copies run on a second stream and
    # overlap the neighbouring steps' compute: two device particle stores
    # alternate (step k computes in one while step k+1's inputs upload into
    # the other), the result of step k downloads while step k+1 computes.
    e2e = None
    if not args.no_e2e:
        from pyrticle_b200.cloud import PicState
        hx = torch.empty_like(s.x, device="cpu").pin_memory()
        hp = torch.empty_like(s.p, device="cpu").pin_memory()
        hq = torch.empty_like(s.q, device="cpu").pin_memory()
        hm = torch.empty_like(s.m, device="cpu").pin_memory()
        he = torch.empty_like(s.el, device="cpu").pin_memory()
        hx.copy_(s.x)
        hp.copy_(s.p)
        hq.copy_(s.q)
        hm.copy_(s.m)
        he.copy_(s.el)
        stores = [s, PicState(m, x=torch.empty_like(s.x), p=torch.empty_like(s.p),
                              q=torch.empty_like(s.q), m=torch.empty_like(s.m),
                              el=torch.empty_like(s.el), ids=s.ids.clone())]
        hrho = [torch.empty((nn,), dtype=torch.float64).pin_memory() for _ in range(2)]
        hj = [torch.empty((3, nn), dtype=torch.float64).pin_memory() for _ in range(2)]
        comp = torch.cuda.current_stream()
        copy = torch.cuda.Stream()
        up = [torch.cuda.Event() for _ in range(2)]
        done = [torch.cuda.Event() for _ in range(2)]

        def upload(st, k):
            with torch.cuda.stream(copy):
                st.x.copy_(hx, non_blocking=True)
                st.p.copy_(hp, non_blocking=True)
                st.q.copy_(hq, non_blocking=True)
                st.m.copy_(hm, non_blocking=True)
                st.el.copy_(he, non_blocking=True)
                up[k].record(copy)

        def one_step_on(st):
            m.depositor.precision = "mixed"
            try:
                if world > 1:
                    m.step(st, fields, w.dt, steps=1, deposit=False, check=False, precision=1)
                    return deposit_densities_exact(m, st)
                rho, j = m.step(st, fields, w.dt, steps=1, check=False, precision=1)
            finally:
                m.depositor.precision = "fp64"
            return rho, j

        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(comp)
        copy.wait_event(f0)
        upload(stores[0], 0)
        keep = []
        for k in range(args.steps):
            cur, nxt = k % 2, (k + 1) % 2
            # the next step's inputs are enqueued before this step (the
            # normalising depositor's statistics make each step wait for
            # itself on the host), into the store the previous step used
            if k + 1 < args.steps:
                if k >= 1:
                    copy.wait_event(done[nxt])  # the store's previous step is done
                upload(stores[nxt], nxt)
            comp.wait_event(up[cur])
            rho, j = one_step_on(stores[cur])
            done[cur].record(comp)
            keep.append((rho, j))
            with torch.cuda.stream(copy):
                copy.wait_event(done[cur])
                hrho[cur].copy_(rho, non_blocking=True)
                hj[cur].copy_(j, non_blocking=True)
        comp.wait_stream(copy)
        f1.record(comp)
        torch.cuda.synchronize()
        ems = f0.elapsed_time(f1)
        if world > 1:
            ems = max_over_ranks(ems, "cuda")
        e2e = {"value": world * n * args.steps / (ems * 1e-3), "unit": METRIC,
               "h2d_bytes_per_step": int(n * (24 + 24 + 8 + 8 + 4)),
               "d2h_bytes_per_step": int(nn * 4 * 8),
               "pipelining": "copies on a second stream overlap the neighbouring steps "
                             "(two alternating device particle stores)"}
        del stores, keep

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return

    peaks, src = measured_peaks()
    fp64 = fp64_peak_tflops(torch)
    fp32 = fp32_peak_tflops(torch)
    bf16 = float(peaks.get("bf16_tflops", 1590.0))
    # chosen form: the tensor-core deposition (tc_deposit_kernel), two passes
    # of the same tile kernel: the normalising integrals, then the deposition
    gms, gk = kernel["deposit_gather"]
    avg_gather = gms / max(gk, 1)
    nms, nk = kernel["deposit_normalize"]
    avg_norm = nms / max(nk, 1)
    # executed tensor work per evaluated (position, particle) pair in dense
    # FP16 equivalents: the score, 2 x 16 (kind::f16, K = 16); the sums,
    # 3 weight digits x 16 columns x 2 int8 ops counted at half (the int8
    # rate is twice the FP16 rate)
    tensor_per_pair = 32 + 48
    achieved = tensor_per_pair * evaluated_tc / (avg_gather * 1e-3) / 1e12
    useful = 15.0 * pairs / (avg_gather * 1e-3) / 1e12
    gms64, gk64 = kernel64["deposit_gather"]
    avg_gather64 = gms64 / max(gk64, 1)
    achieved64 = 15.0 * pairs / (avg_gather64 * 1e-3) / 1e12
    sms, sk = kernel["lsrk_stage"]
    stage_gbs = 216.0 * n / (sms / max(sk, 1) * 1e-3) / 1e9
    algorithmic = (f"15 flops x {pairs} (particle, distinct node position) pairs within the "
                   f"radius per launch ({node_pairs} (particle, node) pairs over all DG nodes; "
                   f"coincident nodes are evaluated once; {evaluated} pairs evaluated after "
                   f"culling)")
    roofline = {"bound": "tensor",
                "kernel": "tc_deposit_kernel (deposition pass, chosen form)",
                "achieved": achieved, "peak": bf16, "unit": "TFLOP/s", "frac": achieved / bf16,
                "traffic": measured_traffic(args, "tc_deposit_kernel<0, 0>"),
                "traffic_normalize_pass": measured_traffic(args, "tc_deposit_kernel<1, 1>"),
                "peak_source": ("MEASURED_PEAKS.json bf16_tflops" if src == "measured" else
                                "fallback 1,590 TFLOP/s (dense BF16, this pool)"),
                "algorithmic": (f"{tensor_per_pair} dense-FP16-equivalent tensor flops per "
                                f"evaluated (position, particle) pair x {evaluated_tc} evaluated "
                                f"pairs per launch (128 tile rows x candidates); {pairs} pairs "
                                f"within the radius; {avg_gather:.3f} ms per launch"),
                "evaluated_per_useful_pair": evaluated_tc / max(pairs, 1),
                "useful_pairs_per_s": pairs / (avg_gather * 1e-3),
                "useful_fp32_equivalent": {
                    "achieved": useful, "peak": fp32, "unit": "TFLOP/s", "frac": useful / fp32,
                    "note": "15 flops per pair within the radius against the FP32 CUDA-core "
                            "rate (cuBLAS SGEMM, TF32 off, measured in this run): the work "
                            "the CUDA-core form of this deposition does per pair"},
                "normalize_pass_ms": avg_norm,
                "secondary": {"bound": "hbm", "kernel": "lsrk_stage_mixed_kernel<3>",
                              "achieved": stage_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                              "frac": stage_gbs / peaks["hbm_gbs"],
                              "traffic": measured_traffic(args, "lsrk_stage_mixed_kernel<3>"),
                              "algorithmic": "216 B per particle per stage",
                              "peak_source": src}}
    fp64_block = {
        "value": value64, "unit": METRIC, "ms_per_step": ms64 / args.steps,
        "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kernel64.items()},
        "roofline": {"bound": "fp64", "kernel": "deposit_groups_kernel (deposition, FP64)",
                     "achieved": achieved64, "peak": fp64, "unit": "TFLOP/s",
                     "frac": achieved64 / fp64,
                     "traffic": measured_traffic(args, "deposit_groups_kernel<1, 1, 2>"),
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                     "algorithmic": algorithmic + f"; {avg_gather64:.3f} ms per launch"},
        "form": ("plain form: FP64 throughout" +
                 ("; NormalizedShapeFunctionDepositor: FP64 integral and scale per particle"
                  if args.depositor == "normalized" else ""))}
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f16/i8 tensor + f32 + f64 (mixed: split-FP16 tensor-core shape scores, "
                     "23-bit integer weights (three digits) summed exactly on the int8 tensor cores, FP64 "
                     "per-node combine and normalisation; split-BF16 tensor-core Lagrange "
                     "values; FP64 state/force/locate)",
            "data": "synthetic (seeded mesh, particles and fields of the workload)",
            "config": {"workload": f"{args.workload}: {w.mesh.element_count} tets order "
                                   f"{w.order}, {n} particles/GPU, shape radius "
                                   f"{w.shape_radius * 100:g} cm, chosen (mixed) form, "
                                   f"{'Normalized' if args.depositor == 'normalized' else ''}"
                                   f"ShapeFunctionDepositor",
                       "particles_per_gpu": n, "elements": w.mesh.element_count,
                       "nodes": nn, "order": w.order, "form": "mixed",
                       "depositor": args.depositor,
                       "l2": f"inputs larger than L2 ({216 * n / 1e9:.1f} GB particle state per stage)",
                       "parallelism": f"particles sharded over {world} GPU(s) (z slabs of "
                                      "the beam), NCCL all-reduce of the integer digit sums "
                                      "per node position" if world > 1 else "1 GPU"},
            "clocks": clk, "gpu_launches": None, "roofline": roofline,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kernel.items()},
            "pairs_per_deposition": {"positions": pairs, "nodes": node_pairs,
                                     "evaluated_fp64_kernel": evaluated,
                                     "evaluated_tensor_core_kernel": evaluated_tc},
            "fp64": fp64_block, "speedup_mixed_vs_fp64": ms64 / ms,
            "accuracy_mixed_vs_fp64": accuracy}
    # libprt's own kernels in the timed region of the headline form (CUB's
    # radix-sort kernels not counted): per sort iota + 5 permutation gathers
    # (x, p, q, m, ids; the residuals are dead at a step boundary); per RK
    # stage one fused kernel; per deposition bin keys, bin starts, payload,
    # the tile work estimate, charges, charge scale, charge digits, the
    # deposition pass and the expansion to nodes (9), and with the
    # normalising depositor position weights, their maximum, scale and
    # digits, the normalisation pass and the two statistics kernels (7).
    per_dep = 9 + (7 if args.depositor == "normalized" else 0)
    line["gpu_launches"] = int(kernel["lsrk_stage"][1] + per_dep * kernel["deposit_gather"][1] +
                               6 * kernel["sort"][1])
    if e2e:
        line["e2e"] = e2e
    if not args.no_adjoint and world == 1:
        line["adjoint"] = adjoint_bench(torch, args.adjoint_scale, peaks["hbm_gbs"])
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(w, args.cpu_seconds)
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
