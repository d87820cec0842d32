"""Benchmark of the matrix-free PA operator path on B200.

Default workload (N=1): the scale-up configuration 128^3 Q2 hex mesh on the
unit cube (257^3 = 16,974,593 DOFs, 3^3 Gauss points), lognormal kappa
(sigma^2 = 1, correlation length 0.1, seeded), FP64.

A step is one application of the constrained FP64 PA diffusion operator
(y = A x, sum-factorised apply + deterministic scatter) to a device-resident
vector; `value` is whole-job GDOF/s (DOFs of all ranks x steps / max-over-ranks
device time).  `e2e` is the same metric through the public C ABI call
(fg_op_apply on pinned host buffers: H2D copy of x, apply, D2H copy of y each
step).  `solve` reports time to FP64 true relative residual 1e-8 of plain FP64
PCG (Chebyshev(4) on D^-1 A, and Jacobi).

--impl reference times the reference's algorithm (the oracle port of
crates/assembly/src/partial.rs's element loop with the Hex8 isoparametric
Jacobian) on the host cores, on a z-slab sample of the same workload.

Multi-GPU: one independent instance per rank (its own seeded kappa), no
data-path collective; scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "fem-rs_b200"))

METRIC = "time to 1e-8 FP64 residual & PA GDOF/s on 1 B200: chosen vs plain FP64 PCG"
WORKLOADS = {
    # name: (n elements per direction, order)
    "q2_128": (128, 2),  # 128^3 Q2, 17.0M DOFs (headline)
    "q3_64": (64, 3),    # 64^3 Q3, 7.2M DOFs
    "q1_128": (128, 1),  # 128^3 Q1, 2.15M DOFs
    "q2_64": (64, 2),    # 64^3 Q2, 2.15M DOFs (profiling case, qdata 340 MB > L2)
}


def canonical_bytes(n, p):
    """Algorithmic bytes of one FP64 diffusion apply: 6 symmetric qdata
    components per quadrature point, an int32 element-to-DOF map, x read and
    y written once."""
    E = n ** 3
    q3 = (p + 1) ** 3
    N = (n * p + 1) ** 3
    return 6 * q3 * E * 8 + q3 * E * 4 + 2 * N * 8, 6 * q3 * E * 8 + 2 * N * 8


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(name):
    """Per-launch DRAM bytes of the apply kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch_full_size:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
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
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [s.strip() for s in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value, world, device):
    """Max of a per-rank float over all ranks (timings are reported as the
    slowest rank's); the identity on one rank."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gdofs(world, n_dofs, steps, t_ms):
    """Whole-job throughput: every rank applies its own instance `steps` times."""
    return world * n_dofs * steps / (t_ms / 1e3) / 1e9


def cpu_apply_sample(n, p, kq_full, reps=2, layers=None):
    """Oracle (reference-algorithm port) apply on a z-slab of the workload, all
    host threads.  Returns (GDOF/s, threads, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nzs = layers or max(1, n // 8)
    q3 = (p + 1) ** 3
    kq = np.ascontiguousarray(kq_full[: n * n * nzs * q3])
    mesh = O.Mesh(n, n, nzs, p)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    x = np.random.default_rng(1).standard_normal(mesh.ndofs)
    y = np.zeros(mesh.ndofs)
    cores = host_threads()
    O.pa_apply(mesh, coef, x, y, nthreads=cores)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    dt = (time.perf_counter() - t0) / reps
    desc = (f"oracle port of the reference PA element loop (partial.rs:154-208 + assembler.rs:96-143), "
            f"{n}x{n}x{nzs} Q{p} z-slab of the workload ({mesh.ndofs} DOFs), {reps} applies, "
            f"OpenMP {cores} threads")
    return mesh.ndofs / dt / 1e9, cores, desc


def cpu_ex1_pipeline(n=24):
    """The mfem_ex1 pipeline through the oracle port on the host cores: source
    form, PCG-Jacobi to rtol 1e-10, L2 error (24^3 Q1 Poisson)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cores = host_threads()
    t0 = time.perf_counter()
    mesh = O.Mesh(n, n, n, 1)
    mask = O.ess_mask(mesh)
    b = O.source(mesh, mask)
    x, info = O.pcg(mesh, O.Coef(O.DIFF), mask, b, precond=1, rtol=1e-10, max_iter=2000, nthreads=cores)
    err = O.l2_error_sin(mesh, x, nq=3)
    return {"pipeline_s": time.perf_counter() - t0, "iterations": info["iterations"], "l2_error": err,
            "threads": cores}


def host_threads():
    """Host threads this process may run on (the CPU baseline uses all of
    them, whatever OMP_NUM_THREADS a launcher such as torchrun has set)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, n, p):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from femgpu.fields import lognormal_kappa_q

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nzs = max(1, n // 32)
    q3 = (p + 1) ** 3
    kq = lognormal_kappa_q(n, n, n, p, seed=0)[: n * n * nzs * q3].copy()
    mesh = O.Mesh(n, n, nzs, p)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    x = np.random.default_rng(1).standard_normal(mesh.ndofs)
    y = np.zeros(mesh.ndofs)
    cores = host_threads()
    for _ in range(args.warmup):
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    dt = time.perf_counter() - t0
    val = mesh.ndofs * args.steps / dt / 1e9
    out = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "GDOF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: lognormal kappa GRF (sigma2=1, ell=0.1, seed 0) at Gauss points, x ~ N(0,1)",
        "config": {"workload": f"{n}^3 Q{p} FP64 PA diffusion apply (sample: {n}x{n}x{nzs} z-slab)",
                   "order": p, "n_elem_1d": n, "l2": "inputs larger than L2 not applicable on CPU"},
        "cpu_baseline": {"value": val, "unit": "GDOF/s", "cores": cores, "kind": "port",
                         "sample": f"{n}x{n}x{nzs} Q{p} z-slab ({mesh.ndofs} DOFs) per step, OpenMP {cores} threads; "
                                   "the reference (Rust) cannot be built here, so this is the C restatement of its algorithm"},
        "e2e": {"value": val, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="q2_128", choices=sorted(WORKLOADS))
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-heat", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-tet", action="store_true")
    ap.add_argument("--no-ex1", action="store_true")
    ap.add_argument("--batch-n", type=int, default=256)
    ap.add_argument("--heat-steps", type=int, default=500)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    n, p = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, n, p)
        return

    import torch
    import torch.distributed as dist

    import femgpu
    from femgpu.fields import lognormal_kappa_q, sin_nodal

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    kq = lognormal_kappa_q(n, n, n, p, sigma2=1.0, ell=0.1, seed=rank)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    stream = torch.cuda.current_stream(dev)
    op.set_stream(stream.cuda_stream)
    N = op.n_dofs()
    gen = np.random.default_rng(1000 + rank)
    x = torch.from_numpy(op.to_native(gen.standard_normal(N))).to(dev)
    y = torch.zeros_like(x)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        op.apply_native(x.data_ptr(), y.data_ptr(), accumulate=False, constrained=True)
    torch.cuda.synchronize()
    op.check()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        op.apply_native(x.data_ptr(), y.data_ptr(), accumulate=False, constrained=True)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    t_ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    t_ms = max_over_ranks(t_ms, world, dev)
    op.check()
    per_apply_s = t_ms / 1e3 / args.steps
    value = whole_job_gdofs(world, N, args.steps, t_ms)
    bytes_canon, bytes_nomap = canonical_bytes(n, p)
    peak, peak_kind = measured_peak()
    achieved = bytes_canon / per_apply_s / 1e9
    tr = profile_traffic("pa_apply_fp64_q2_64.txt") if (n, p) == (128, 2) else None
    launches_per_apply = 2 if (op.nx > 32 or op.ny > 4 or op.nz > 1) else 1

    # e2e through the public C ABI with pinned host buffers
    xh = torch.from_numpy(gen.standard_normal(N)).pin_memory()
    yh = torch.zeros(N, dtype=torch.float64).pin_memory()
    k_e2e = max(3, min(args.steps, 20))
    for _ in range(2):
        op.apply_zero(xh, yh, constrained=True)
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        op.apply_zero(xh, yh, constrained=True)
    f1.record(stream)
    torch.cuda.synchronize()
    te_ms = f0.elapsed_time(f1)
    te_ms = max_over_ranks(te_ms, world, dev)
    e2e_val = whole_job_gdofs(world, N, k_e2e, te_ms)
    _ = float(yh[0])

    solve = None
    if not args.no_solve:
        solve = {}
        mass = femgpu.PAMassOperator((n, n, n), p)
        mass.set_stream(stream.cuda_stream)
        b = np.zeros(N)
        mass.apply_zero(sin_nodal(n, n, n, p), b, constrained=False)
        # homogeneous Dirichlet: zero boundary rows of the RHS
        bb = b.reshape(op.NK, op.NJ, op.NI)
        bb[0], bb[-1], bb[:, 0], bb[:, -1], bb[:, :, 0], bb[:, :, -1] = 0, 0, 0, 0, 0, 0
        mass.close()
        runs = (("plain_fp64_chebyshev4", femgpu.PC_CHEBYSHEV, femgpu.FP64),
                ("plain_fp64_jacobi", femgpu.PC_JACOBI, femgpu.FP64),
                ("fp32_ir_chebyshev4", femgpu.PC_CHEBYSHEV, femgpu.FP32_IR),
                ("fp32_ir_jacobi", femgpu.PC_JACOBI, femgpu.FP32_IR))
        x_plain = None
        for fmt, suffix in ((femgpu.QDATA_FULL, ""), (femgpu.QDATA_AFFINE, "_affine")):
            op.set_qdata_format(fmt)
            for name, pc, prec in runs:
                xs = np.zeros(N)
                cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=20000, cheb_degree=4, precision=prec)
                r = op.pcg(b, xs, cfg, pc)
                if x_plain is None:
                    x_plain = xs.copy()
                solve[name + suffix] = {
                    "iterations": r.iterations, "reliable_updates": r.outer_iterations if prec else 0,
                    "solve_s": r.solve_ms / 1e3, "true_residual": r.true_residual, "converged": r.converged,
                    "applies": r.applies, "lmax": r.lmax if pc == femgpu.PC_CHEBYSHEV else None,
                    "rel_err_vs_plain_fp64_chebyshev": float(np.linalg.norm(xs - x_plain) / np.linalg.norm(x_plain))}
        op.set_qdata_format(femgpu.QDATA_FULL)

        def best(keys):
            return min(solve[k]["solve_s"] for k in keys)
        plain = best(["plain_fp64_chebyshev4", "plain_fp64_jacobi"])
        solve["speedup"] = {
            "fp32_vs_plain_same_full_qdata": plain / best(["fp32_ir_chebyshev4", "fp32_ir_jacobi"]),
            "fp32_affine_vs_plain_full_qdata": plain / best(["fp32_ir_chebyshev4_affine", "fp32_ir_jacobi_affine"]),
            "fp32_affine_vs_plain_affine": best(["plain_fp64_chebyshev4_affine", "plain_fp64_jacobi_affine"])
            / best(["fp32_ir_chebyshev4_affine", "fp32_ir_jacobi_affine"]),
            "note": "plain = drop-in FP64 PCG with the full (general-geometry) quadrature data; "
                    "_affine = compressed qdata valid for constant-J elements, reported as such"}

        # learned coarse correction (flexible CG, z = Chebyshev(r) + network
        # correction) with the committed weights trained for this mesh and order
        # on other kappa seeds; budget = the plain iteration count of the same
        # form, beyond which the solve falls back to plain Chebyshev-PCG
        wpath = os.path.join(ROOT, "fem-rs_b200", "femgpu", "weights", f"unet_q{p}_{n}.npz")
        meta = None
        if os.path.exists(wpath):
            from femgpu import learned as learned_mod
            net, meta = learned_mod.load(wpath)
            if meta["first_seed"] <= rank < meta["first_seed"] + meta["train_fields"]:
                # this rank's kappa seed was a training field: no held-out number
                solve["learned_skipped"] = f"kappa seed {rank} is among the training seeds of {os.path.basename(wpath)}"
                meta = None
        if meta is not None:
            femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n, p), int(meta["levels"]))
            femgpu.attach_unet(op, net)
            for name, prec, fmt, plain_key in (
                    ("learned_fp64_chebyshev4", femgpu.FP64, femgpu.QDATA_FULL, "plain_fp64_chebyshev4"),
                    ("learned_fp32_ir_chebyshev4_affine", femgpu.FP32_IR, femgpu.QDATA_AFFINE,
                     "fp32_ir_chebyshev4_affine")):
                op.set_qdata_format(fmt)
                xs = np.zeros(N)
                cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=20000, cheb_degree=4, precision=prec,
                                          nn_budget=solve[plain_key]["iterations"])
                r = op.pcg(b, xs, cfg, femgpu.PC_CHEB_NN)
                solve[name] = {
                    "iterations": r.iterations, "solve_s": r.solve_ms / 1e3, "true_residual": r.true_residual,
                    "converged": r.converged, "nn_fallback": r.extra["nn_fallback"],
                    "iterations_of_plain_same_form": solve[plain_key]["iterations"],
                    "rel_err_vs_plain_fp64_chebyshev": float(np.linalg.norm(xs - x_plain) / np.linalg.norm(x_plain))}
            femgpu.attach_unet(op, None)
            op.set_qdata_format(femgpu.QDATA_FULL)
            solve["learned_weights"] = {"file": os.path.relpath(wpath, ROOT), "levels": meta["levels"],
                                        "train_fields": meta["train_fields"], "first_seed": meta["first_seed"],
                                        "params": meta["params"]}
            solve["speedup"]["learned_fp64_vs_plain_fp64"] = plain / solve["learned_fp64_chebyshev4"]["solve_s"]
            solve["speedup"]["learned_fp32_affine_vs_plain_fp64"] = (
                plain / solve["learned_fp32_ir_chebyshev4_affine"]["solve_s"])
            del net

    # FP32 apply throughput (chosen precision form) and the affine-compressed
    # format, same workload
    x32 = x.float()
    y32 = torch.zeros_like(x32)

    def time_apply(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            fn()
        g1.record(stream)
        torch.cuda.synchronize()
        return g0.elapsed_time(g1) / args.steps

    E = n ** 3
    q3 = (p + 1) ** 3
    variants = {}
    for fmt, tag in ((femgpu.QDATA_FULL, "full"), (femgpu.QDATA_AFFINE, "affine")):
        op.set_qdata_format(fmt)
        for prec, es in (("fp64", 8), ("fp32", 4)):
            if prec == "fp64":
                t = time_apply(lambda: op.apply_native(x.data_ptr(), y.data_ptr()))
            else:
                t = time_apply(lambda: op.apply_native_f32(x32.data_ptr(), y32.data_ptr()))
            qbytes = (6 * q3 * E if tag == "full" else (6 + q3) * E) * es
            nbytes = qbytes + 2 * N * es
            variants[f"{prec}_{tag}"] = {"ms": t, "gdof_s": N / (t / 1e3) / 1e9, "bytes_per_apply": nbytes,
                                         "achieved_gbs": nbytes / (t / 1e3) / 1e9,
                                         "frac": nbytes / (t / 1e3) / 1e9 / peak}
    op.set_qdata_format(femgpu.QDATA_FULL)
    fp32_apply = variants

    # SDIRK-2 heat stepping, 64^3 Q2, lognormal kappa, dt = 1e-3,
    # u0 = sin sin sin; FP64 stage solves vs FP32 (reliable-update) stage solves
    heat = None
    if not args.no_heat:
        hn, hp, dt = 64, 2, 1e-3
        hk = lognormal_kappa_q(hn, hn, hn, hp, sigma2=1.0, ell=0.1, seed=rank)
        K = femgpu.PADiffusionOperator((hn, hn, hn), hp, kappa=hk)
        S = femgpu.PAMassDiffusionOperator((hn, hn, hn), hp, 1.0, femgpu.SDIRK2_GAMMA * dt, kappa=hk)
        K.set_stream(stream.cuda_stream)
        S.set_stream(stream.cuda_stream)
        xs1 = np.linspace(0, 1, hn * hp + 1)
        u0 = (np.sin(np.pi * xs1)[:, None, None] * np.sin(np.pi * xs1)[None, :, None]
              * np.sin(np.pi * xs1)[None, None, :]).ravel()
        u0.reshape(hn * hp + 1, hn * hp + 1, hn * hp + 1)[[0, -1], :, :] = 0.0
        u0.reshape(hn * hp + 1, hn * hp + 1, hn * hp + 1)[:, [0, -1], :] = 0.0
        u0.reshape(hn * hp + 1, hn * hp + 1, hn * hp + 1)[:, :, [0, -1]] = 0.0
        heat = {"workload": f"{hn}^3 Q2 SDIRK-2, dt={dt}, {args.heat_steps} steps, stage rtol 1e-10, warm start"}
        finals = {}
        # _affine: the quadrature data of both operators in the affine-compressed
        # format (constant-J elements: |detJ| J^-1 J^-T per element, kappa per point)
        for name, prec, pc, fmt in (("fp64_chebyshev4", femgpu.FP64, femgpu.PC_CHEBYSHEV, femgpu.QDATA_FULL),
                                    ("fp32_chebyshev4", femgpu.FP32_IR, femgpu.PC_CHEBYSHEV, femgpu.QDATA_FULL),
                                    ("fp32_chebyshev4_affine", femgpu.FP32_IR, femgpu.PC_CHEBYSHEV,
                                     femgpu.QDATA_AFFINE)):
            K.set_qdata_format(fmt)
            S.set_qdata_format(fmt)
            u = u0.copy()
            info = femgpu.sdirk2(K, S, u, dt, args.heat_steps,
                                 femgpu.SolverConfig(rtol=1e-10, max_iter=5000, precision=prec), pc)
            finals[name] = u
            heat[name] = {"time_s": info["time_ms"] / 1e3, "stage_iterations": info["total_iterations"],
                          "max_stage_iterations": info["max_stage_iterations"], "applies": info["applies"]}
        ref = finals["fp64_chebyshev4"]
        for name in finals:
            heat[name]["rel_l2_diff_vs_fp64_chebyshev"] = float(np.linalg.norm(finals[name] - ref) / np.linalg.norm(ref))
        K.close()
        S.close()

    # batched uneven solves, n ~ U{8..48}, p ~ U{1,2,3}, own lognormal
    # kappa (sigma2 ~ U[0.25,2], ell ~ U[0.05,0.3]) and RHS M xi, FP32 mixed precision
    batch = None
    if not args.no_batch:
        brng = np.random.default_rng(7000 + rank)
        bops, bbs = [], []
        total = 0
        t_setup = time.perf_counter()
        for i in range(args.batch_n):
            bn, bp = int(brng.integers(8, 49)), int(brng.integers(1, 4))
            kq = lognormal_kappa_q(bn, bn, bn, bp, sigma2=float(brng.uniform(0.25, 2.0)),
                                   ell=float(brng.uniform(0.05, 0.3)), seed=100000 * rank + i, device=dev)
            o = femgpu.PADiffusionOperator((bn, bn, bn), bp, kappa=kq)
            m = femgpu.PAMassOperator((bn, bn, bn), bp)
            xi = brng.standard_normal(o.n_dofs())
            bb = m.matvec(xi)
            m.close()
            bb3 = bb.reshape(o.NK, o.NJ, o.NI)
            bb3[[0, -1]] = 0.0
            bb3[:, [0, -1]] = 0.0
            bb3[:, :, [0, -1]] = 0.0
            bops.append(o)
            bbs.append(bb)
            total += o.n_dofs()
        t_setup = time.perf_counter() - t_setup
        cfgb = femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR, check_interval=10)
        # the same solves one after another (single-instance launches, default tiles)
        t_seq = 0.0
        seq_iters = []
        for o, v in zip(bops, bbs):
            xs1 = np.zeros_like(v)
            r1 = o.pcg(v, xs1, cfgb, femgpu.PC_CHEBYSHEV)
            t_seq += r1.solve_ms / 1e3
            seq_iters.append(r1.iterations)
        # batched with the default tiles
        bxs = [np.zeros_like(v) for v in bbs]
        ok0, bres0 = femgpu.batch_pcg(bops, bbs, bxs, cfgb, femgpu.PC_CHEBYSHEV)
        t_batch0 = bres0[0].solve_ms / 1e3
        # autotuner: item depth per (order, size class) from timed batched applies
        t_tune = time.perf_counter()
        tune = femgpu.batch_autotune(bops, reps=3)
        t_tune = time.perf_counter() - t_tune
        bxs = [np.zeros_like(v) for v in bbs]
        ok, bres = femgpu.batch_pcg(bops, bbs, bxs, cfgb, femgpu.PC_CHEBYSHEV)
        t_batch = bres[0].solve_ms / 1e3
        batch = {"instances": len(bops), "total_dofs": total, "all_converged": bool(ok and ok0),
                 "max_true_residual": max(r.true_residual for r in bres),
                 "iterations_min_max": [min(r.iterations for r in bres), max(r.iterations for r in bres)],
                 "max_iteration_diff_vs_single": int(max(abs(a.iterations - b) for a, b in zip(bres, seq_iters))),
                 "sequential_single_solves_s": t_seq, "batched_default_tiles_s": t_batch0,
                 "batched_solve_s": t_batch, "speedup_batched_vs_sequential": t_seq / t_batch,
                 "speedup_autotune": t_batch0 / t_batch,
                 "dof_iterations_per_s": sum(o.n_dofs() * r.iterations for o, r in zip(bops, bres)) / t_batch,
                 "setup_s": t_setup, "autotune_s": t_tune,
                 "autotune": [{"order": e["order"], "size_class": e["size_class"], "instances": e["instances"],
                               "tz": e["tz"], "us_per_candidate_tz": e["us"]} for e in tune]}
        for o in bops:
            o.close()

    # tetrahedral PA apply (TetP1/TetP2 on unit_cube_tet, partial.rs on Tet4):
    # element gather + per-point contraction + CSR transpose scatter
    tet = None
    if not args.no_tet:
        from femgpu import tet as tetmesh
        tet = {}
        for tn, tp in ((64, 2), (96, 1)):
            coords, dofs, nd, mask = tetmesh.unit_cube_space(tn, tp)
            qo = 2 * tp
            top = femgpu.TetOperator(tp, coords, dofs, nd, quad_order=qo, ess=mask)
            xt = torch.randn(nd, dtype=torch.float64, device=dev)
            yt = torch.zeros_like(xt)
            for _ in range(3):
                top.apply_zero(xt, yt, True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            reps = 20
            for _ in range(reps):
                top.apply_zero(xt, yt, True)
            torch.cuda.synchronize()
            dt = (time.perf_counter() - t0) / reps
            E, nl, nqt = dofs.shape[0], dofs.shape[1], top.nq
            # element map + geometry + per-point scalars + local results (write, read) + slots; offsets, x, y
            tb = E * (nl * 4 + 6 * 8 + nqt * 8 + 2 * nl * 8 + nl * 4) + nd * (8 + 8 + 8)
            tet[f"p{tp}_n{tn}"] = {"elements": int(E), "dofs": int(nd), "ms_per_apply": dt * 1e3,
                                   "gdof_s": nd / dt / 1e9, "bytes_per_apply": int(tb),
                                   "achieved_gbs": tb / dt / 1e9, "frac": tb / dt / 1e9 / peak,
                                   "timing": "host wall clock over 20 synchronised applies"}
            top.close()
            del xt, yt

    # the mfem_ex1 pipeline on the 24^3 Q1 Poisson case (kappa = 1, f = 3 pi^2 sin sin sin,
    # homogeneous Dirichlet, PCG-Jacobi, rtol 1e-10): source form, solve and L2 error on the GPU
    ex1 = None
    if not args.no_ex1:
        n1 = 24
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        op1 = femgpu.PADiffusionOperator((n1, n1, n1), 1)
        qp2 = femgpu.quadrature_points(n1, n1, n1, 2)
        b1 = femgpu.assemble_source(n1, n1, n1, 1, 3 * np.pi ** 2 * np.prod(np.sin(np.pi * qp2), axis=-1))
        x1 = np.zeros(op1.n_dofs())
        r1 = femgpu.solve_pcg_jacobi(op1, b1, x1, femgpu.SolverConfig(rtol=1e-10, max_iter=2000))
        qp3 = femgpu.quadrature_points(n1, n1, n1, 3)
        err1 = femgpu.l2_error(n1, n1, n1, 1, x1, np.prod(np.sin(np.pi * qp3), axis=-1), nq=3)
        t_ex1 = time.perf_counter() - t0
        ex1 = {"workload": "mfem_ex1: 24^3 Q1 Poisson, PCG-Jacobi rtol 1e-10 (15,625 DOFs)",
               "iterations": r1.iterations, "solve_ms": r1.solve_ms, "l2_error": err1,
               "pipeline_s": t_ex1, "converged": r1.converged,
               "timing": "host wall clock: operator setup, source form, solve, L2 error"}
        op1.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            v, cores, desc = cpu_apply_sample(n, p, kq)
            cpu = {"value": v, "unit": "GDOF/s", "cores": cores, "kind": "port", "sample": desc}
            if ex1 is not None:
                cpu["ex1_pipeline"] = cpu_ex1_pipeline()
        except Exception as exc:  # keep the bench line even if the oracle is unavailable
            cpu = {"value": None, "unit": "GDOF/s", "cores": host_threads(), "kind": "port",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "GDOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: lognormal kappa GRF (sigma2=1, ell=0.1, seed=rank) at Gauss points, x ~ N(0,1)",
            "config": {"workload": f"{n}^3 Q{p} unit-cube hex, FP64 PA diffusion apply (constrained), "
                                   f"{N} DOFs per rank", "order": p, "n_elem_1d": n,
                       "l2": "inputs larger than L2 (qdata %.2f GB per apply)" % (6 * (p + 1) ** 3 * n ** 3 * 8 / 1e9),
                       "parallelism": f"{world} independent instances"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": tr,
                         "bytes_per_apply_canonical": bytes_canon, "bytes_per_apply_no_map": bytes_nomap,
                         "frac_no_map": bytes_nomap / per_apply_s / 1e9 / peak, "peak_kind": peak_kind,
                         "kernel": "pa_apply_kernel + fixup_kernel (timed together per apply)"},
            "e2e": {"value": e2e_val, "unit": "GDOF/s", "h2d_bytes_per_step": N * 8, "d2h_bytes_per_step": N * 8,
                    "steps": k_e2e},
            "gpu_launches": launches_per_apply * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
            "solve": solve,
            "apply_variants": fp32_apply,
            "heat": heat,
            "batch": batch,
            "tet": tet,
            "ex1": ex1,
        }
        print(json.dumps(out), flush=True)
    op.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
