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
PCG (Chebyshev(4) on D^-1 A) and of the chosen forms (FP32 applies inside FP64
reliable updates, affine-compressed quadrature data, the learned coarse
correction), for 128^3 Q2 and 64^3 Q3.

The JSON line carries summaries; the full record (per-form iteration counts,
autotuner table, heat, batch, tet details) goes to --detail (default
gpurun_out/bench_detail.json when that folder exists).

--impl reference times the reference's algorithm (the oracle port of
crates/assembly/src/partial.rs's element loop with the Hex8 isoparametric
Jacobian) on the host cores, on the same full mesh as the GPU arm.

Multi-GPU (--mode): "sharded" (the default for N > 1) splits ONE global
problem into z slabs, one per rank: a step is one sharded apply (local apply
+ halo sum of the interface planes over NCCL), value = global DOFs x steps /
max-over-ranks time (strong scaling), plus a sharded Jacobi-PCG solve to
1e-8 with the vector work in the library's kernels.  "replicas" (the default
for N = 1) runs one independent instance per rank (weak scaling).
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


def host_threads():
    """Host threads this process may run on (the CPU baseline uses all of
    them, whatever OMP_NUM_THREADS a launcher such as torchrun has set)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def bench_config(n, p, world):
    """The workload description shared by both arms of the bench."""
    N = (n * p + 1) ** 3
    return {"workload": f"{n}^3 Q{p} unit-cube hex, FP64 PA diffusion apply (constrained), {N} DOFs per rank",
            "order": p, "n_elem_1d": n,
            "l2": "inputs larger than L2 (qdata %.2f GB per apply)" % (6 * (p + 1) ** 3 * n ** 3 * 8 / 1e9),
            "parallelism": f"{world} independent instances"}


def dirichlet_rhs(n, p):
    """Load of the scale-up configuration: M sin(pi x) sin(pi y) sin(pi z) with
    the Dirichlet rows zeroed."""
    import femgpu
    from femgpu.fields import sin_nodal

    mass = femgpu.PAMassOperator((n, n, n), p)
    b = mass.matvec(sin_nodal(n, n, n, p))
    mass.close()
    s = n * p + 1
    bb = b.reshape(s, s, s)
    bb[0], bb[-1], bb[:, 0], bb[:, -1], bb[:, :, 0], bb[:, :, -1] = 0, 0, 0, 0, 0, 0
    return b


# ---------------------------------------------------------------------------
# CPU legs (the oracle port of the reference algorithm; outside every timed
# GPU region)
# ---------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_apply_time(n, p, kq, reps):
    """Seconds per oracle apply on the full mesh, all host threads."""
    O = _oracle()
    mesh = O.Mesh(n, n, n, p)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    x = np.random.default_rng(1).standard_normal(mesh.ndofs)
    y = np.zeros(mesh.ndofs)
    cores = host_threads()
    O.pa_apply(mesh, coef, x, y, nthreads=cores)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    return (time.perf_counter() - t0) / reps, mesh.ndofs, cores


def cpu_solve_extrapolated(n, p, kq, gpu_iterations, t_apply):
    """Time to 1e-8 of the reference algorithm's Chebyshev(4)-PCG on the host
    cores, extrapolated: the per-iteration time measured over 2 iterations of
    the oracle's PCG on the full mesh (difference of 3 and 1 iterations, so
    set-up cancels), times the GPU plain solve's iteration count, plus the 20
    power-iteration applies of the lambda_max estimate at the measured apply
    time."""
    O = _oracle()
    mesh = O.Mesh(n, n, n, p)
    coef = O.Coef(O.DIFF, kappa_q=kq)
    mask = O.ess_mask(mesh)
    b = dirichlet_rhs(n, p)
    cores = host_threads()
    lm = 1.0  # any bounds: the iteration cost does not depend on them
    ts = []
    for k in (1, 3):
        t0 = time.perf_counter()
        O.pcg(mesh, coef, mask, b, precond=2, cheb_degree=4, lmin=lm / 30, lmax=lm, rtol=1e-30,
              max_iter=k, nthreads=cores)
        ts.append(time.perf_counter() - t0)
    t_iter = max(ts[1] - ts[0], 0.0) / 2
    total = 20 * t_apply + gpu_iterations * t_iter
    return {"kind": "extrapolated", "t_iter_s": t_iter, "t_apply_s": t_apply, "iterations": gpu_iterations,
            "time_to_1e8_s": total, "cores": cores,
            "method": "oracle Chebyshev(4)-PCG (par_solver.rs:262-342 loop) per-iteration time on the full "
                      "mesh x the GPU plain FP64 iteration count + 20 lambda_max applies"}


def cpu_ex1_pipeline(n=24):
    """The mfem_ex1 pipeline through the oracle port on the host cores: source
    form, PCG-Jacobi to rtol 1e-10, L2 error (24^3 Q1 Poisson)."""
    O = _oracle()
    cores = host_threads()
    t0 = time.perf_counter()
    mesh = O.Mesh(n, n, n, 1)
    mask = O.ess_mask(mesh)
    b = O.source(mesh, mask)
    x, info = O.pcg(mesh, O.Coef(O.DIFF), mask, b, precond=1, rtol=1e-10, max_iter=2000, nthreads=cores)
    err = O.l2_error_sin(mesh, x, nq=3)
    return {"pipeline_s": time.perf_counter() - t0, "iterations": info["iterations"], "l2_error": err,
            "threads": cores}


def run_reference(args, n, p):
    """The reference arm: the oracle port of the reference PA element loop on
    the host cores, on the GPU arm's full mesh and kappa (seed 0).  If the
    warm-up shows that --steps full applies would take longer than about four
    minutes, each step is a z-slab of the mesh instead (stated in `sample`)."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from femgpu.fields import lognormal_kappa_q

    O = _oracle()
    kq_full = lognormal_kappa_q(n, n, n, p, seed=0)
    cores = host_threads()
    q3 = (p + 1) ** 3

    def setup(nz):
        kq = kq_full if nz == n else np.ascontiguousarray(kq_full[: n * n * nz * q3])
        mesh = O.Mesh(n, n, nz, p)
        coef = O.Coef(O.DIFF, kappa_q=kq)
        x = np.random.default_rng(1).standard_normal(mesh.ndofs)
        return mesh, coef, x, np.zeros(mesh.ndofs)

    nzs = n
    mesh, coef, x, y = setup(nzs)
    t0 = time.perf_counter()
    for _ in range(args.warmup):
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    t_w = (time.perf_counter() - t0) / max(args.warmup, 1)
    if t_w * args.steps > 240.0:
        nzs = max(1, int(n * 240.0 / (t_w * args.steps)))
        mesh, coef, x, y = setup(nzs)
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.pa_apply(mesh, coef, x, y, nthreads=cores)
    dt = time.perf_counter() - t0
    val = mesh.ndofs * args.steps / dt / 1e9
    sample = (f"the full {n}^3 Q{p} mesh ({mesh.ndofs} DOFs) per step" if nzs == n else
              f"{n}x{n}x{nzs} Q{p} z-slab ({mesh.ndofs} DOFs) per step (full-mesh steps would exceed 4 min)")
    out = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "GDOF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: lognormal kappa GRF (sigma2=1, ell=0.1, seed 0) at Gauss points, x ~ N(0,1)",
        "config": bench_config(n, p, world),
        "cpu_baseline": {"value": val, "unit": "GDOF/s", "cores": cores, "kind": "port",
                         "sample": f"{sample}, OpenMP {cores} threads; the reference (Rust) cannot be built "
                                   "here, so this is the C restatement of its algorithm"},
        "e2e": {"value": val, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# GPU sections
# ---------------------------------------------------------------------------
def learned_weights(n, p):
    return os.path.join(ROOT, "fem-rs_b200", "femgpu", "weights", f"unet_q{p}_{n}.npz")


def run_solves(op, n, p, kq, rank):
    """Time to FP64 true relative residual 1e-8 for every form on one operator.
    Returns (summary, detail)."""
    import femgpu

    b = dirichlet_rhs(n, p)
    N = op.n_dofs()
    detail = {}
    x_plain = None
    runs = (("plain_fp64_chebyshev4", femgpu.PC_CHEBYSHEV, femgpu.FP64, femgpu.QDATA_FULL),
            ("plain_fp64_jacobi", femgpu.PC_JACOBI, femgpu.FP64, femgpu.QDATA_FULL),
            ("fp32_ir_chebyshev4", femgpu.PC_CHEBYSHEV, femgpu.FP32_IR, femgpu.QDATA_FULL),
            ("plain_fp64_chebyshev4_affine", femgpu.PC_CHEBYSHEV, femgpu.FP64, femgpu.QDATA_AFFINE),
            ("fp32_ir_chebyshev4_affine", femgpu.PC_CHEBYSHEV, femgpu.FP32_IR, femgpu.QDATA_AFFINE))
    for name, pc, prec, fmt in runs:
        op.set_qdata_format(fmt)
        xs = np.zeros(N)
        r = op.pcg(b, xs, femgpu.SolverConfig(rtol=1e-8, max_iter=20000, cheb_degree=4, precision=prec), pc)
        if x_plain is None:
            x_plain = xs.copy()
        detail[name] = {"iterations": r.iterations, "reliable_updates": r.outer_iterations if prec else 0,
                        "solve_s": r.solve_ms / 1e3, "true_residual": r.true_residual, "converged": r.converged,
                        "applies": r.applies, "lmax": r.lmax if pc == femgpu.PC_CHEBYSHEV else None,
                        "rel_err_vs_plain_fp64": float(np.linalg.norm(xs - x_plain) / np.linalg.norm(x_plain))}
    op.set_qdata_format(femgpu.QDATA_FULL)

    # learned coarse correction (flexible CG, z = Chebyshev(r) + network
    # correction) with the committed weights trained for this mesh and order on
    # other kappa seeds; budget = the plain iteration count of the same form
    wpath = learned_weights(n, p)
    if os.path.exists(wpath):
        from femgpu import learned as learned_mod
        net, meta = learned_mod.load(wpath)
        if meta["first_seed"] <= rank < meta["first_seed"] + meta["train_fields"]:
            detail["learned_skipped"] = f"kappa seed {rank} is a training seed of {os.path.basename(wpath)}"
        else:
            femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n, p), int(meta["levels"]))
            femgpu.attach_unet(op, net)
            for name, prec, fmt, plain_key in (
                    ("learned_fp64_chebyshev4", femgpu.FP64, femgpu.QDATA_FULL, "plain_fp64_chebyshev4"),
                    ("learned_fp32_ir_chebyshev4", femgpu.FP32_IR, femgpu.QDATA_FULL, "fp32_ir_chebyshev4"),
                    ("learned_fp32_ir_chebyshev4_affine", femgpu.FP32_IR, femgpu.QDATA_AFFINE,
                     "fp32_ir_chebyshev4_affine")):
                op.set_qdata_format(fmt)
                xs = np.zeros(N)
                cfg = femgpu.SolverConfig(rtol=1e-8, max_iter=20000, cheb_degree=4, precision=prec,
                                          nn_budget=detail[plain_key]["iterations"],
                                          nn_iter_ratio=float(meta.get("iter_ratio", 0.0)))
                r = op.pcg(b, xs, cfg, femgpu.PC_CHEB_NN)
                detail[name] = {
                    "iterations": r.iterations, "solve_s": r.solve_ms / 1e3, "true_residual": r.true_residual,
                    "converged": r.converged, "nn_fallback": r.extra["nn_fallback"],
                    "iterations_of_plain_same_form": detail[plain_key]["iterations"],
                    "rel_err_vs_plain_fp64": float(np.linalg.norm(xs - x_plain) / np.linalg.norm(x_plain))}
            femgpu.attach_unet(op, None)
            op.set_qdata_format(femgpu.QDATA_FULL)
            detail["learned_weights"] = {"file": os.path.relpath(wpath, ROOT), "levels": meta["levels"],
                                         "train_fields": meta["train_fields"], "first_seed": meta["first_seed"],
                                         "params": meta["params"]}
        del net

    plain = detail["plain_fp64_chebyshev4"]["solve_s"]
    short = {"plain_fp64_chebyshev4": "plain", "plain_fp64_jacobi": "plain_jacobi", "fp32_ir_chebyshev4": "fp32",
             "plain_fp64_chebyshev4_affine": "fp64_affine", "fp32_ir_chebyshev4_affine": "fp32_affine",
             "learned_fp64_chebyshev4": "nn_fp64", "learned_fp32_ir_chebyshev4": "nn_fp32",
             "learned_fp32_ir_chebyshev4_affine": "nn_fp32_affine"}
    summary = {"dofs": N}
    for k, s in short.items():
        if k in detail:
            d = detail[k]
            summary[s] = [round(d["solve_s"], 4), d["iterations"]]
    summary["max_rel_err_vs_plain"] = max(d["rel_err_vs_plain_fp64"] for k, d in detail.items() if k in short)
    summary["all_converged"] = all(d["converged"] for k, d in detail.items() if k in short)
    sp = {}
    for k, s in short.items():
        if k in detail and s != "plain":
            sp[s] = round(plain / detail[k]["solve_s"], 3)
    if "learned_fp32_ir_chebyshev4" in detail:
        # like-for-like: learned vs plain in the same precision and qdata format
        sp["nn_fp32_vs_fp32"] = round(detail["fp32_ir_chebyshev4"]["solve_s"]
                                      / detail["learned_fp32_ir_chebyshev4"]["solve_s"], 3)
        sp["nn_fp32_affine_vs_fp32_affine"] = round(
            detail["fp32_ir_chebyshev4_affine"]["solve_s"] / detail["learned_fp32_ir_chebyshev4_affine"]["solve_s"], 3)
    summary["speedup_vs_plain"] = sp
    summary["format"] = "[solve_s, iterations]; plain = drop-in FP64 Chebyshev(4) PCG on full qdata"
    return summary, detail


def time_apply_variants(op, n, p, x, steps, peak, stream):
    """FP64 / FP32 applies on the full and the affine-compressed quadrature
    data, CUDA events on the launching stream."""
    import torch

    import femgpu

    x32 = x.float()
    y = torch.zeros_like(x)
    y32 = torch.zeros_like(x32)

    def time_apply(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(steps):
            fn()
        g1.record(stream)
        torch.cuda.synchronize()
        return g0.elapsed_time(g1) / steps

    E, q3, N = n ** 3, (p + 1) ** 3, op.n_dofs()
    out = {}
    for fmt, tag in ((femgpu.QDATA_FULL, "full"), (femgpu.QDATA_AFFINE, "affine")):
        op.set_qdata_format(fmt)
        for prec, es in (("fp64", 8), ("fp32", 4)):
            if prec == "fp64":
                t = time_apply(lambda: op.apply_native(x.data_ptr(), y.data_ptr()))
            else:
                t = time_apply(lambda: op.apply_native_f32(x32.data_ptr(), y32.data_ptr()))
            qbytes = (6 * q3 * E if tag == "full" else (6 + q3) * E) * es
            nbytes = qbytes + 2 * N * es
            out[f"{prec}_{tag}"] = {"ms": round(t, 5), "gdof_s": round(N / (t / 1e3) / 1e9, 3),
                                    "frac": round(nbytes / (t / 1e3) / 1e9 / peak, 4)}
    op.set_qdata_format(femgpu.QDATA_FULL)
    return out


def run_heat(rank, steps, stream):
    """SDIRK-2 heat stepping, 64^3 Q2, lognormal kappa, dt = 1e-3, u0 = sin sin sin."""
    import femgpu
    from femgpu.fields import lognormal_kappa_q

    hn, hp, dt = 64, 2, 1e-3
    hk = lognormal_kappa_q(hn, hn, hn, hp, sigma2=1.0, ell=0.1, seed=rank)
    K = femgpu.PADiffusionOperator((hn, hn, hn), hp, kappa=hk)
    S = femgpu.PAMassDiffusionOperator((hn, hn, hn), hp, 1.0, femgpu.SDIRK2_GAMMA * dt, kappa=hk)
    K.set_stream(stream.cuda_stream)
    S.set_stream(stream.cuda_stream)
    xs1 = np.linspace(0, 1, hn * hp + 1)
    u0 = (np.sin(np.pi * xs1)[:, None, None] * np.sin(np.pi * xs1)[None, :, None]
          * np.sin(np.pi * xs1)[None, None, :])
    u0[[0, -1]], u0[:, [0, -1]], u0[:, :, [0, -1]] = 0.0, 0.0, 0.0
    u0 = u0.ravel()
    detail = {"workload": f"{hn}^3 Q2 SDIRK-2, dt={dt}, {steps} steps, stage rtol 1e-10, warm start"}
    finals = {}
    for name, prec, fmt in (("fp64", femgpu.FP64, femgpu.QDATA_FULL),
                            ("fp32", femgpu.FP32_IR, femgpu.QDATA_FULL),
                            ("fp32_affine", femgpu.FP32_IR, femgpu.QDATA_AFFINE)):
        K.set_qdata_format(fmt)
        S.set_qdata_format(fmt)
        u = u0.copy()
        info = femgpu.sdirk2(K, S, u, dt, steps, femgpu.SolverConfig(rtol=1e-10, max_iter=5000, precision=prec),
                             femgpu.PC_CHEBYSHEV)
        finals[name] = u
        detail[name] = {"time_s": info["time_ms"] / 1e3, "stage_iterations": info["total_iterations"],
                        "max_stage_iterations": info["max_stage_iterations"], "applies": info["applies"]}
    ref = finals["fp64"]
    for name in finals:
        detail[name]["rel_l2_diff_vs_fp64"] = float(np.linalg.norm(finals[name] - ref) / np.linalg.norm(ref))
    K.close()
    S.close()
    summary = {k: [round(detail[k]["time_s"], 3), detail[k]["stage_iterations"], detail[k]["rel_l2_diff_vs_fp64"]]
               for k in ("fp64", "fp32", "fp32_affine")}
    summary["format"] = "[time_s, stage_iterations, rel_l2_diff_vs_fp64]"
    summary["speedup_fp32_affine"] = round(detail["fp64"]["time_s"] / detail["fp32_affine"]["time_s"], 3)
    return summary, detail


def measure_pcie(nbytes, dev, reps=5):
    """Pinned host <-> device copy bandwidth (GB/s) for buffers of `nbytes`:
    host-to-device alone, device-to-host alone, and both at once on two
    streams (total bytes of both directions / time), CUDA events."""
    import torch

    n = nbytes // 8
    hs = torch.empty(n, dtype=torch.float64).pin_memory()
    hd = torch.empty(n, dtype=torch.float64).pin_memory()
    d_in = torch.empty(n, dtype=torch.float64, device=dev)
    d_out = torch.zeros(n, dtype=torch.float64, device=dev)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def timed(fn_list):
        for _ in range(2):
            for st, fn in fn_list:
                with torch.cuda.stream(st):
                    fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in fn_list]
        start = torch.cuda.Event(enable_timing=True)
        start.record(fn_list[0][0])
        for (st, fn), (a, b) in zip(fn_list, ev):
            st.wait_event(start)
            a.record(st)
            with torch.cuda.stream(st):
                for _ in range(reps):
                    fn()
            b.record(st)
        torch.cuda.synchronize()
        return max(start.elapsed_time(b) for _, b in ev) / 1e3

    h2d = lambda: d_in.copy_(hs, non_blocking=True)
    d2h = lambda: hd.copy_(d_out, non_blocking=True)
    t_h = timed([(s1, h2d)])
    t_d = timed([(s2, d2h)])
    t_b = timed([(s1, h2d), (s2, d2h)])
    return {"h2d_gbs": round(nbytes * reps / t_h / 1e9, 2), "d2h_gbs": round(nbytes * reps / t_d / 1e9, 2),
            "both_directions_gbs": round(2 * nbytes * reps / t_b / 1e9, 2), "bytes": int(nbytes)}


def run_batch(rank, batch_n, dev):
    """256 uneven solves, n ~ U{8..48}, p ~ U{1,2,3}, own lognormal kappa
    (sigma2 ~ U[0.25,2], ell ~ U[0.05,0.3]) and RHS M xi, FP32 mixed precision.
    Sequential and batched with the default tiles and full quadrature data,
    then the autotuner's (format, tile) per group, sequential and batched again;
    iterations are compared between the two tuned runs."""
    import femgpu
    from femgpu.fields import lognormal_kappa_q

    brng = np.random.default_rng(7000 + rank)
    bops, bbs = [], []
    total = 0
    t_setup = time.perf_counter()
    for i in range(batch_n):
        bn, bp = int(brng.integers(8, 49)), int(brng.integers(1, 4))
        kq = lognormal_kappa_q(bn, bn, bn, bp, sigma2=float(brng.uniform(0.25, 2.0)),
                               ell=float(brng.uniform(0.05, 0.3)), seed=100000 * rank + i, device=dev)
        o = femgpu.PADiffusionOperator((bn, bn, bn), bp, kappa=kq)
        m = femgpu.PAMassOperator((bn, bn, bn), bp)
        bb = m.matvec(brng.standard_normal(o.n_dofs()))
        m.close()
        bb3 = bb.reshape(o.NK, o.NJ, o.NI)
        bb3[[0, -1]], bb3[:, [0, -1]], bb3[:, :, [0, -1]] = 0.0, 0.0, 0.0
        bops.append(o)
        bbs.append(bb)
        total += o.n_dofs()
    t_setup = time.perf_counter() - t_setup
    cfgb = femgpu.SolverConfig(rtol=1e-8, max_iter=5000, precision=femgpu.FP32_IR, check_interval=10)

    def sequential():
        t, its = 0.0, []
        for o, v in zip(bops, bbs):
            r1 = o.pcg(v, np.zeros_like(v), cfgb, femgpu.PC_CHEBYSHEV)
            t += r1.solve_ms / 1e3
            its.append(r1.iterations)
        return t, its

    t_seq0, seq_iters = sequential()  # default tiles
    bxs = [np.zeros_like(v) for v in bbs]
    ok0, bres0 = femgpu.batch_pcg(bops, bbs, bxs, cfgb, femgpu.PC_CHEBYSHEV)
    t_batch0 = bres0[0].solve_ms / 1e3
    t_tune = time.perf_counter()
    tune = femgpu.batch_autotune(bops, reps=3)
    t_tune = time.perf_counter() - t_tune
    t_seq, seq_iters = sequential()  # tuned tiles and formats: the batching gain alone
    bxs = [np.zeros_like(v) for v in bbs]
    ok, bres = femgpu.batch_pcg(bops, bbs, bxs, cfgb, femgpu.PC_CHEBYSHEV)
    t_batch = bres[0].solve_ms / 1e3
    dof_its = sum(int(o.n_dofs()) * int(r.iterations) for o, r in zip(bops, bres))
    for o in bops:
        o.close()
    summary = {"instances": len(bops), "total_dofs": total, "all_converged": bool(ok and ok0),
               "max_true_residual": max(r.true_residual for r in bres),
               "iterations_min_max": [min(r.iterations for r in bres), max(r.iterations for r in bres)],
               "max_iteration_diff_vs_single": int(max(abs(a.iterations - b) for a, b in zip(bres, seq_iters))),
               "sequential_default_tiles_s": round(t_seq0, 3), "sequential_tuned_tiles_s": round(t_seq, 3),
               "batched_default_tiles_s": round(t_batch0, 3), "batched_tuned_s": round(t_batch, 3),
               "speedup_batching_same_tiles": round(t_seq / t_batch, 3),
               "speedup_autotune_batched": round(t_batch0 / t_batch, 3),
               "affine_groups": sum(e["format"] == femgpu.QDATA_AFFINE for e in tune), "groups": len(tune)}
    detail = dict(summary, setup_s=t_setup, autotune_s=t_tune,
                  dof_iterations=dof_its, dof_iterations_per_s=dof_its / t_batch,
                  autotune=[{"order": e["order"], "size_class": e["size_class"], "instances": e["instances"],
                             "format": "affine" if e["format"] == femgpu.QDATA_AFFINE else "full", "tz": e["tz"],
                             "us_per_candidate_tz": e["us"], "us_other_format": e["us_other"]} for e in tune])
    return summary, detail


def run_tet(dev, peak):
    """Tetrahedral PA apply (TetP1/TetP2 on unit_cube_tet, partial.rs on Tet4)."""
    import torch

    import femgpu
    from femgpu import tet as tetmesh

    out = {}
    for tn, tp in ((64, 2), (96, 1)):
        coords, dofs, nd, mask = tetmesh.unit_cube_space(tn, tp)
        top = femgpu.TetOperator(tp, coords, dofs, nd, quad_order=2 * tp, ess=mask)
        xt = torch.randn(nd, dtype=torch.float64, device=dev)
        yt = torch.zeros_like(xt)
        stream = torch.cuda.current_stream(dev)
        top.set_stream(stream.cuda_stream)
        for _ in range(3):
            top.apply_native(xt.data_ptr(), yt.data_ptr())
        torch.cuda.synchronize()
        reps = 20
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(reps):
            top.apply_native(xt.data_ptr(), yt.data_ptr())
        g1.record(stream)
        torch.cuda.synchronize()
        top.check()
        dt = g0.elapsed_time(g1) / 1e3 / reps
        E, nl, nqt = dofs.shape[0], dofs.shape[1], top.nq
        # algorithmic bytes of the diffusion apply in the moment form: element map (int32), geometry G
        # (6 doubles), diffusion moments (10 doubles for P2, 1 for P1), x read once, y written once;
        # the point form would read nq point scalars instead of the moments
        nmom = 10 if tp == 2 else 1
        ab = E * (nl * 4 + 6 * 8 + nmom * 8) + nd * (8 + 8)
        ab_pt = E * (nl * 4 + 6 * 8 + nqt * 8) + nd * (8 + 8)
        out[f"p{tp}_n{tn}"] = {"elements": int(E), "dofs": int(nd), "points": int(nqt), "ms": round(dt * 1e3, 4),
                               "gdof_s": round(nd / dt / 1e9, 3), "frac_algorithmic": round(ab / dt / 1e9 / peak, 4),
                               "point_form_bytes_per_s_frac": round(ab_pt / dt / 1e9 / peak, 4)}
        top.close()
        del xt, yt
    out["timing"] = ("CUDA events over 20 asynchronous applies (chunk kernel + shared-DOF kernel each); "
                     "diffusion in the moment form")
    return out


def box_as_hex_mesh(n, p):
    """The unit-cube n^3 box of order p handed over as an unstructured Hex8 mesh:
    node coordinates, HexQ1-ordered connectivity and tensor-order element DOF
    maps (order 1: DOF = node), in lexicographic element order."""
    m = n + 1
    k, j, i = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    coords = np.stack([i / n, j / n, k / n], axis=-1).reshape(-1, 3)
    ez, ey, ex = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    conn = np.stack([((ez + c) * m + ey + b) * m + ex + a for a, b, c in corners], axis=1).astype(np.uint32)
    if p == 1:
        return coords, conn, None
    s = n * p + 1
    q = p + 1
    loc = [(a, b, c) for c in range(q) for b in range(q) for a in range(q)]
    maps = np.stack([((ez * p + c) * s + ey * p + b) * s + ex * p + a for a, b, c in loc], axis=1).astype(np.uint32)
    return coords, conn, maps


def run_hex_unstructured(n, p, kq, steps, peak, dev):
    """The same operator as the headline apply built through the unstructured
    Hex8 constructor (the drop-in for a caller's own mesh and DofManager
    numbering; chunked scatter), against the structured fast path."""
    import torch

    import femgpu

    coords, conn, maps = box_as_hex_mesh(n, p)
    N = (n * p + 1) ** 3
    sn = n * p + 1
    ids = np.arange(N).reshape(sn, sn, sn)
    ess = np.unique(np.concatenate([ids[[0, -1]].ravel(), ids[:, [0, -1]].ravel(), ids[:, :, [0, -1]].ravel()]))
    t0 = time.perf_counter()
    op = femgpu.HexMeshOperator(p, coords, conn, elem_dofs=maps, n_dofs=N, kappa=kq.reshape(n ** 3, -1),
                                ess_dofs=ess.astype(np.uint32))
    t_setup = time.perf_counter() - t0
    stream = torch.cuda.current_stream(dev)
    op.set_stream(stream.cuda_stream)
    x = torch.from_numpy(op.to_native(np.random.default_rng(3).standard_normal(N))).to(dev)
    y = torch.zeros_like(x)
    for _ in range(3):
        op.apply_native(x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(steps):
        op.apply_native(x.data_ptr(), y.data_ptr())
    g1.record(stream)
    torch.cuda.synchronize()
    op.check()
    ms = g0.elapsed_time(g1) / steps
    E, q3 = n ** 3, (p + 1) ** 3
    nbytes = 6 * q3 * E * 8 + q3 * E * 4 + 2 * N * 8  # qdata + element map + x, y
    out = {"ms": round(ms, 4), "gdof_s": round(N / (ms / 1e3) / 1e9, 3), "frac": round(nbytes / (ms / 1e3) / 1e9 / peak, 4),
           "chunks": op.chunks, "setup_s": round(t_setup, 2)}
    op.close()
    return out


def run_ex1():
    """mfem_ex1 on 24^3 Q1: source form, PCG-Jacobi rtol 1e-10, L2 error, on the GPU."""
    import torch

    import femgpu

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
    op1.close()
    return {"iterations": r1.iterations, "l2_error": err1, "pipeline_s": round(t_ex1, 4),
            "converged": r1.converged}


def run_sharded(args, n, p, world, rank, local, dev):
    """One global n^3 Q{p} problem over all ranks (z slabs): the sharded apply
    as the step, and a sharded Jacobi-PCG solve to 1e-8 (the solve of
    crates/parallel/src/par_solver.rs:262-342)."""
    import torch
    import torch.distributed as dist

    from femgpu import SolverConfig
    from femgpu import sharded as S
    from femgpu.fields import lognormal_kappa_q

    comm = S.TorchComm() if world > 1 else S.ThreadGroup(1).comm(0)
    kq = lognormal_kappa_q(n, n, n, p, sigma2=1.0, ell=0.1, seed=0)  # one global field
    A = S.ShardedPAOperator(comm, (n, n, n), p, kappa=kq)
    del kq
    stream = torch.cuda.current_stream(dev)
    N = (n * p + 1) ** 3
    x = A.scatter(np.random.default_rng(1000).standard_normal(N))
    y = A.zeros()

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        A.apply(x, y)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        A.apply(x, y)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1), world, dev)
    value = N * args.steps / (t_ms / 1e3) / 1e9
    # e2e: the rank's slab vector from pinned host memory, apply, result back
    xh = x.cpu().pin_memory()
    yh = torch.zeros_like(xh).pin_memory()
    k_e2e = max(3, min(args.steps, 20))
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        x.copy_(xh, non_blocking=True)
        A.apply(x, y)
        yh.copy_(y, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize()
    te_ms = max_over_ranks(f0.elapsed_time(f1), world, dev)
    solve = None
    if not args.no_solve:
        b = A.scatter(dirichlet_rhs(n, p))
        xs = A.zeros()
        barrier()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        res = S.par_solve_pcg_jacobi(A, b, xs, SolverConfig(rtol=1e-8, max_iter=5000))
        s1.record(stream)
        torch.cuda.synchronize()
        t_s = max_over_ranks(s0.elapsed_time(s1), world, dev) / 1e3
        solve = {"jacobi_pcg_s": t_s, "iterations": res.iterations, "converged": res.converged,
                 "final_residual": res.final_residual}
    bytes_canon, _ = canonical_bytes(n, p)
    peak, peak_kind = measured_peak()
    achieved = bytes_canon / world / (t_ms / 1e3 / args.steps) / 1e9  # per GPU
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "GDOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: one lognormal kappa GRF (sigma2=1, ell=0.1, seed 0) at Gauss points, x ~ N(0,1)",
            "config": {"workload": f"{n}^3 Q{p} unit-cube hex, FP64 PA diffusion apply (constrained), {N} DOFs "
                                   f"split into {world} z slabs", "order": p, "n_elem_1d": n,
                       "l2": "inputs larger than L2 (qdata %.2f GB over all ranks)" % (6 * (p + 1) ** 3 * n ** 3 * 8 / 1e9),
                       "parallelism": f"sharded over {world} ranks: slab apply + halo sum of the interface planes"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": peak_kind,
                         "kernel": "per-rank pa_apply_kernel + fixup_kernel + plane exchange (per-GPU share of the "
                                   "canonical bytes)"},
            "e2e": {"value": N * k_e2e / (te_ms / 1e3) / 1e9, "unit": "GDOF/s",
                    "h2d_bytes_per_step": int(xh.numel() * 8 * world), "d2h_bytes_per_step": int(yh.numel() * 8 * world),
                    "steps": k_e2e},
            "gpu_launches": 2 * args.steps, "clocks": clk, "cpu_baseline": None, "sharded_solve": solve,
        }
        print(json.dumps(out), flush=True)
    A.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="q2_128", choices=sorted(WORKLOADS))
    ap.add_argument("--detail", default=None, help="file for the full record (default: gpurun_out/bench_detail.json "
                                                   "if that folder exists)")
    for opt in ("solve", "q3", "cpu", "heat", "batch", "tet", "ex1", "hex"):
        ap.add_argument(f"--no-{opt}", action="store_true")
    ap.add_argument("--mode", default=None, choices=["replicas", "sharded"],
                    help="multi-GPU form (default: replicas for 1 GPU, sharded for more)")
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
    from femgpu.fields import lognormal_kappa_q

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    mode = args.mode or ("sharded" if world > 1 else "replicas")
    if mode == "sharded":
        run_sharded(args, n, p, world, rank, local, dev)
        if world > 1:
            dist.destroy_process_group()
        return

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
    te_ms = max_over_ranks(f0.elapsed_time(f1), world, dev)
    e2e_val = whole_job_gdofs(world, N, k_e2e, te_ms)
    _ = float(yh[0])
    # the PCIe ceiling of the e2e step: N doubles each way, both directions at once
    pcie = measure_pcie(N * 8, dev)
    e2e_ideal_ms = 2 * N * 8 / (pcie["both_directions_gbs"] * 1e9) * 1e3

    detail = {}
    variants = time_apply_variants(op, n, p, x, args.steps, peak, stream)
    solve = None
    if not args.no_solve:
        solve = {}
        solve[args.workload], detail["solve_" + args.workload] = run_solves(op, n, p, kq, rank)
    del x, y

    # the 64^3 Q3 configuration beside the headline mesh: applies and solves
    q3 = None
    if not args.no_q3 and (n, p) == (128, 2):
        qn, qp = WORKLOADS["q3_64"]
        kq3 = lognormal_kappa_q(qn, qn, qn, qp, sigma2=1.0, ell=0.1, seed=rank)
        op3 = femgpu.PADiffusionOperator((qn, qn, qn), qp, kappa=kq3)
        op3.set_stream(stream.cuda_stream)
        x3 = torch.from_numpy(op3.to_native(gen.standard_normal(op3.n_dofs()))).to(dev)
        q3 = {"apply": time_apply_variants(op3, qn, qp, x3, args.steps, peak, stream)}
        del x3
        if solve is not None:
            solve["q3_64"], detail["solve_q3_64"] = run_solves(op3, qn, qp, kq3, rank)
        op3.close()
        del kq3

    hexu = None if args.no_hex else run_hex_unstructured(n, p, kq, args.steps, peak, dev)

    heat = None
    if not args.no_heat:
        heat, detail["heat"] = run_heat(rank, args.heat_steps, stream)
    batch = None
    if not args.no_batch:
        batch, detail["batch"] = run_batch(rank, args.batch_n, dev)
    tet = None if args.no_tet else run_tet(dev, peak)
    ex1 = None if args.no_ex1 else run_ex1()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            t_apply, ndof, cores = cpu_apply_time(n, p, kq, reps=2)
            cpu = {"value": ndof / t_apply / 1e9, "unit": "GDOF/s", "cores": cores, "kind": "port",
                   "sample": f"oracle port of the reference PA element loop (partial.rs:154-208 + "
                             f"assembler.rs:96-143) on the full {n}^3 Q{p} mesh ({ndof} DOFs), 2 applies, "
                             f"OpenMP {cores} threads"}
            if solve is not None:
                gpu_it = detail["solve_" + args.workload]["plain_fp64_chebyshev4"]["iterations"]
                ext = cpu_solve_extrapolated(n, p, kq, gpu_it, t_apply)
                cpu["time_to_1e8_s_extrapolated"] = ext["time_to_1e8_s"]
                cpu["time_to_1e8_vs_gpu_plain"] = ext["time_to_1e8_s"] / (
                    detail["solve_" + args.workload]["plain_fp64_chebyshev4"]["solve_s"])
                detail["cpu_solve_extrapolated"] = ext
            if ex1 is not None:
                cpu["ex1_pipeline_s"] = cpu_ex1_pipeline()["pipeline_s"]
        except Exception as exc:  # keep the bench line even if the oracle is unavailable
            cpu = {"value": None, "unit": "GDOF/s", "cores": host_threads(), "kind": "port",
                   "sample": f"unavailable: {exc}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "GDOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: lognormal kappa GRF (sigma2=1, ell=0.1, seed=rank) at Gauss points, x ~ N(0,1)",
            "config": bench_config(n, p, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": tr, "peak_kind": peak_kind,
                         "bytes_per_apply_canonical": bytes_canon,
                         "frac_no_map": bytes_nomap / per_apply_s / 1e9 / peak,
                         "kernel": "pa_apply_kernel + fixup_kernel (timed together per apply)"},
            "e2e": {"value": e2e_val, "unit": "GDOF/s", "h2d_bytes_per_step": N * 8, "d2h_bytes_per_step": N * 8,
                    "steps": k_e2e, "ms_per_step": te_ms / k_e2e, "pcie": pcie,
                    "pcie_bound_ms": e2e_ideal_ms, "frac_of_pcie": e2e_ideal_ms / (te_ms / k_e2e)},
            "gpu_launches": launches_per_apply * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
            "solve": solve,
            "apply": variants,
            "q3_64": q3,
            "hex_unstructured": hexu,
            "heat": heat,
            "batch": batch,
            "tet": tet,
            "ex1": ex1,
        }
        print(json.dumps(out), flush=True)
        path = args.detail
        if path is None and os.path.isdir(os.path.join(ROOT, "gpurun_out")):
            path = os.path.join(ROOT, "gpurun_out", "bench_detail.json")
        if path:
            with open(path, "w") as f:
                json.dump(dict(out, detail=detail), f, indent=1)
    op.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
