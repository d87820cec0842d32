"""Training and evaluation of the learned coarse correction.

Problem family: -div(kappa grad u) = b on the unit cube, 128^3 Q1 hexahedra
(129^3 DOFs), homogeneous Dirichlet on all faces, kappa = exp(g) with g a
Gaussian random field (sigma^2 = 1, correlation length 0.1) drawn per seed,
b = M xi with xi i.i.d. N(0,1) nodal values (zero on the boundary).

Training data: the recurrence residuals r_k of plain Chebyshev(4)-PCG from
x0 = 0 on each training field, every `every` iterations
(fg_op_collect_residuals).  Loss: the energy functional of the correction
c = s 8^L P^L UNet(R^L r / s, R^L log kappa),  s = rms(R^L r),
    (c.Ac/2 - c.r) / (s^2 64^L Nc),
minimised by the Galerkin coarse correction on range(P^L); its gradient is
computed by the library's FP64 operator and the network's hand-written BF16
backward pass (fg_unet_train_energy), followed by Adam.  Fields are streamed:
each is solved once, trained on for a few steps, then dropped.

Evaluation: flexible CG with z = Chebyshev(r) + correction against plain
Chebyshev-PCG on held-out fields, both to the FP64 true relative residual
1e-8; the learned solve gets the plain iteration count as its budget and
falls back to plain Chebyshev-PCG beyond it.

The same procedure trains the correction for Q2 operators (--p 2): the DOF
lattice of equispaced Q2 nodes is uniform, so the network volume is that
lattice coarsened `levels` times (128^3 Q2: 257^3 -> 33^3 with levels 3).

Run on a GPU:  python -m femgpu.learned --out fem-rs_b200/femgpu/weights/unet_q1_128.npz
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import femgpu
from femgpu.fields import lognormal_kappa_q

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "unet_q1_128.npz")


def make_problem(n, seed, levels=2, p=1, rhs="random", device="cuda"):
    """Operator with a seeded lognormal kappa and its RHS: M xi (xi ~ N(0,1)
    nodal values) or M sin(pi x) sin(pi y) sin(pi z); zero on the boundary."""
    from femgpu.fields import sin_nodal

    kq = lognormal_kappa_q(n, n, n, p, sigma2=1.0, ell=0.1, seed=seed, device=device)
    op = femgpu.PADiffusionOperator((n, n, n), p, kappa=kq)
    femgpu.set_nodal_kappa(op, femgpu.nodal_kappa_from_q(kq, n, n, n, p), levels)
    del kq
    m = femgpu.PAMassOperator((n, n, n), p)
    if rhs == "sin":
        b = m.matvec(sin_nodal(n, n, n, p))
    else:
        rng = np.random.default_rng(10_000 + seed)
        b = m.matvec(rng.standard_normal(op.n_dofs()))
    m.close()
    b3 = b.reshape(op.NK, op.NJ, op.NI)
    b3[[0, -1]] = 0.0
    b3[:, [0, -1]] = 0.0
    b3[:, :, [0, -1]] = 0.0
    return op, b


def train(net, n, seeds, levels=2, every=2, max_res=48, steps_per_field=10, batch=4,
          lr0=2e-3, lr1=1e-4, log=print, log_every=20, p=1):
    import torch

    g = torch.Generator(device="cpu")
    g.manual_seed(0)
    total = len(seeds) * steps_per_field
    hist = []
    t0 = time.perf_counter()
    it = 0
    for i, s in enumerate(seeds):
        op, b = make_problem(n, s, levels, p)
        res = femgpu.collect_residuals(op, b, every, max_res)
        for _ in range(steps_per_field):
            idx = torch.randperm(res.shape[0], generator=g)[:batch].to(res.device)
            lr = lr0 + (lr1 - lr0) * it / max(1, total - 1)
            hist.append(net.train_energy(op, res[idx].contiguous(), lr))
            it += 1
        op.close()
        del res
        if log and (i + 1) % log_every == 0:
            k = log_every * steps_per_field
            log(f"train: {i + 1}/{len(seeds)} fields, loss {np.mean(hist[-k:]):.4e}, "
                f"{time.perf_counter() - t0:.1f} s")
    return hist


FORMS = {  # name: (precision, qdata format)
    "fp64": (femgpu.FP64, femgpu.QDATA_FULL),
    "fp32_mixed": (femgpu.FP32_IR, femgpu.QDATA_FULL),
    "fp32_mixed_affine": (femgpu.FP32_IR, femgpu.QDATA_AFFINE),
}


def calibrate(net, n, seeds, levels=2, p=1, form="fp32_mixed", rhs="random", rtol=1e-8):
    """Expected ratio of learned to plain iterations of the network on its
    problem family, measured on validation fields (seeds disjoint from the
    training and the held-out test seeds) with the network always on.  The
    solver uses it (SolverConfig.nn_iter_ratio) to decide whether the network
    pays on a given operator and form."""
    prec, fmt = FORMS[form]
    plain, learned = [], []
    for s in seeds:
        op, b = make_problem(n, s, levels, p, rhs)
        op.set_qdata_format(fmt)
        r0 = op.pcg(b, np.zeros(op.n_dofs()), femgpu.SolverConfig(rtol=rtol, max_iter=20000, precision=prec),
                    femgpu.PC_CHEBYSHEV)
        femgpu.attach_unet(op, net)
        r1 = op.pcg(b, np.zeros(op.n_dofs()), femgpu.SolverConfig(rtol=rtol, max_iter=20000, precision=prec),
                    femgpu.PC_CHEB_NN)
        femgpu.attach_unet(op, None)
        plain.append(r0.iterations)
        learned.append(r1.iterations)
        op.close()
    return float(np.sum(learned) / np.sum(plain)), {"seeds": [int(s) for s in seeds], "form": form,
                                                      "plain_iterations": plain, "learned_iterations": learned}


def evaluate(net, n, seeds, levels=2, p=1, forms=("fp64",), rhs="random", rtol=1e-8, iter_ratio=0.0):
    """Per held-out field: plain FP64 Chebyshev(4)-PCG (full qdata) against
    plain and learned flexible CG in each form; the learned solve's budget is
    the plain iteration count of the same form, and with iter_ratio > 0 the
    solver decides from measured per-iteration costs whether the network pays
    (fallback 2: not used)."""
    rows = []
    for s in seeds:
        op, b = make_problem(n, s, levels, p, rhs)
        row = {"seed": int(s)}
        x_ref = None
        for form in forms:
            prec, fmt = FORMS[form]
            op.set_qdata_format(fmt)
            cfg = femgpu.SolverConfig(rtol=rtol, max_iter=20000, precision=prec)
            x0 = np.zeros(op.n_dofs())
            r0 = op.pcg(b, x0, cfg, femgpu.PC_CHEBYSHEV)
            if x_ref is None:
                x_ref = x0.copy()
            femgpu.attach_unet(op, net)
            x1 = np.zeros(op.n_dofs())
            cfg1 = femgpu.SolverConfig(rtol=rtol, max_iter=20000, precision=prec, nn_budget=r0.iterations,
                                       nn_iter_ratio=iter_ratio)
            r1 = op.pcg(b, x1, cfg1, femgpu.PC_CHEB_NN)
            femgpu.attach_unet(op, None)
            row[form] = {"plain_iterations": r0.iterations, "plain_s": r0.solve_ms / 1e3,
                         "learned_iterations": r1.iterations, "learned_s": r1.solve_ms / 1e3,
                         "plain_true_residual": r0.true_residual, "learned_true_residual": r1.true_residual,
                         "fallback": r1.extra["nn_fallback"],
                         "learned_rel_diff_vs_fp64_plain": float(np.linalg.norm(x1 - x_ref) / np.linalg.norm(x_ref))}
        rows.append(row)
        op.close()
    return rows


def save(net, path, meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, params=net.get_params(), channels=np.array(net.channels),
                        meta=json.dumps(meta))


def load(path=WEIGHTS):
    d = np.load(path)
    net = femgpu.UNet(tuple(int(c) for c in d["channels"]))
    net.set_params(d["params"])
    return net, json.loads(str(d["meta"]))


def summarise(rows, form):
    r = [row[form] for row in rows]
    return {"mean_plain_iterations": float(np.mean([x["plain_iterations"] for x in r])),
            "mean_learned_iterations": float(np.mean([x["learned_iterations"] for x in r])),
            "mean_plain_s": float(np.mean([x["plain_s"] for x in r])),
            "mean_learned_s": float(np.mean([x["learned_s"] for x in r])),
            "learned_not_slower": int(sum(x["learned_s"] <= x["plain_s"] for x in r)),
            "fallbacks": int(sum(x["fallback"] == 1 for x in r)),
            "network_not_used": int(sum(x["fallback"] == 2 for x in r))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--p", type=int, default=1)
    ap.add_argument("--levels", type=int, default=2)
    ap.add_argument("--train-fields", type=int, default=200)
    ap.add_argument("--first-seed", type=int, default=0)
    ap.add_argument("--eval-fields", type=int, default=10)
    ap.add_argument("--eval-rhs", default="random", choices=["random", "sin"])
    ap.add_argument("--forms", default="fp64,fp32_mixed")
    ap.add_argument("--every", type=int, default=2)
    ap.add_argument("--max-res", type=int, default=48)
    ap.add_argument("--steps-per-field", type=int, default=10)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--channels", default="16,32,48")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--calibrate-fields", type=int, default=0,
                    help="validation fields (seeds 50000+) for the expected iteration ratio stored with the weights")
    ap.add_argument("--calibrate-form", default="fp32_mixed")
    args = ap.parse_args()
    t0 = time.perf_counter()
    init_meta = None
    if args.init:
        net, init_meta = load(args.init)
    else:
        net = femgpu.UNet(tuple(int(c) for c in args.channels.split(",")), seed=1)
    seeds = list(range(args.first_seed, args.first_seed + args.train_fields))
    hist = train(net, args.n, seeds, args.levels, args.every, args.max_res,
                 args.steps_per_field, args.batch, lr0=args.lr, p=args.p) if seeds else [0.0]
    t_train = time.perf_counter() - t0
    k = args.steps_per_field * 10
    meta = {"n": args.n, "p": args.p, "levels": args.levels, "train_fields": args.train_fields,
            "first_seed": args.first_seed, "every": args.every, "max_res": args.max_res,
            "steps_per_field": args.steps_per_field, "batch": args.batch, "lr": args.lr,
            "first_loss": float(np.mean(hist[:k])), "final_loss": float(np.mean(hist[-k:])),
            "train_s": t_train, "params": net.num_params, "channels": list(net.channels)}
    if args.init and seeds:  # fine-tuned from earlier weights
        meta["init_from"] = {"file": os.path.basename(args.init),
                             **{k: init_meta[k] for k in ("train_fields", "first_seed", "steps_per_field", "lr")
                                if k in init_meta}}
    if seeds:
        save(net, args.out, meta)
    elif init_meta is not None:  # evaluation of stored weights
        meta = dict(init_meta, evaluation_only=True)
    if args.calibrate_fields > 0:
        ratio, cal = calibrate(net, args.n, list(range(50_000, 50_000 + args.calibrate_fields)), args.levels,
                               args.p, args.calibrate_form, args.eval_rhs)
        meta = {k: v for k, v in meta.items() if k != "evaluation_only"}
        meta["iter_ratio"] = ratio
        meta["calibration"] = cal
        save(net, args.out, meta)
        if not seeds:
            meta = dict(meta, evaluation_only=True)
    forms = args.forms.split(",")
    eval_seeds = list(range(100_000, 100_000 + args.eval_fields))
    rows = evaluate(net, args.n, eval_seeds, args.levels, args.p, forms, args.eval_rhs,
                    iter_ratio=float(meta.get("iter_ratio", 0.0)))
    summary = {"meta": meta, **{f: summarise(rows, f) for f in forms}, "eval": rows}
    print(json.dumps(summary))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
