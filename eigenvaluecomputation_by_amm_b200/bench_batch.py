"""Batched λ_max benchmarks: many matrices per launch, and the differentiable λ_max.

    python -m eigenvaluecomputation_by_amm_b200.bench_batch [--which batch,grad]

``batch`` (512 FP32 matrices, m log-uniform in [64, 2048], n log-uniform in [256, 8192],
entries N(0,1) times lognormal(0,1) column scales, matrix b generated from seed b): block power
iteration with 8 vectors and Rayleigh–Ritz, a fixed number of products per matrix, exact and
previous-AMM (c = n/8) products, the latter without and with variance reduction; matrices/s of
the persistent launch (replayed from a CUDA graph), the HBM rate of the exact run, the λ_max
error against FP64 eigvalsh on a subset, and two comparators that give each matrix the whole
GPU: libamm's single-matrix exact power method per matrix and FP32 eigvalsh per matrix.

``grad`` (64 FP32 matrices of 512 x 2048, lognormal(0,0.5) column scales): forward (block power
iteration to convergence) plus backward (2·v(vᵀA)) time per batch, and the gradient's error
against FP64 torch.linalg.eigvalsh autograd and against central differences (h = 1e-3, FP64) on
32 entries.  Prints one JSON line per benchmark.
"""
from __future__ import annotations

import argparse
import json
import math
import statistics

import numpy as np
import torch

from .api import BatchSolver


def _events():
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _peak():
    from pathlib import Path
    p = Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_batch(count=512, seed0=0, mlo=64, mhi=2048, nlo=256, nhi=8192, scale=1.0):
    """Column-major FP32 matrices on the GPU (ld = m rounded up to 4), from seeds seed0 + b."""
    mats, stores, shapes = [], [], []
    for b in range(count):
        g = torch.Generator(device="cuda").manual_seed(seed0 + b)
        gh = np.random.default_rng(seed0 + b)
        m = int(round(math.exp(gh.uniform(math.log(mlo), math.log(mhi)))))
        n = int(round(math.exp(gh.uniform(math.log(nlo), math.log(nhi)))))
        ld = (m + 3) // 4 * 4
        buf = torch.zeros(n, ld, device="cuda")
        buf[:, :m] = torch.randn(n, m, device="cuda", generator=g)
        buf[:, :m] *= torch.exp(scale * torch.randn(n, 1, device="cuda", generator=g))
        stores.append(buf)
        mats.append(buf.t()[:m])
        shapes.append((m, n))
    return mats, stores, shapes


def time_runs(bs, each, reps=3):
    bs.run(each=each)  # warm (and autotune)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = _events()
        e0.record()
        bs.run(each=each)
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return min(ts)


def _per_matrix_exact(stores, shapes, steps, reps=2):
    """Comparator with the whole GPU per matrix: libamm's single-matrix exact power method
    (amm_power_exact, one CUDA graph per call) on each matrix in turn, `steps` products each (the
    same passes over A as the batch's `steps` block products), timed over all matrices."""
    from .api import AMMContext
    ctxs = []
    for buf, (m, n) in zip(stores, shapes):
        ld = buf.shape[1]
        ctx = AMMContext(ld, n, step=steps, dtype="f32")  # rows m..ld-1 are zero: same λ
        ctx.set_matrix(buf.t())
        ctxs.append(ctx)
    x0s = [torch.ones(buf.shape[1], device="cuda") for buf in stores]
    for ctx, x0 in zip(ctxs, x0s):  # warm (graph capture)
        ctx.power_method("exact", x0)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0, e1 = _events()
        e0.record()
        for ctx, x0 in zip(ctxs, x0s):
            ctx.power_method("exact", x0)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1)
        best = t if best is None else min(best, t)
    lam = [float(ctx.trace()["eigs"][-1]) for ctx in ctxs]
    for ctx in ctxs:
        ctx.close()
    return best, lam


def _per_matrix_eigvalsh(mats):
    """Comparator: FP32 C = A·Aᵀ (cuBLAS) and torch.linalg.eigvalsh (cuSOLVER) per matrix."""
    for A in mats[:4]:
        torch.linalg.eigvalsh(A @ A.t())
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    lam = [torch.linalg.eigvalsh(A @ A.t())[-1] for A in mats]
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1), [float(x) for x in lam]


def batch_report(count=512, iters=20, check=32, modes=("exact", "amm", "amm_vr"), tiles="",
                 vr_period=4, comparators=True):
    """The batched configuration: one dict with a result per mode (exact block products, AMM
    c = n/8 without and with variance reduction every `vr_period` products) and, with
    `comparators`, the whole-GPU-per-matrix comparators."""
    mats, stores, shapes = make_batch(count)
    bytes_per_product = sum(m * n * 4 for m, n in shapes)
    out = {"metric": "batched λ_max: matrices/s (8-vector block power iteration, Rayleigh–Ritz)",
           "unit": "matrices/s", "n_gpus": 1, "data": "synthetic",
           "config": {"workload": f"{count} FP32 matrices, m log-uniform [64, 2048], n "
                                  "log-uniform [256, 8192], N(0,1) x lognormal(0,1) columns, "
                                  f"{iters} products per matrix, 8 vectors",
                      "total_bytes": bytes_per_product}}
    hbm, src = _peak()
    fix_gc, fix_cl = (int(v) for v in tiles.split(",")) if tiles else (0, 0)
    table = {"exact": (0, 0), "amm": (8, 0), "amm_vr": (8, vr_period)}
    truth = {}
    idx = list(range(0, count, max(1, count // check)))
    for i in idx:
        A = mats[i].double()
        truth[i] = torch.linalg.eigvalsh(A @ A.t())[-1].item()
    for mode in modes:
        cdiv, vr = table[mode]
        bs = BatchSolver(mats, nvec=8, max_iter=iters, tol=0.0, c_divisor=cdiv, vr_period=vr,
                         tile_gc=fix_gc, cluster=fix_cl)
        t_one = time_runs(bs, each=False)
        k, gc, cl = bs.tile_choice()
        lam = bs.lam[:, 0].double().cpu().numpy()
        errs = [abs(lam[i] - truth[i]) / truth[i] for i in idx]
        res = {"matrices_per_s": count * 1000.0 / t_one, "ms_per_launch": t_one,
               "tile_cols_per_group": gc, "ctas_per_matrix": cl, "wide_plan": bs.wide_plan(),
               "lambda_rel_err_max": max(errs),
               "lambda_rel_err_median": float(np.median(errs)), "checked": len(errs)}
        if cdiv:
            res["c"] = "n/8"
            res["vr_period"] = vr
            exact_products = (iters if not vr else
                              sum(1 for p in range(iters) if (p + 1) % vr == 0 or p + 1 >= iters))
            res["exact_products_per_matrix"] = exact_products if vr else 0
        if mode == "exact":
            ach = bytes_per_product * iters / (t_one * 1e-3) / 1e9
            res["roofline"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                               "frac": ach / hbm, "peak_source": src}
            t_each = time_runs(bs, each=True)
            res["one_cta_launch_per_matrix_matrices_per_s"] = count * 1000.0 / t_each
        out[mode] = res
        bs.close()
    if comparators:
        t_pm, lam_pm = _per_matrix_exact(stores, shapes, iters)
        err_pm = [abs(lam_pm[i] - truth[i]) / truth[i] for i in idx]
        out["per_matrix_power_exact"] = {
            "matrices_per_s": count * 1000.0 / t_pm, "ms": t_pm, "steps": iters,
            "lambda_rel_err_median": float(np.median(err_pm)), "lambda_rel_err_max": max(err_pm),
            "how": "libamm amm_power_exact on each matrix in turn (whole GPU per matrix, one "
                   f"CUDA graph per call), {iters} single-vector exact products each"}
        t_ev, lam_ev = _per_matrix_eigvalsh(mats)
        err_ev = [abs(lam_ev[i] - truth[i]) / truth[i] for i in idx]
        out["per_matrix_eigvalsh_fp32"] = {
            "matrices_per_s": count * 1000.0 / t_ev, "ms": t_ev,
            "lambda_rel_err_median": float(np.median(err_ev)), "lambda_rel_err_max": max(err_ev),
            "how": "torch: C = A·Aᵀ (cuBLAS FP32) and linalg.eigvalsh (cuSOLVER FP32) per matrix"}
        for mode in modes:
            out[mode]["speedup_vs_per_matrix_power_exact"] = t_pm / out[mode]["ms_per_launch"]
            out[mode]["speedup_vs_per_matrix_eigvalsh"] = t_ev / out[mode]["ms_per_launch"]
    out["value"] = out[modes[0]]["matrices_per_s"]
    return out


def bench_batch(args):
    modes = [md for md in ("exact", "amm", "amm_vr") if md in args.modes.split(",")]
    print(json.dumps(batch_report(args.count, args.iters, args.check, modes, args.tiles,
                                  args.vr_period)), flush=True)


def grad_report(reps=5, fd_entries=32):
    """The differentiation configuration: forward + backward time per batch (the first call of
    the shape, which creates the solver and autotunes it, is untimed), the backward kernel's
    rate against its algorithmic bytes, and the gradient's errors."""
    from .autograd import LambdaMax, _SOLVERS
    B, m, n = 64, 512, 2048
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(B, m, n, device="cuda", generator=g)
    A *= torch.exp(0.5 * torch.randn(B, 1, n, device="cuda", generator=g))
    def timed(route):
        out = []
        for r in range(reps + 1):
            X = A.clone().requires_grad_(True)
            torch.cuda.synchronize()
            e0, e1 = _events()
            e0.record()
            lam, iters = LambdaMax.apply(X, 2000, 1e-6, 8, route)
            lam.sum().backward()
            e1.record()
            e1.synchronize()
            if r:
                out.append(e0.elapsed_time(e1))
        return out, X, lam, iters

    t_tr, _, _, _ = timed("transposed")
    ts, X, lam, iters = timed("auto")       # m = 512 < n = 2048: the column-major copy
    # the backward kernel alone (grad_kernel: reads A, writes ∂λ/∂A; m·n·(4 + 4) bytes each)
    solver = next(s for k, s in _SOLVERS.items() if k[1:4] == (B, m, n) and k[-1] == "transposed")
    vec = solver.vectors.clone()
    out = torch.empty(B, m, n, device="cuda")
    views = [out[b].t() for b in range(B)]  # the transposed route's layout (rows of A contiguous)
    solver.grad(views, vectors=vec)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(20):
        solver.grad(views, vectors=vec)
    e1.record()
    e1.synchronize()
    t_grad = e0.elapsed_time(e1) / 20
    grad_bytes = B * m * n * 8
    hbm, src = _peak()
    grad = X.grad.double()
    A64 = A.double().requires_grad_(True)
    w = torch.linalg.eigvalsh(A64 @ A64.transpose(1, 2))[:, -1]
    w.sum().backward()
    rel = ((grad - A64.grad).norm() / A64.grad.norm()).item()
    lam_err = ((lam.detach() - w.detach()).abs() / w.detach()).max().item()
    rng = np.random.default_rng(1)
    h = 1e-3
    fd_err = 0.0
    gmax = grad.abs().max().item()
    An = A.double().cpu().numpy()
    for _ in range(fd_entries):
        b, i, j = int(rng.integers(B)), int(rng.integers(m)), int(rng.integers(n))
        Ap, Am = An[b].copy(), An[b].copy()
        Ap[i, j] += h
        Am[i, j] -= h
        fd = (np.linalg.eigvalsh(Ap @ Ap.T)[-1] - np.linalg.eigvalsh(Am @ Am.T)[-1]) / (2 * h)
        fd_err = max(fd_err, abs(grad[b, i, j].item() - fd) / gmax)
    return {"metric": "Σ_b λ_max(A_b·A_bᵀ) forward + backward time per batch", "unit": "ms",
            "value": statistics.mean(ts), "ms_min": min(ts), "higher_is_better": False,
            "n_gpus": 1, "data": "synthetic",
            "config": {"workload": "64 FP32 matrices 512 x 2048, N(0,1) x lognormal(0,0.5) "
                                   "columns, 8-vector block power iteration to ‖Cv − λv‖ <= 1e-6·λ",
                       "timed": f"mean of {reps} calls after a first (solver creation, autotune)"},
            "route": "copy (A copied column-major; 512 rows)",
            "ms_transposed_route": statistics.mean(t_tr),
            "products_per_matrix_max": int(iters.max()),
            "products_per_matrix_min": int(iters.min()),
            "grad_kernel": {"ms": t_grad, "bytes": grad_bytes,
                            "achieved_gbs": grad_bytes / (t_grad * 1e-3) / 1e9,
                            "frac": grad_bytes / (t_grad * 1e-3) / 1e9 / hbm, "peak": hbm,
                            "peak_source": src,
                            "note": "m·n·(4 + 4) bytes per matrix: A read, ∂λ/∂A written; "
                                    "268 MB of each per launch, larger than L2"},
            "grad_rel_err_vs_fp64_eigvalsh": rel, "lambda_rel_err_max": lam_err,
            "fd_max_abs_err_over_max_grad": fd_err, "fd_entries": fd_entries, "fd_h": h}


def bench_grad(args):
    print(json.dumps(grad_report()), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--which", default="batch,grad")
    p.add_argument("--count", type=int, default=512)
    p.add_argument("--iters", type=int, default=20)
    p.add_argument("--check", type=int, default=32, help="matrices checked against FP64")
    p.add_argument("--modes", default="exact,amm,amm_vr",
                   help="batch products: exact, amm (c = n/8), amm_vr (with variance reduction)")
    p.add_argument("--vr-period", type=int, default=4)
    p.add_argument("--tiles", default="",
                   help="fixed tile shape 'cols_per_group,ctas_per_matrix' (default: autotuned)")
    args = p.parse_args()
    for w in args.which.split(","):
        {"batch": bench_batch, "grad": bench_grad}[w](args)


if __name__ == "__main__":
    main()
