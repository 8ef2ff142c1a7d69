"""Batched λ_max benchmarks: many matrices per launch, and the differentiable λ_max.

    python -m eigenvaluecomputation_by_amm_b200.bench_batch [--which batch,grad]

``batch`` (512 FP32 matrices, m log-uniform in [64, 2048], n log-uniform in [256, 8192],
entries N(0,1) times lognormal(0,1) column scales, matrix b generated from seed b): block power
iteration with 8 vectors and Rayleigh–Ritz, a fixed number of products per matrix, exact and
previous-AMM (c = n/8) products; matrices/s of the persistent launch (replayed from a CUDA
graph) against one launch per matrix, the HBM rate of the exact run, and the λ_max error
against FP64 eigvalsh on a subset.

``grad`` (64 FP32 matrices of 512 x 2048, lognormal(0,0.5) column scales): forward (block power
iteration to convergence) plus backward (2·v(vᵀA)) time per batch, and the gradient's error
against FP64 torch.linalg.eigvalsh autograd and against central differences (h = 1e-3, FP64) on
32 entries.  Prints one JSON line per benchmark.
"""
from __future__ import annotations

import argparse
import json
import math

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


def bench_batch(args):
    mats, stores, shapes = make_batch(args.count)
    bytes_per_product = sum(m * n * 4 for m, n in shapes)
    out = {"metric": "batched λ_max: matrices/s (8-vector block power iteration, Rayleigh–Ritz)",
           "unit": "matrices/s", "n_gpus": 1, "data": "synthetic",
           "config": {"workload": f"{args.count} FP32 matrices, m log-uniform [64, 2048], n "
                                  "log-uniform [256, 8192], N(0,1) x lognormal(0,1) columns, "
                                  f"{args.iters} products per matrix, 8 vectors",
                      "total_bytes": bytes_per_product}}
    hbm, src = _peak()
    fix_gc, fix_cl = (int(v) for v in args.tiles.split(",")) if args.tiles else (0, 0)
    modes = [(md, cd) for md, cd in (("exact", 0), ("amm_c_n_over_8", 8))
             if md.split("_")[0] in args.modes.split(",")]
    for mode, cdiv in modes:
        bs = BatchSolver(mats, nvec=8, max_iter=args.iters, tol=0.0, c_divisor=cdiv,
                         tile_gc=fix_gc, cluster=fix_cl)
        t_one = time_runs(bs, each=False)
        t_each = time_runs(bs, each=True)
        k, gc, cl = bs.tile_choice()
        lam = bs.lam[:, 0].double().cpu().numpy()
        errs = []
        for i in range(0, args.count, max(1, args.count // args.check)):
            A = mats[i].double()
            w = torch.linalg.eigvalsh(A @ A.t())[-1].item()
            errs.append(abs(lam[i] - w) / w)
        res = {"matrices_per_s": args.count * 1000.0 / t_one, "ms_per_launch": t_one,
               "one_launch_per_matrix_matrices_per_s": args.count * 1000.0 / t_each,
               "ms_one_launch_per_matrix": t_each, "speedup_vs_launch_per_matrix": t_each / t_one,
               "tile_cols_per_group": gc, "ctas_per_matrix": cl, "wide_plan": bs.wide_plan(),
               "lambda_rel_err_max": max(errs),
               "lambda_rel_err_median": float(np.median(errs)), "checked": len(errs)}
        if cdiv == 0:
            ach = bytes_per_product * args.iters / (t_one * 1e-3) / 1e9
            res["roofline"] = {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                               "frac": ach / hbm, "peak_source": src}
        out[mode] = res
        bs.close()
    out["value"] = out[modes[0][0]]["matrices_per_s"]
    print(json.dumps(out), flush=True)


def bench_grad(args):
    from .autograd import LambdaMax
    B, m, n = 64, 512, 2048
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(B, m, n, device="cuda", generator=g)
    A *= torch.exp(0.5 * torch.randn(B, 1, n, device="cuda", generator=g))
    ts = []
    for r in range(4):
        X = A.clone().requires_grad_(True)
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        lam, iters = LambdaMax.apply(X, 2000, 1e-6, 8)
        lam.sum().backward()
        e1.record()
        e1.synchronize()
        if r:
            ts.append(e0.elapsed_time(e1))
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
    for _ in range(32):
        b, i, j = int(rng.integers(B)), int(rng.integers(m)), int(rng.integers(n))
        Ap, Am = An[b].copy(), An[b].copy()
        Ap[i, j] += h
        Am[i, j] -= h
        fd = (np.linalg.eigvalsh(Ap @ Ap.T)[-1] - np.linalg.eigvalsh(Am @ Am.T)[-1]) / (2 * h)
        fd_err = max(fd_err, abs(grad[b, i, j].item() - fd) / gmax)
    out = {"metric": "Σ_b λ_max(A_b·A_bᵀ) forward + backward time per batch", "unit": "ms",
           "value": min(ts), "higher_is_better": False, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": "64 FP32 matrices 512 x 2048, N(0,1) x lognormal(0,0.5) "
                                  "columns, 8-vector block power iteration to ‖Cv − λv‖ <= 1e-6·λ"},
           "products_per_matrix_max": int(iters.max()), "products_per_matrix_min": int(iters.min()),
           "grad_rel_err_vs_fp64_eigvalsh": rel, "lambda_rel_err_max": lam_err,
           "fd_max_abs_err_over_max_grad": fd_err, "fd_entries": 32, "fd_h": h}
    print(json.dumps(out), flush=True)


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--which", default="batch,grad")
    p.add_argument("--count", type=int, default=512)
    p.add_argument("--iters", type=int, default=20)
    p.add_argument("--check", type=int, default=32, help="matrices checked against FP64")
    p.add_argument("--modes", default="exact,amm", help="batch products: exact, amm or both")
    p.add_argument("--tiles", default="",
                   help="fixed tile shape 'cols_per_group,ctas_per_matrix' (default: autotuned)")
    args = p.parse_args()
    for w in args.which.split(","):
        {"batch": bench_batch, "grad": bench_grad}[w](args)


if __name__ == "__main__":
    main()
