"""λ_max as a differentiable torch operation over libamm's batched kernels.

``lambda_max(A)`` returns λ_max(A_b·A_bᵀ) for every matrix of a batch (B, m, n) (or one matrix
(m, n)) of FP32 CUDA tensors.  The forward pass is libamm's batched block power iteration
(``amm_batch_run``: one persistent launch, 8 vectors, Rayleigh–Ritz, FP64 reductions); the
backward pass is libamm's kernel for ∂λ/∂A = 2·v(vᵀA) (``amm_batch_grad``), v being the unit
top eigenvector of A_b·A_bᵀ that the forward pass returns.  The gradient formula holds for a
simple top eigenvalue (a gap between λ_1 and λ_2).

A contiguous (B, m, n) input with n <= m (and n <= 2048) is not copied: the memory of a
row-major m x n matrix is the column-major n x m matrix Aᵀ, and λ_max(AᵀA) = λ_max(AAᵀ).  The
solver then runs on Aᵀ (top eigenvector u of AᵀA), and the same gradient kernel applied to the
transposed problem, 2·u·(uᵀAᵀ), is (∂λ/∂A)ᵀ — whose column-major n x m layout is exactly the
row-major m x n gradient (indeed ∂λ/∂A = 2·(A·u)·uᵀ).  Otherwise A is copied into a column-major
buffer first: the batched kernel runs faster on the orientation with fewer rows (measured on
the 64 x 512 x 2048 batch: 11.4 ms per forward + backward with the copy, 12.1 ms on the
2048-row transposed problem), so the copy pays when m < n.

One solver (batch context, tile choice) is kept per input shape and rebound to each call's
matrices (``amm_batch_set_matrices``, stream-ordered), so a call allocates no device context and
runs no autotuning after the first call of its shape.
"""
from __future__ import annotations

from typing import Dict, Tuple

import torch

from .api import BatchSolver

__all__ = ["lambda_max", "LambdaMax"]

# one solver per (device, B, m, n, nvec, max_iter, tol, route)
_SOLVERS: Dict[Tuple, BatchSolver] = {}


def _route(A: torch.Tensor, nvec: int) -> str:
    B, m, n = A.shape
    if (A.is_contiguous() and nvec <= n <= min(m, 2048) and n % 4 == 0
            and A.data_ptr() % 16 == 0):
        return "transposed"
    return "copy"


def _column_major_batch(A: torch.Tensor) -> torch.Tensor:
    """(B, n, ld) storage holding each A_b column-major with ld = m rounded up to 4."""
    B, m, n = A.shape
    ld = (m + 3) // 4 * 4
    buf = torch.zeros(B, n, ld, dtype=torch.float32, device=A.device)
    buf[:, :, :m] = A.transpose(1, 2)
    return buf


def _views(A: torch.Tensor, route: str):
    """The column-major matrices the solver runs on, and the storage they live in."""
    B, m, n = A.shape
    if route == "transposed":
        return [A[b].t() for b in range(B)], A           # (n, m), stride (1, n): Aᵀ_b
    buf = _column_major_batch(A)
    return [buf[b].t()[:m] for b in range(B)], buf       # (m, n), stride (1, ld)


def _solver(key, mats, max_iter, tol, nvec):
    s = _SOLVERS.get(key)
    if s is None:
        # the first call of a shape autotunes the tile shape on its own batch (untimed after)
        s = BatchSolver(mats, nvec=nvec, max_iter=max_iter, tol=tol, use_graph=False)
        _SOLVERS[key] = s
    else:
        s.set_matrices(mats)
    return s


class LambdaMax(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A: torch.Tensor, max_iter: int = 1000, tol: float = 1e-6,
                nvec: int = 8, route: str = "auto"):
        if not A.is_cuda or A.dtype != torch.float32 or A.dim() != 3:
            raise ValueError("lambda_max expects an FP32 CUDA tensor of shape (B, m, n)")
        B, m, n = A.shape
        if route == "auto":
            route = _route(A, nvec)
        elif route not in ("copy", "transposed") or (
                route == "transposed" and not (A.is_contiguous() and nvec <= n <= 2048
                                               and n % 4 == 0 and A.data_ptr() % 16 == 0)):
            raise ValueError(f"lambda_max: route {route!r} is not available for this input")
        mats, store = _views(A, route)
        key = (A.device.index, B, m, n, nvec, int(max_iter), float(tol), route)
        solver = _solver(key, mats, max_iter, tol, nvec)
        lam, vec, iters = solver.run()
        ctx.key = key
        ctx.mats = mats
        ctx.store = store
        ctx.vectors = vec.clone()      # a later forward of the same shape reuses the solver
        ctx.shape = (B, m, n)
        ctx.route = route
        lam, iters = lam.clone(), iters.clone()
        ctx.mark_non_differentiable(iters)
        return lam, iters

    @staticmethod
    def backward(ctx, g_lam, g_iters):
        B, m, n = ctx.shape
        solver = _SOLVERS[ctx.key]
        solver.set_matrices(ctx.mats)  # this call's matrices (stream-ordered)
        if ctx.route == "transposed":
            # ∂λ/∂Aᵀ_b column-major (n x m, ld = n) is ∂λ/∂A_b row-major (m x n)
            out = torch.empty(B, m, n, dtype=torch.float32, device=ctx.store.device)
            grads = [out[b].t() for b in range(B)]
            solver.grad(grads, scale=g_lam.to(torch.float32), vectors=ctx.vectors)
            return out, None, None, None, None
        ld = ctx.store.shape[2]
        gbuf = torch.empty(B, n, ld, dtype=torch.float32, device=ctx.store.device)
        grads = [gbuf[b].t()[:m] for b in range(B)]
        solver.grad(grads, scale=g_lam.to(torch.float32), vectors=ctx.vectors)
        return gbuf[:, :, :m].transpose(1, 2), None, None, None, None


def lambda_max(A: torch.Tensor, max_iter: int = 1000, tol: float = 1e-6, nvec: int = 8,
               route: str = "auto"):
    """λ_max(A_b·A_bᵀ) (FP64, shape (B,) or scalar) with a libamm backward for A.

    Iteration stops at ‖C·v − λ·v‖ <= tol·λ (or max_iter products); the eigenvector, and so the
    gradient, is then accurate to about tol·λ_1/(λ_1 − λ_2).  ``route``: "auto" (in place as
    the transposed problem when the input allows it), "copy" or "transposed"."""
    single = A.dim() == 2
    lam, _ = LambdaMax.apply(A.unsqueeze(0) if single else A, max_iter, tol, nvec, route)
    return lam[0] if single else lam
