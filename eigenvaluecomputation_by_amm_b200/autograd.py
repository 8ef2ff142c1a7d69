"""λ_max as a differentiable torch operation over libamm's batched kernels.

``lambda_max(A)`` returns λ_max(A_b·A_bᵀ) for every matrix of a batch (B, m, n) (or one matrix
(m, n)) of FP32 CUDA tensors.  The forward pass is libamm's batched block power iteration
(``amm_batch_run``: one persistent launch, 8 vectors, Rayleigh–Ritz, FP64 reductions); the
backward pass is libamm's kernel for ∂λ/∂A = 2·v(vᵀA) (``amm_batch_grad``), v being the unit
top eigenvector of A_b·A_bᵀ that the forward pass returns.  The gradient formula holds for a
simple top eigenvalue (a gap between λ_1 and λ_2).
"""
from __future__ import annotations

from typing import Dict, Tuple

import torch

from .api import BatchSolver

__all__ = ["lambda_max", "LambdaMax"]

# tile shape (columns per group, CTAs per matrix) picked by the autotuner, per batch shape
_TILES: Dict[Tuple, int] = {}


def _column_major_batch(A: torch.Tensor) -> torch.Tensor:
    """(B, n, ld) storage holding each A_b column-major with ld = m rounded up to 4."""
    B, m, n = A.shape
    ld = (m + 3) // 4 * 4
    buf = torch.zeros(B, n, ld, dtype=torch.float32, device=A.device)
    buf[:, :, :m] = A.transpose(1, 2)
    return buf


class LambdaMax(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A: torch.Tensor, max_iter: int = 1000, tol: float = 1e-6,
                nvec: int = 8):
        if not A.is_cuda or A.dtype != torch.float32 or A.dim() != 3:
            raise ValueError("lambda_max expects an FP32 CUDA tensor of shape (B, m, n)")
        B, m, n = A.shape
        buf = _column_major_batch(A)
        mats = [buf[b].t()[:m] for b in range(B)]            # (m, n) views, stride (1, ld)
        key = (B, m, n, nvec)
        gc, cl = _TILES.get(key, (0, 0))
        solver = BatchSolver(mats, nvec=nvec, max_iter=max_iter, tol=tol, tile_gc=gc,
                             cluster=cl, use_graph=False)
        lam, _, iters = solver.run()
        if key not in _TILES:
            _TILES[key] = solver.tile_choice()[1:]
        lam = lam.clone()
        ctx.solver = solver
        ctx.buf = buf
        ctx.shape = (B, m, n)
        ctx.mark_non_differentiable(iters)
        return lam, iters

    @staticmethod
    def backward(ctx, g_lam, g_iters):
        B, m, n = ctx.shape
        solver = ctx.solver
        gbuf = torch.empty(B, n, ctx.buf.shape[2], dtype=torch.float32, device=ctx.buf.device)
        grads = [gbuf[b].t()[:m] for b in range(B)]
        solver.grad(grads, scale=g_lam.to(torch.float32))
        solver.close()
        return gbuf[:, :, :m].transpose(1, 2), None, None, None


def lambda_max(A: torch.Tensor, max_iter: int = 1000, tol: float = 1e-6, nvec: int = 8):
    """λ_max(A_b·A_bᵀ) (FP64, shape (B,) or scalar) with a libamm backward for A.

    Iteration stops at ‖C·v − λ·v‖ <= tol·λ (or max_iter products); the eigenvector, and so the
    gradient, is then accurate to about tol·λ_1/(λ_1 − λ_2)."""
    single = A.dim() == 2
    lam, _ = LambdaMax.apply(A.unsqueeze(0) if single else A, max_iter, tol, nvec)
    return lam[0] if single else lam
