"""B200-native power method for λ_max(A·Aᵀ): exact, previous AMM and proposed AMM.

The compute path is libamm.so (hand-written sm_100a CUDA behind the C ABI of include/amm.h);
this package is its Python face.  The library is loaded on first use and every entry point
fails loudly (ImportError) when it has not been built
(``python -m eigenvaluecomputation_by_amm_b200.build``); there is no CPU fallback.
"""
from ._lib import AmmError  # noqa: F401
from .api import AMMContext, BatchSolver, column_major  # noqa: F401


def lambda_max(A, max_iter: int = 1000, tol: float = 1e-6, nvec: int = 8):
    """λ_max(A·Aᵀ) per matrix with a libamm backward (see ``autograd.lambda_max``)."""
    from .autograd import lambda_max as _lm
    return _lm(A, max_iter=max_iter, tol=tol, nvec=nvec)


__all__ = ["AMMContext", "BatchSolver", "column_major", "lambda_max", "AmmError"]
