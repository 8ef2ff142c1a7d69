"""Column-sharded previous-AMM power method over several GPUs, one process per GPU.

The reference runs one matrix on one GPU (``powerMethod_by_previous.cuh:100-210``).  Here the
columns of A are split over G ranks: rank g holds the n_g contiguous columns [col0_g, col0_g +
n_g).  The power method's state (x, x_memo, y_memo, the xorshift states) is replicated, so that
every rank takes the same decisions:

* set-up, once per matrix: each rank's one-pass column statistics give its FP64 CDF of ‖A_j‖²
  (set_weights / the CDF scan, ``common.h:34-40``, ``powerMethod_by_previous.cuh:26-32``); the
  ranks' CDFs and totals are all-gathered into the global CDF, cdf[j] = (Σ_{h<g} total_h) +
  cdf_g[j − col0_g] for j in rank g's columns;
* an AMM step (``powerMethod_by_previous.cuh:7-98``): every rank draws the same c picks from the
  global CDF with the same states (pick_index, ``device_memory.h:506-545``) and multiplies by its
  own picked columns only (``amm_shard_product``); a variance-reduction step
  (``powerMethod_by_previous.cuh:135-157``) multiplies by all of its columns;
* one all-reduce of the m partial products per step gives y on every rank (rank 0 adds y_memo);
  the Rayleigh step (``dotProduct_and_generate_x``, ``common.h:89-154``) then runs on every rank
  on the same y.

So each step moves m floats over NVLink (NCCL all-reduce) against m·c_d·s/G bytes of column
reads per GPU.  The products are libamm's kernels; the driver orders them and the collective.
``backend`` exists so that the host logic (partition, global CDF, collective, replicated state)
can also run on CPU ranks with gloo; the default is libamm on the rank's GPU.
"""
from __future__ import annotations

import torch
import torch.distributed as dist

__all__ = ["ShardedPowerMethod", "LibammShard", "shard_bounds"]


def shard_bounds(n_global: int, world: int, rank: int):
    """[col0, col1) of rank `rank`: contiguous shards, the first n_global % world one wider."""
    base, extra = divmod(int(n_global), int(world))
    col0 = rank * base + min(rank, extra)
    return col0, col0 + base + (1 if rank < extra else 0)


class LibammShard:
    """The rank's columns in a libamm context (previous AMM, one product per call)."""

    def __init__(self, A_local: torch.Tensor, c: int, dtype: str = "f32"):
        from .api import AMMContext
        m, n = A_local.shape
        self.ctx = AMMContext(m, n, c=c, step=1, dtype=dtype)
        self.ctx.set_matrix(A_local)

    def local_cdf(self) -> torch.Tensor:
        cdf, _ = self.ctx.sampling_tables(0)
        return cdf

    def exact(self, x):
        return self.ctx.exact_product(x)

    def sampled(self, cdf_global, col0, states, x, x_memo, y_memo):
        return self.ctx.shard_product(cdf_global, col0, states, x, x_memo, y_memo)

    def normalize(self, x):
        return self.ctx.normalize(x)

    def rayleigh(self, x, y):
        return self.ctx.rayleigh_normalize(x, y)

    def close(self):
        self.ctx.close()


class ShardedPowerMethod:
    """``step`` iterations of previous AMM over the column shards of all ranks of ``group``.

    ``vr_period`` P > 0: step i is an exact, memoised step when (i + 1) % P == 0, as the
    reference's previous driver decides (``powerMethod_by_previous.cuh:135-137``)."""

    def __init__(self, backend, col0: int, n_global: int, c: int, step: int,
                 vr_period: int = 0, group=None):
        self.be = backend
        self.col0 = int(col0)
        self.n_global = int(n_global)
        self.c = int(c)
        self.step = int(step)
        self.vr_period = int(vr_period)
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.cdf = self._global_cdf()

    def _global_cdf(self) -> torch.Tensor:
        """All ranks' CDFs, each shifted by the totals of the ranks before it (rank order)."""
        local = self.be.local_cdf().to(torch.float64)
        if self.world == 1:
            cdf = local.contiguous()
        else:
            n_loc = torch.tensor([local.numel()], dtype=torch.int64, device=local.device)
            sizes = [torch.zeros_like(n_loc) for _ in range(self.world)]
            dist.all_gather(sizes, n_loc, group=self.group)
            sizes = [int(v.item()) for v in sizes]
            pad = torch.zeros(max(sizes), dtype=torch.float64, device=local.device)
            pad[:local.numel()] = local
            parts = [torch.zeros_like(pad) for _ in range(self.world)]
            dist.all_gather(parts, pad, group=self.group)
            out, offset = [], 0.0
            for g in range(self.world):
                cg = parts[g][:sizes[g]]
                out.append(cg + offset)  # FP64; the ranks' totals summed in rank order
                offset = offset + float(cg[-1].item())
            cdf = torch.cat(out).contiguous()
        if cdf.numel() != self.n_global:
            raise ValueError(f"the shards hold {cdf.numel()} columns, not {self.n_global}")
        return cdf

    def _all_reduce(self, y):
        if self.world > 1:
            dist.all_reduce(y, op=dist.ReduceOp.SUM, group=self.group)
        return y

    def run(self, x0: torch.Tensor, states: torch.Tensor) -> dict:
        """One power-method call from the raw start vector x0 with the c sampling states
        (advanced in place, the same on every rank).  Returns the λ, err, cos traces and kinds."""
        x = x0.clone()
        self.be.normalize(x)
        x_memo = y_memo = None
        eigs, errs, coss, kinds = [], [], [], []
        for i in range(self.step):
            if self.vr_period > 0 and (i + 1) % self.vr_period == 0:
                y = self._all_reduce(self.be.exact(x))
                x_memo, y_memo = x.clone(), y.clone()
                kinds.append("exact")
            else:
                ym = y_memo if self.rank == 0 else None
                y = self._all_reduce(self.be.sampled(self.cdf, self.col0, states, x, x_memo, ym))
                kinds.append("previous")
            lam, err, cosv = self.be.rayleigh(x, y)  # x <- y/‖y‖
            eigs.append(lam)
            errs.append(err)
            coss.append(cosv)
        return {"eigs": eigs, "errs": errs, "coss": coss, "kinds": kinds, "x": x}
