"""Python face of libamm over the C ABI (include/amm.h).

PyTorch provides device memory and streams; every computation runs in libamm's CUDA kernels.
Matrices are column-major m x n: a torch tensor ``A`` of shape (m, n) with ``A.stride(0) == 1``
(``column_major(t)`` makes one), exactly the layout the reference uses (lda = m).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import AmmError, amm_config, check

__all__ = ["AMMContext", "BatchSolver", "column_major", "AmmError", "generate_matrix",
           "read_matrix_file"]


def column_major(A: torch.Tensor) -> torch.Tensor:
    """A column-major copy (stride (1, m)) of a 2-D tensor, keeping shape (m, n)."""
    return A.t().contiguous().t()


# torch's raw accessors of the current device and stream: a fraction of the host time of
# torch.cuda.current_stream(), which builds a Stream object on every call (this runs once per
# library call, while the GPU may be idle waiting for the launch)
_raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_cur_device = getattr(torch._C, "_cuda_getDevice", None)


def _stream(stream=None) -> int:
    if stream is None:
        if _raw_stream is not None and _cur_device is not None:
            return int(_raw_stream(_cur_device()))
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


def _u32(t: torch.Tensor) -> torch.Tensor:
    """View an int32/uint32 tensor as the int32 carrier used for uint32 buffers."""
    if t.dtype == torch.int32:
        return t
    if t.dtype == torch.uint32:
        return t.view(torch.int32)
    raise TypeError("sampling states/indices must be int32 or uint32 tensors (bit pattern kept)")


class AMMContext:
    """One libamm context (the reference's ``device_memory`` with its buffers and handles).

    Parameters mirror ``host_memory`` (host_memory.h:26-50): ``c`` samples (0 = n), ``step``
    iterations, ``vr_period`` / ``vr_adaptive_threshold`` variance reduction, ``sanity``.
    ``dtype`` is the storage type of A ("f32" or "bf16"); ``cdf_precision`` "f64" (default)
    or "f32" (the reference's FP32 CDF and target).
    """

    def __init__(self, m: int, n: int, c: int = 0, step: int = 10, vr_period: int = 0,
                 vr_adaptive_threshold: float = 0.0, tol: float = 0.0, dtype: str = "f32",
                 cdf_precision: str = "f64", sanity: bool = False, use_graph: bool = True,
                 device: Optional[int] = None):
        self.lib = _lib.load()
        cfg = amm_config()
        self.lib.amm_config_default(C.byref(cfg))
        cfg.m, cfg.n, cfg.c, cfg.step = int(m), int(n), int(c), int(step)
        cfg.vr_period = int(vr_period)
        cfg.vr_adaptive_threshold = float(vr_adaptive_threshold)
        cfg.tol = float(tol)
        cfg.dtype = {"f32": _lib.AMM_F32, "bf16": _lib.AMM_BF16}[dtype]
        cfg.cdf_precision = {"f64": _lib.AMM_CDF_F64, "f32": _lib.AMM_CDF_F32}[cdf_precision]
        cfg.sanity = 1 if sanity else 0
        cfg.use_graph = 1 if use_graph else 0
        self.cfg = cfg
        self.m, self.n = int(m), int(n)
        self.c = int(c) if c else int(n)
        self.step = int(step)
        self.dtype = dtype
        self.cdf_precision = cdf_precision
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._ctx = C.c_void_p()
        check(self.lib.amm_create(C.byref(self._ctx), C.byref(cfg), self.device), "amm_create")
        self._A = None
        self._vstar = None
        self._dev = torch.device("cuda", self.device)

    # -- lifetime ---------------------------------------------------------------------
    def close(self):
        if self._ctx:
            check(self.lib.amm_destroy(self._ctx), "amm_destroy")
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- inputs -------------------------------------------------------------------------
    def set_matrix(self, A: torch.Tensor, stream=None):
        """Bind A (kept referenced) and run the one-pass set-up (stats, z, v, CDFs)."""
        want = torch.float32 if self.dtype == "f32" else torch.bfloat16
        if A.dtype != want or A.device.type != "cuda" or A.dim() != 2:
            raise AmmError(_lib.AMM_ERR_INVALID_ARGUMENT, f"set_matrix: need a CUDA {want} matrix")
        if tuple(A.shape) != (self.m, self.n):
            raise AmmError(_lib.AMM_ERR_INVALID_ARGUMENT, "set_matrix: shape must be (m, n)")
        if A.stride(0) != 1 and self.n > 1:
            raise AmmError(_lib.AMM_ERR_INVALID_ARGUMENT, "set_matrix: A must be column-major")
        ld = A.stride(1) if self.n > 1 else self.m
        check(self.lib.amm_set_matrix(self._ctx, _ptr(A), ld, _stream(stream)), "amm_set_matrix")
        self._A = A

    def set_rng_state(self, states: torch.Tensor, stream=None):
        s = _u32(states)
        check(self.lib.amm_set_rng_state(self._ctx, _ptr(s), s.numel(), _stream(stream)),
              "amm_set_rng_state")

    def get_rng_state(self, count: Optional[int] = None, stream=None) -> torch.Tensor:
        count = self.c if count is None else int(count)
        out = torch.empty(count, dtype=torch.int32, device=self._dev)
        check(self.lib.amm_get_rng_state(self._ctx, _ptr(out), count, _stream(stream)),
              "amm_get_rng_state")
        return out

    def seed_rng(self, seed: int, count: Optional[int] = None, stream=None):
        count = max(self.m, self.c) if count is None else int(count)
        check(self.lib.amm_seed_rng(self._ctx, int(seed), count, _stream(stream)), "amm_seed_rng")

    def seed_start_vectors(self, seed: int):
        check(self.lib.amm_seed_start_vectors(self._ctx, int(seed)), "amm_seed_start_vectors")

    def draw_start_vector(self, stream=None) -> torch.Tensor:
        x0 = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        check(self.lib.amm_draw_start_vector(self._ctx, _ptr(x0), _stream(stream)),
              "amm_draw_start_vector")
        return x0

    def set_cdf(self, which: int, cdf: torch.Tensor, stream=None):
        want = torch.float32 if self.cdf_precision == "f32" else torch.float64
        cdf = cdf.to(device=self._dev, dtype=want).contiguous()
        check(self.lib.amm_set_cdf(self._ctx, int(which), _ptr(cdf), _stream(stream)),
              "amm_set_cdf")
        torch.cuda.current_stream().synchronize()

    def set_eigenvector(self, vstar: Optional[torch.Tensor], stream=None):
        if vstar is None:
            check(self.lib.amm_set_eigenvector(self._ctx, None, _stream(stream)), "amm_set_eigenvector")
            self._vstar = None
            return
        v = vstar.to(device=self._dev, dtype=torch.float64).contiguous()
        check(self.lib.amm_set_eigenvector(self._ctx, _ptr(v), _stream(stream)), "amm_set_eigenvector")
        self._vstar = v

    # -- power method ---------------------------------------------------------------------
    def power_method(self, method: str, x0: torch.Tensor, stream=None) -> "AMMContext":
        """Enqueue one power-method call (asynchronous); read it with trace()/vectors()."""
        if not (x0.dtype == torch.float32 and x0.is_cuda and x0.get_device() == self.device
                and x0.is_contiguous()):
            x0 = x0.to(device=self._dev, dtype=torch.float32).contiguous()
        check(self.lib.amm_power_method(self._ctx, _lib.METHODS[method], _ptr(x0), _stream(stream)),
              f"amm_power_method({method})")
        self._x0_keep = x0
        return self

    def trace(self, stream=None) -> dict:
        cap = self.step
        eigs = np.zeros(cap, np.float64)
        errs = np.zeros(cap, np.float64)
        coss = np.zeros(cap, np.float64)
        kinds = np.zeros(cap, np.int32)
        distinct = np.zeros(cap, np.int64)
        t_ns = np.zeros(cap, np.float64)
        run = C.c_int64(0)
        p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        check(self.lib.amm_get_trace(self._ctx, p(eigs), p(errs), p(coss), p(kinds), p(distinct),
                                     p(t_ns), C.byref(run), _stream(stream)), "amm_get_trace")
        k = int(run.value)
        return {"eigs": eigs[:k], "errs": errs[:k], "coss": coss[:k],
                "kinds": [_lib.STEP_KINDS[int(v)] for v in kinds[:k]], "distinct": distinct[:k],
                "t_ns": t_ns[:k], "steps_run": k}

    def device_clock(self, out: torch.Tensor, stream=None):
        """Enqueue a write of the device clock (%globaltimer, ns) into out[0] (int64, CUDA)."""
        if out.dtype != torch.int64 or out.device.type != "cuda":
            raise AmmError(_lib.AMM_ERR_INVALID_ARGUMENT, "device_clock: need a CUDA int64 tensor")
        check(self.lib.amm_device_clock(_ptr(out), _stream(stream)), "amm_device_clock")

    def step_clocks(self, stream=None) -> np.ndarray:
        """Raw device clock stamps of the last call: [0] end of its first kernel, [i+1] end of
        step i (ns)."""
        out = np.zeros(self.step + 1, np.uint64)
        k = C.c_int64(0)
        check(self.lib.amm_get_step_clocks(self._ctx, out.ctypes.data_as(C.c_void_p), out.size,
                                           C.byref(k), _stream(stream)), "amm_get_step_clocks")
        return out[:k.value]

    def vectors(self, stream=None):
        x = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        y = torch.empty_like(x)
        check(self.lib.amm_get_vectors(self._ctx, _ptr(x), _ptr(y), _stream(stream)), "amm_get_vectors")
        return x, y

    # -- single products and helpers (the reference's per-step functions) -----------------
    def _vec(self, t):
        return None if t is None else t.to(device=self._dev, dtype=torch.float32).contiguous()

    def core_previousAMM(self, x, x_memo=None, y_memo=None, stream=None):
        x, xm, ym = self._vec(x), self._vec(x_memo), self._vec(y_memo)
        y = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        idx = torch.empty(self.c, dtype=torch.int32, device=self._dev)
        check(self.lib.amm_core_previousAMM(self._ctx, _ptr(x), _ptr(xm), _ptr(ym), _ptr(y), _ptr(idx),
                                            _stream(stream)), "amm_core_previousAMM")
        return y, idx

    def core_proposedAMM(self, x, x_memo=None, y_memo=None, stream=None):
        x, xm, ym = self._vec(x), self._vec(x_memo), self._vec(y_memo)
        y = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        idx = torch.empty(self.c, dtype=torch.int32, device=self._dev)
        check(self.lib.amm_core_proposedAMM(self._ctx, _ptr(x), _ptr(xm), _ptr(ym), _ptr(y), _ptr(idx),
                                            _stream(stream)), "amm_core_proposedAMM")
        return y, idx

    def core_list_product(self, method: str, cols: torch.Tensor, wm: torch.Tensor, x,
                          x_memo=None, y_memo=None, stream=None):
        """The sampled product over a given work list (amm_core_list_product): distinct column
        indices ``cols`` (int32) with weights ``wm`` = w_j·multiplicity (FP32)."""
        cols = _u32(cols.to(self._dev).contiguous())
        wm = wm.to(device=self._dev, dtype=torch.float32).contiguous()
        x, xm, ym = self._vec(x), self._vec(x_memo), self._vec(y_memo)
        y = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        check(self.lib.amm_core_list_product(self._ctx, _lib.METHODS[method], _ptr(cols), _ptr(wm),
                                             cols.numel(), _ptr(x), _ptr(xm), _ptr(ym), _ptr(y),
                                             _stream(stream)), "amm_core_list_product")
        return y

    def shard_product(self, cdf_global: torch.Tensor, col0: int, states: torch.Tensor, x,
                      x_memo=None, y_memo=None, stream=None):
        """This rank's part of a previous-AMM product over a column-sharded matrix
        (amm_shard_product): the context holds global columns [col0, col0 + n); ``cdf_global``
        (FP64, all columns) and the c ``states`` (advanced in place) are the same on every
        rank."""
        st = _u32(states)
        x, xm, ym = self._vec(x), self._vec(x_memo), self._vec(y_memo)
        y = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        check(self.lib.amm_shard_product(self._ctx, _ptr(cdf_global), cdf_global.numel(),
                                         int(col0), _ptr(st), _ptr(st), _ptr(x), _ptr(xm),
                                         _ptr(ym), _ptr(y), _stream(stream)), "amm_shard_product")
        return y

    def exact_product(self, x, stream=None):
        x = self._vec(x)
        y = torch.empty(self.m, dtype=torch.float32, device=self._dev)
        check(self.lib.amm_exact_product(self._ctx, _ptr(x), _ptr(y), _stream(stream)), "amm_exact_product")
        return y

    def rayleigh_normalize(self, x: torch.Tensor, y: torch.Tensor, stream=None):
        """Returns (λ, err, cos) and normalises x <- y/‖y‖ in place."""
        out = torch.zeros(4, dtype=torch.float64, device=self._dev)
        check(self.lib.amm_rayleigh_normalize(self._ctx, _ptr(x), _ptr(self._vec(y)), _ptr(out),
                                              _stream(stream)), "amm_rayleigh_normalize")
        o = out.cpu().numpy()
        return float(o[0]), float(o[1]), float(o[2])

    def normalize(self, x: torch.Tensor, stream=None):
        check(self.lib.amm_normalize(self._ctx, _ptr(x), _stream(stream)), "amm_normalize")
        return x

    def column_stats(self, stream=None) -> dict:
        n, m = self.n, self.m
        out = {k: torch.empty(n, dtype=torch.float32, device=self._dev) for k in ("alpha", "norm", "normp")}
        out.update({k: torch.empty(m, dtype=torch.float32, device=self._dev) for k in ("z", "v")})
        a2 = C.c_double(0.0)
        check(self.lib.amm_get_column_stats(self._ctx, _ptr(out["alpha"]), _ptr(out["norm"]),
                                            _ptr(out["normp"]), _ptr(out["z"]), _ptr(out["v"]),
                                            C.byref(a2), _stream(stream)), "amm_get_column_stats")
        out["alpha2"] = a2.value
        return out

    def sampling_tables(self, which: int, stream=None):
        dt = torch.float32 if self.cdf_precision == "f32" else torch.float64
        cdf = torch.empty(self.n, dtype=dt, device=self._dev)
        w = torch.empty(self.n, dtype=torch.float32, device=self._dev)
        check(self.lib.amm_get_sampling_tables(self._ctx, int(which), _ptr(cdf), _ptr(w), _stream(stream)),
              "amm_get_sampling_tables")
        return cdf, w

    def sample_indices(self, which: int, stream=None) -> torch.Tensor:
        idx = torch.empty(self.c, dtype=torch.int32, device=self._dev)
        check(self.lib.amm_sample_indices(self._ctx, int(which), _ptr(idx), _stream(stream)),
              "amm_sample_indices")
        return idx

    def benchmark_product(self, kind: str, reps: int = 10, stream=None):
        """Mean CUDA-event time (ms) of one fused product launch (or of the set-up pass, kind
        "setup") and the distinct columns it reads."""
        k = {"exact": 1, "previous": 2, "proposed": 3, "setup": 16}[kind]
        ms = C.c_float(0.0)
        d = C.c_int64(0)
        check(self.lib.amm_benchmark_product(self._ctx, k, int(reps), C.byref(ms), C.byref(d),
                                             _stream(stream)), "amm_benchmark_product")
        return float(ms.value), int(d.value)

    def geometry(self) -> dict:
        out = (C.c_int32 * 10)()
        check(self.lib.amm_get_geometry(self._ctx, out), "amm_get_geometry")
        keys = ("cluster", "rows_per_cta", "clusters", "threads", "slots", "cols_per_stage",
                "stages", "stage_bytes", "smem_bytes", "worklist_cap")
        return dict(zip(keys, list(out)))

    def grad_lambda(self, v: torch.Tensor, stream=None) -> torch.Tensor:
        """∂λ/∂A = 2·v·(vᵀA) as an (m, n) column-major FP32 tensor."""
        v = self._vec(v)
        g = torch.empty(self.n, self.m, dtype=torch.float32, device=self._dev).t()
        check(self.lib.amm_grad_lambda(self._ctx, _ptr(v), _ptr(g), self.m, _stream(stream)),
              "amm_grad_lambda")
        return g


class BatchSolver:
    """λ_max of A_b·A_bᵀ for many FP32 matrices in one persistent launch (amm_batch_*).

    ``mats`` is a list of column-major FP32 CUDA tensors (shape (m_b, n_b), stride(0) == 1,
    stride(1) % 4 == 0, m_b <= 2048).  ``nvec`` vectors per matrix (1, 4 or 8) with
    Rayleigh–Ritz every ``rr_period`` products; iteration stops when the residual of the top
    Ritz pair ‖C·v − λ·v‖ is at most ``tol``·λ, or after ``max_iter`` products.  ``c_divisor`` k > 0 replaces the exact
    product by the previous-AMM estimate with c = n/k sampled columns per step; ``vr_period``
    P > 0 then makes every P-th product (and the last) exact and memoised, the others
    estimating C·X = Y_memo·S + Ĉ·(X − X_memo·S) with S = X_memoᵀX (variance reduction), and
    convergence is tested on exact products only.  The tensors are borrowed: keep them alive.
    """

    def __init__(self, mats, nvec: int = 8, max_iter: int = 500, tol: float = 1e-6,
                 rr_period: int = 1, seed: int = 1234, use_graph: bool = True, tile_gc: int = 0,
                 c_divisor: int = 0, cluster: int = 0, wide: int = 0, vr_period: int = 0,
                 device: Optional[int] = None):
        self.lib = _lib.load()
        self.mats = list(mats)
        self.count = len(self.mats)
        self.nvec = int(nvec)
        self.device = torch.cuda.current_device() if device is None else int(device)
        self._dev = torch.device("cuda", self.device)
        descs = self._descs(self.mats)
        cfg = _lib.amm_batch_config()
        self.lib.amm_batch_config_default(C.byref(cfg))
        cfg.nvec, cfg.max_iter, cfg.tol = int(nvec), int(max_iter), float(tol)
        cfg.rr_period, cfg.seed = int(rr_period), int(seed)
        cfg.use_graph, cfg.tile_gc = (1 if use_graph else 0), int(tile_gc)
        cfg.c_divisor = int(c_divisor)
        cfg.cluster = int(cluster)
        cfg.wide = int(wide)
        cfg.vr_period = int(vr_period)
        self.vr_period = int(vr_period)
        self.c_divisor = int(c_divisor)
        self.max_iter = int(max_iter)
        self._b = C.c_void_p()
        check(self.lib.amm_batch_create(C.byref(self._b), descs, self.count, C.byref(cfg),
                                        self.device), "amm_batch_create")
        offs = np.zeros(self.count + 1, np.int64)
        check(self.lib.amm_batch_vector_offsets(self._b, offs.ctypes.data_as(C.c_void_p)),
              "amm_batch_vector_offsets")
        self.offsets = offs
        self.lam = torch.empty(self.count, self.nvec, dtype=torch.float64, device=self._dev)
        self.vectors = torch.empty(int(offs[-1]), dtype=torch.float32, device=self._dev)
        self.iters = torch.empty(self.count, dtype=torch.int32, device=self._dev)

    def _descs(self, mats):
        descs = (_lib.amm_batch_matrix * len(mats))()
        for i, A in enumerate(mats):
            if A.dtype != torch.float32 or A.dim() != 2 or A.stride(0) != 1:
                raise ValueError("batch matrices must be column-major FP32 CUDA tensors")
            descs[i].A = A.data_ptr()
            descs[i].ld = A.stride(1) if A.shape[1] > 1 else max(A.shape[0], 4)
            descs[i].m, descs[i].n = A.shape
        return descs

    def set_matrices(self, mats, stream=None):
        """Rebind to new matrices of the same shapes (amm_batch_set_matrices; stream-ordered).
        The tile choice, the launch plan and the captured graph are kept."""
        mats = list(mats)
        descs = self._descs(mats)
        check(self.lib.amm_batch_set_matrices(self._b, descs, len(mats), _stream(stream)),
              "amm_batch_set_matrices")
        self.mats = mats

    def run(self, each: bool = False, stream=None):
        """One persistent launch (or one launch per matrix with ``each``); asynchronous."""
        fn = self.lib.amm_batch_run_each if each else self.lib.amm_batch_run
        check(fn(self._b, _ptr(self.lam), _ptr(self.vectors), _ptr(self.iters), _stream(stream)),
              "amm_batch_run_each" if each else "amm_batch_run")
        return self.lam[:, 0], self.vectors, self.iters

    def vector(self, i: int) -> torch.Tensor:
        return self.vectors[int(self.offsets[i]):int(self.offsets[i + 1])]

    def grad(self, grads, scale: Optional[torch.Tensor] = None, vectors=None, stream=None):
        """grads[b] <- scale_b · 2·v_b(v_bᵀA_b) (column-major tensors shaped like A_b), with the
        top vectors of the last run, or ``vectors`` (a copy of them) if given."""
        ptrs = (C.c_void_p * self.count)(*[g.data_ptr() for g in grads])
        lds = np.array([g.stride(1) if g.shape[1] > 1 else max(g.shape[0], 1) for g in grads],
                       np.int64)
        sc = None if scale is None else scale.to(device=self._dev, dtype=torch.float32).contiguous()
        vec = self.vectors if vectors is None else vectors
        check(self.lib.amm_batch_grad(self._b, _ptr(vec), ptrs,
                                      lds.ctypes.data_as(C.c_void_p), _ptr(sc), _stream(stream)),
              "amm_batch_grad")
        self._grad_keep = sc

    def record(self, products: int):
        """Record, on every later run, each matrix's FP32 sampling CDF and the raw picks of its
        first ``products`` AMM products (amm_batch_record).  Returns (cdf, picks, offsets):
        matrix b's CDF is cdf[col_off[b]:col_off[b+1]] and its picks of product p are
        picks[st_off[b]*products + p*c_b :][:c_b], with offsets = (col_off, st_off, c)."""
        cols = [int(A.shape[1]) for A in self.mats]
        cs = [max(1, n // self.c_divisor) for n in cols] if self.c_divisor else [0] * len(cols)
        col_off = np.concatenate([[0], np.cumsum(cols)]).astype(np.int64)
        st_off = np.concatenate([[0], np.cumsum(cs)]).astype(np.int64)
        self._rec_cdf = torch.zeros(int(col_off[-1]), dtype=torch.float32, device=self._dev)
        self._rec_picks = torch.full((int(st_off[-1]) * int(products),), -1, dtype=torch.int32,
                                     device=self._dev)
        check(self.lib.amm_batch_record(self._b, _ptr(self._rec_cdf), _ptr(self._rec_picks),
                                        int(products)), "amm_batch_record")
        return self._rec_cdf, self._rec_picks, (col_off, st_off, np.array(cs, np.int64))

    def tile_choice(self):
        """(vectors, columns per group, CTAs per matrix) picked by the autotuner."""
        k, gc, cl = C.c_int32(0), C.c_int32(0), C.c_int32(0)
        check(self.lib.amm_batch_tile_choice(self._b, C.byref(k), C.byref(gc), C.byref(cl)),
              "amm_batch_tile_choice")
        return int(k.value), int(gc.value), int(cl.value)

    def wide_plan(self) -> dict:
        """The autotuner's launch plan for uneven batches: the heaviest `count` matrices on a
        first launch with clusters of `cluster` CTAs (`ctas` in all), the rest shared with a
        second launch queued behind it; count 0 means one launch per run.  `ms`: the plan's time
        in the autotuner (0 if it was not timed)."""
        n, cl, g, ms = C.c_int32(0), C.c_int32(0), C.c_int32(0), C.c_float(0.0)
        check(self.lib.amm_batch_wide_plan(self._b, C.byref(n), C.byref(cl), C.byref(g),
                                           C.byref(ms)), "amm_batch_wide_plan")
        return {"count": int(n.value), "cluster": int(cl.value), "ctas": int(g.value),
                "ms": float(ms.value)}

    def close(self):
        if self._b:
            self.lib.amm_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_matrix(matrix_type: str, size: int, seed: int, stream=None, device=None):
    """The reference's -matrixType generator (amm_generate_matrix): a symmetric size x size FP32
    matrix (column-major; symmetric, so also row-major) with the diagonal offset added, and the
    offset."""
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
    A = torch.empty(int(size), int(size), dtype=torch.float32, device=dev)
    off = C.c_float(0.0)
    check(lib.amm_generate_matrix(matrix_type.encode(), int(size), int(seed), _ptr(A),
                                  C.byref(off), _stream(stream)), "amm_generate_matrix")
    return A, float(off.value)


def read_matrix_file(path: str, size: Optional[int] = None):
    """The reference's -filepath loader (amm_read_matrix_file): (host FP32 array of shape
    (size, size), original size).  size defaults to the file's size rounded up to 128, as the
    reference pads it."""
    lib = _lib.load()
    orig = C.c_int64(0)
    check(lib.amm_read_matrix_file(str(path).encode(), None, 0, C.byref(orig)),
          "amm_read_matrix_file")
    n0 = int(orig.value)
    size = int(size) if size else (n0 + 127) // 128 * 128
    out = np.empty((size, size), np.float32)
    check(lib.amm_read_matrix_file(str(path).encode(), out.ctypes.data_as(C.c_void_p), size,
                                   C.byref(orig)), "amm_read_matrix_file")
    return out, n0
