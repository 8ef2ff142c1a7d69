"""Launch the fused product kernel in isolation, for profilers (ncu) and quick timing.

    python -m eigenvaluecomputation_by_amm_b200.profile_product --m 16384 --n 8192 \
        --dtype bf16 --kinds exact,proposed --reps 1

Builds a context on a seeded N(0,1) x lognormal(0,1) matrix, runs one warm-up call (which also
runs the set-up pass), then times `reps` launches of the product kernel per kind with CUDA
events and prints the mean time and the algorithmic HBM rate per launch.

This is the driver that the ncu captures summarised under profiles/ were taken with (each
summary gives its exact command line); it ships with the package so that those commands run
on any install, and the library itself never imports it.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

from .api import AMMContext, column_major


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--m", type=int, default=16384)
    p.add_argument("--n", type=int, default=8192)
    p.add_argument("--c", type=int, default=4096)
    p.add_argument("--dtype", default="bf16", choices=["f32", "bf16"])
    p.add_argument("--kinds", default="exact,proposed")
    p.add_argument("--reps", type=int, default=1)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--solve", default=None, choices=[None, "exact", "previous", "proposed"],
                   help="instead of single launches: one warm-up and one timed solve")
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--vr", type=int, default=4)
    a = p.parse_args()
    g = torch.Generator(device="cuda").manual_seed(a.seed)
    At = torch.randn(a.n, a.m, device="cuda", generator=g)
    At *= torch.randn(a.n, 1, device="cuda", generator=g).exp()
    A = At.t() if a.dtype == "f32" else At.to(torch.bfloat16).t()
    del At
    es = 4 if a.dtype == "f32" else 2
    if a.solve:
        ctx = AMMContext(a.m, a.n, c=a.c, step=a.steps, vr_period=a.vr, dtype=a.dtype)
        x0 = torch.randn(a.m, device="cuda", generator=g)
        gs = torch.Generator().manual_seed(a.seed + 7)
        states = torch.randint(1, 2**31 - 1, (a.c,), generator=gs, dtype=torch.int64)
        states = states.to(torch.int32).cuda()
        for rep in range(2):
            ctx.set_rng_state(states)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            ctx.set_matrix(A)
            ctx.power_method(a.solve, x0)
            e1.record()
            e1.synchronize()
            tr = ctx.trace()
            steps_us = np.diff(np.concatenate([[0.0], tr["t_ns"]])) / 1e3
            print(f"solve {a.solve} rep {rep}: {e0.elapsed_time(e1):.3f} ms, kinds {tr['kinds']}, "
                  f"distinct {tr['distinct'].tolist()}, step us (device clock) "
                  f"{np.round(steps_us, 1).tolist()}")
        # device-clock timeline of one more solve: stamps before set_matrix, after it, and after
        # the call, against the call's own stamps (end of its first kernel, end of each step)
        ctx.set_rng_state(states)
        stamps = torch.zeros(3, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        ctx.device_clock(stamps[0:1])
        ctx.set_matrix(A)
        ctx.device_clock(stamps[1:2])
        ctx.power_method(a.solve, x0)
        ctx.device_clock(stamps[2:3])
        clk = ctx.step_clocks()
        s0, s1, s2 = (int(v) for v in stamps.cpu())
        print(f"timeline us: set_matrix (host, GPU idle) {(s1 - s0) / 1e3:.1f}; set-up + CDF + "
              f"call start {(int(clk[0]) - s1) / 1e3:.1f}; steps {(int(clk[-1]) - int(clk[0])) / 1e3:.1f}; "
              f"call end {(s2 - int(clk[-1])) / 1e3:.1f}; total {(s2 - s0) / 1e3:.1f}")
        ctx.close()
        return
    ctx = AMMContext(a.m, a.n, c=a.c, step=2, dtype=a.dtype)
    print("geometry", ctx.geometry())
    ctx.set_matrix(A)
    ctx.set_rng_state(torch.arange(1, a.c + 1, dtype=torch.int32, device="cuda") * 2654435761 % (2**31))
    x0 = torch.randn(a.m, device="cuda", generator=g)
    ctx.power_method("proposed", x0)
    ctx.trace()
    for kind in a.kinds.split(","):
        ms, cd = ctx.benchmark_product(kind, reps=a.reps)
        byts = a.m * cd * es + (0 if kind in ("exact", "setup") else 8 * a.c) + 16 * a.m
        print(f"{kind:9s} dtype={a.dtype} m={a.m} n={a.n} c={a.c}: {ms * 1e3:9.2f} us/launch, "
              f"{cd} columns, {byts / ms / 1e6:8.1f} GB/s algorithmic")
    ctx.close()


if __name__ == "__main__":
    main()
