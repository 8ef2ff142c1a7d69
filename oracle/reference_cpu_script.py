"""Run the reference's CPU baseline script unchanged on the 1024 x 4096 configuration.

Test infrastructure (a recipe, like ``oracle/Makefile``): the reference's
``calculate_largest_eigenvalue.py`` reads ``matrix.dat`` (square float32 C, no header) from its
working directory and prints the largest and smallest eigenvalue of C by FP64 LAPACK ``eigh``.
This writes C = A·Aᵀ for the bench's small exact case (A 1024 x 4096 FP32, N(0,1) entries times
lognormal(0, 1) column scales from seed 0, as ``bench.py`` builds it) into a temporary directory,
runs the script there ``--reps`` times with the interpreter this runs under, and prints one JSON
line: the script's λ_max, the FP64 λ_max of the same float32 C computed here, and the wall
times (each run includes interpreter start-up and the numpy import, as running the script does).

    REF=<reference checkout> python oracle/reference_cpu_script.py --reps 5

The reference checkout is taken from ``REF`` (or ``--ref``); there is no default.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np


def c1_matrix() -> np.ndarray:
    g = np.random.default_rng(0)
    A = (g.standard_normal((1024, 4096)) * g.lognormal(0.0, 1.0, 4096)).astype(np.float32)
    return (A.astype(np.float64) @ A.astype(np.float64).T).astype(np.float32)


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--ref", default=os.environ.get("REF"))
    p.add_argument("--reps", type=int, default=5)
    a = p.parse_args()
    if not a.ref:
        sys.exit("set REF (or --ref) to the reference checkout")
    script = Path(a.ref) / "calculate_largest_eigenvalue.py"
    if not script.exists():
        sys.exit(f"{script} not found")
    C = c1_matrix()
    lam64 = float(np.linalg.eigvalsh(C.astype(np.float64))[-1])
    walls, lam_script = [], None
    with tempfile.TemporaryDirectory() as td:
        C.tofile(os.path.join(td, "matrix.dat"))
        for _ in range(a.reps):
            t0 = time.perf_counter()
            out = subprocess.run([sys.executable, str(script)], cwd=td, check=True,
                                 capture_output=True, text=True).stdout
            walls.append(time.perf_counter() - t0)
            m = re.search(r"Largest eigenvalue\s*=\s*([-0-9.eE+]+)", out)
            lam_script = float(m.group(1))
        t0 = time.perf_counter()
        subprocess.run([sys.executable, "-c", "import numpy"], check=True)
        startup = time.perf_counter() - t0
    print(json.dumps({
        "workload": "calculate_largest_eigenvalue.py unchanged, matrix.dat = float32 C = A·Aᵀ, "
                    "A 1024 x 4096 (seed 0)",
        "lambda_script": lam_script, "lambda_fp64_here": lam64,
        "rel_diff": abs(lam_script - lam64) / lam64,
        "wall_s_median": statistics.median(walls), "wall_s_min": min(walls),
        "interpreter_and_numpy_import_s": startup, "reps": a.reps,
        "cpu_threads": os.cpu_count()}))


if __name__ == "__main__":
    main()
