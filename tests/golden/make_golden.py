"""Generate tests/golden/ref_golden.npz by running the REFERENCE's own kernels and drivers
(oracle/_ref/libamm_ref.so, built from the reference sources by oracle/Makefile) on the
seeded inputs of inputs.py.  Needs a CUDA device; run it on the GPU machine:

    python tests/golden/make_golden.py [out.npz]
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1] / "oracle"))

import inputs as I  # noqa: E402
import ref_harness as R  # noqa: E402


def main(out=HERE / "ref_golden.npz"):
    A = I.symmetric_matrix()
    st = I.states()
    x0 = I.start_vector()
    vstar = I.top_eigenvector(A)
    g = {}
    cdf, pst = I.pick_inputs()
    g["pick_idx"], g["pick_states"] = R.pick_index(cdf, pst)
    g["seed_states_42"] = R.seed_states(I.M, 42)
    g["x0_seed_1276"] = R.draw_x0(I.M, 1276)
    for k in ("previousAMM", "proposedAMM"):
        d = R.amm_steps(k, A, x0, st, c=I.C, nsteps=I.NSTEPS)
        for key, v in d.items():
            g[f"steps_{k}_{key}"] = v
        d = R.amm_steps(k, A, x0, st, c=I.M, nsteps=3, sanity=True)
        g[f"sanity_{k}_eigs"] = d["eigs"]
    runs = {
        "exact": dict(vr_period=0),
        "previousAMM": dict(vr_period=I.VR),
        "proposedAMM": dict(vr_period=I.VR),
        "proposedAMM_v2": dict(vr_period=I.VR),
        "previousAMM_adaptive": dict(vr_period=0, vr_thr=1e-3),
    }
    for name, kw in runs.items():
        kernel = name.replace("_adaptive", "")
        d = R.power_method(kernel, A, 1276, st, c=I.C, step=I.STEPS, vstar=vstar, **kw)
        for key, v in d.items():
            if key != "time_ms":
                g[f"run_{name}_{key}"] = v
    np.savez_compressed(out, **g)
    print(f"wrote {out} ({len(g)} arrays)")


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
