"""The scheme's own FP32 rounding error: the FP32 oracle against the FP64
oracle (the same C restatement compiled in double) on the synthetic
configurations, with advect_density off (the configurations' setting) and
on.  Test infrastructure: it measures the reference scheme, not the GPU
kernels.  Prints, per case, the worst field's max relative error (floor
1e-6 * max|q|; over all levels and below the top 8), its 99.9th
percentile, max |difference| / max|q|, and the count of negative FP32
values.

    OMP_NUM_THREADS=16 python oracle/fp32_vs_fp64.py [c1] [c2] [c5]
"""
import sys
import time
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
from hicar_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def compare(name, case, steps, advect_density):
    for n in steps:
        t = time.time()
        opts = O.make_opts(advect_density=advect_density)
        r32 = O.run_steps(case, opts, case.dt, n)
        r64 = O.run_steps(case, opts, case.dt, n, dtype=np.float64)
        res = {}
        for k in r32:
            a, b = r32[k].astype(np.float64), r64[k]
            scale = max(float(np.abs(b).max()), 1e-30)
            d = np.abs(a - b)
            rel = d / np.maximum(np.abs(b), 1e-6 * scale)
            below = float(rel[:, : max(case.nz - 8, 1), :].max())   # levels below the top 8
            res[k] = (float(rel.max()), float(np.quantile(rel, 0.999)), float(d.max() / scale), int((a < 0).sum()),
                      below)
        worst = lambda i: max(v[i] for v in res.values())
        print(f"{name} advect_density={advect_density} {n} steps ({time.time() - t:.0f} s): max rel {worst(0):.2e} "
              f"({worst(4):.2e} below the top 8 levels), p99.9 {worst(1):.2e}, max abs/max {worst(2):.2e}, "
              f"negative cells {sum(v[3] for v in res.values())}", flush=True)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c2", "c5"]
    for ad in (0, 1):
        if "c1" in which:
            compare("config 1", synth.config1(seed=11), (1, 100), ad)
        if "c5" in which:
            compare("config 5 generator 512x512x60", synth.config5(seed=3, nx=512, ny=512, nz=60), (1, 5), ad)
        if "c2" in which:
            compare("config 2", synth.config2(seed=2), (1, 100), ad)
