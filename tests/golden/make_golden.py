"""Generates the golden fixtures tests/golden/*.npz from the CPU oracle.

Run from the repository root:  python -m tests.golden.make_golden
Each fixture is a small seeded case advanced a few steps; the GPU parity
tests compare the CUDA path against them, and test_oracle checks that the
oracle still reproduces them.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from hicar_b200 import synth

HERE = Path(__file__).resolve().parent


def cases(O):
    small2 = synth.config2(seed=7, nx=40, ny=36, nz=10)
    return {
        "mpdata_c1_small": (synth.config1(seed=1, nx=32, ny=28, nz=8), O.make_opts(), 3),
        "mpdata_c2_small": (small2, O.make_opts(), 2),
        "mpdata_nofct": (synth.config1(seed=2, nx=24, ny=20, nz=6), O.make_opts(mpdata_fct=0), 2),
        "mpdata_order3": (synth.config1(seed=3, nx=24, ny=20, nz=6), O.make_opts(mpdata_order=3), 2),
        "std_h3v3": (synth.config1(seed=4, nx=24, ny=20, nz=8), O.make_opts(advection=1, h_order=3, v_order=3), 2),
        "std_h5v5_fc": (synth.config1(seed=5, nx=26, ny=22, nz=10),
                        O.make_opts(advection=1, h_order=5, v_order=5, flux_corr=1), 2),
        "std_rk3_fc": (synth.config1(seed=6, nx=24, ny=20, nz=8),
                       O.make_opts(advection=1, h_order=3, v_order=3, flux_corr=1, rk3=1), 2),
    }


def main():
    from hicar_b200.build import build_oracle
    build_oracle()
    from oracle import oracle as O
    for name, (case, opts, nsteps) in cases(O).items():
        out = O.run_steps(case, opts, case.dt, nsteps)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
