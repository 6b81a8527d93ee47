"""In-tree build of libicar_adv.so (sm_100a) and of the CPU oracle.

The CUDA library is compiled with nvcc straight for sm_100a; ``-fmad=false``
keeps every multiply and add separately rounded so the kernels reproduce
the reference's FP32 arithmetic bit for bit (division stays IEEE-rounded,
the nvcc default).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libicar_adv.so"
ORACLE_DIR = ROOT / "oracle"

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-fmad=false",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-v",
    "--extended-lambda",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libicar_adv.so")
    return cand


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "icar_adv.h"]


def build_cuda(force: bool = False, verbose: bool = False) -> Path:
    srcs = _sources()
    if LIB.exists() and not force:
        mtime = LIB.stat().st_mtime
        if all(s.stat().st_mtime <= mtime for s in srcs):
            return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", "-o", str(LIB), str(CSRC / "icar_adv.cu"), "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = PKG / "build.log"
    log.write_text(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stderr[-4000:])
        raise RuntimeError(f"nvcc failed (see {log})")
    if verbose:
        sys.stderr.write(res.stderr)
    return LIB


def build_oracle(force: bool = False, native: bool = False) -> Path:
    out = ORACLE_DIR / "liboracle.so"
    srcs = [ORACLE_DIR / "icar_adv_oracle.c", ORACLE_DIR / "oracle_body.inc"]
    if out.exists() and not force and not native:
        if all(s.stat().st_mtime <= out.stat().st_mtime for s in srcs):
            return out
    march = "-march=native" if native else "-march=x86-64-v3"
    cflags = f"-O3 {march} -fopenmp -fPIC -ffp-contract=off -fno-fast-math -std=c11 -Wall -Wno-unused-function"
    env = dict(os.environ)
    res = subprocess.run(["make", "-B" if (force or native) else "-s", "-C", str(ORACLE_DIR), f"CFLAGS={cflags}"],
                         capture_output=True, text=True, env=env)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("oracle build failed")
    return out


if __name__ == "__main__":
    build_cuda(force="--force" in sys.argv, verbose=True)
    build_oracle(force="--force" in sys.argv)
    print(LIB)
