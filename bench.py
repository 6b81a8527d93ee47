#!/usr/bin/env python3
"""Benchmark of the ICAR tracer-advection step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload full_species|plain_c1]

A step is one model time step of the advected fields: the relaxation-zone
boundary update (fixed inflow forcing) followed by MPDATA order 2 with the
FCT limiter for every species.  Default workload: the full-species single
domain (512x512x40, 12 advected FP32 fields, dt 4 s, seeded synthetic
inputs).  Each rank advances its own replica (independent domains; the path
has no exchange step), so value = all ranks' cell-species updates / max time.

Prints one JSON line (rank 0).  `value` is device time of the resident step
(inputs already in HBM); `e2e` drives the same step through the C ABI with
pinned host buffers, copying every species in and out each step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "MPDATA cell-species updates/s"
UNIT = "cell-species updates/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="full_species", choices=["full_species", "plain_c1", "mid_species"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--staged", action="store_true", help="use the staged kernels instead of the fused one")
    p.add_argument("--quick", action="store_true",
                   help="timed region only (no e2e, no CPU baseline): the profiling run")
    return p.parse_args()


def make_case(workload: str, seed: int):
    from hicar_b200 import synth
    if workload == "plain_c1":
        return synth.config1(seed=seed), "plain MPDATA single domain 128x128x20, 1 field (qv), dt 20 s"
    if workload == "mid_species":
        return (synth.config2(seed=seed, nx=256, ny=256, nz=40),
                "full-species domain at quarter area 256x256x40, 12 fields, dt 4 s (profiling case)")
    return synth.config2(seed=seed), "full-species single domain 512x512x40, 12 fields, dt 4 s"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- CPU oracle
def cpu_rate(case, steps: int, threads: int) -> tuple[float, float]:
    """Cell-species updates/s of the oracle (C restatement, OpenMP) on case."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from hicar_b200.build import build_oracle
    build_oracle()
    from oracle import oracle as O
    opts = O.make_opts()
    O.advect(case, opts, case.dt)  # warm (page-in, thread pool)
    t0 = time.perf_counter()
    c = case
    for _ in range(steps):
        c.species = O.advect(c, opts, c.dt)
    dt = time.perf_counter() - t0
    return case.cells() * len(case.species) * steps / dt, dt


def cpu_sample(case, rows: int):
    """A y-slab of the workload's domain: the first `rows` rows."""
    from hicar_b200 import synth
    c = case.copy()
    ny = rows
    c.ny = ny
    for k in ("u", "w", "density", "jacobian", "jacobian_u", "jacobian_w", "advection_dz", "z"):
        setattr(c, k, np.ascontiguousarray(getattr(case, k)[:ny]))
    for k in ("v", "jacobian_v"):
        setattr(c, k, np.ascontiguousarray(getattr(case, k)[:ny + 1]))
    c.terrain = np.ascontiguousarray(case.terrain[:ny])
    c.species = {k: np.ascontiguousarray(v[:ny]) for k, v in case.species.items()}
    return c


def run_reference(args):
    """--impl reference: the oracle port of the reference's CPU advection on
    this host's cores, on a bounded y-slab sample of the workload per step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    case, desc = make_case(args.workload, 100)
    rows = 16 if args.workload == "full_species" else case.ny
    sample = cpu_sample(case, rows)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from hicar_b200.build import build_oracle
    build_oracle()
    from oracle import oracle as O
    opts = O.make_opts()
    c = sample
    for _ in range(args.warmup):
        c.species = O.advect(c, opts, c.dt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        c.species = O.advect(c, opts, c.dt)
    el = time.perf_counter() - t0
    cs = sample.cells() * len(sample.species)
    val = cs * args.steps / el
    samp = f"{sample.nx}x{sample.ny}x{sample.nz} slab of the {desc.split(',')[0]}, {len(sample.species)} fields"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "scheme": "MPDATA order 2 + FCT"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": samp},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------- GPU arm
def run_b200(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    from hicar_b200 import _lib as L
    from hicar_b200.advection import Domain, Options, adv_init

    lib = L.load()
    case, desc = make_case(args.workload, 100 + rank)
    S = len(case.species)
    cells = case.cells()
    opts = Options()
    d = Domain.from_case(case, device=local)
    for k, q in case.species.items():
        d.set_forcing(k, q.copy(), None)            # fixed inflow: forcing = initial state, dqdt = 0
    adv_init(d, opts)
    if args.staged:
        d.use_staged_kernels(True)
    # a dedicated stream: the library and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(stream.cuda_stream)), d.handle)
    h = d.handle

    def step():
        L.check(lib.icar_adv_step(h, C.c_double(case.dt), 0), h)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- resident timed region --------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    L.check(lib.icar_adv_profile(h, 1), h)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    kms, klaunch, alll, passes = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
    L.check(lib.icar_adv_profile_read(h, C.byref(kms), C.byref(klaunch), C.byref(alll), C.byref(passes)), h)
    L.check(lib.icar_adv_profile(h, 0), h)
    t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = cells * S * args.steps * world / (ms_max / 1e3)

    # ---- roofline of the species kernels ------------------------------
    from hicar_b200 import roofline
    rl = roofline.species_pass(case.nx, case.ny, case.nz, S, kms.value, passes.value)

    # ---- end to end through the C ABI with pinned host buffers ---------
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "quick": True,
                              "ms_per_step": ms_max / args.steps, "roofline": rl}), flush=True)
        d.close()
        if world > 1:
            dist.destroy_process_group()
        return
    host = {k: torch.from_numpy(v.copy()).pin_memory() for k, v in case.species.items()}
    ids = {k: L.SPECIES_IDS[k] for k in case.species}
    e2e_steps = max(3, min(args.steps, 20))

    def e2e_step():
        for k, tns in host.items():
            L.check(lib.icar_adv_set_field(h, ids[k], C.c_void_p(tns.data_ptr()), None), h)
        step()
        for k, tns in host.items():
            L.check(lib.icar_adv_get_field(h, ids[k], C.c_void_p(tns.data_ptr()), None), h)

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    t = torch.tensor([e2e_s], device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_val = cells * S * e2e_steps * world / float(t.item())
    bytes_io = cells * S * 4

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = cpu_sample(case, 16 if args.workload == "full_species" else case.ny)
        rate, el = cpu_rate(sample, 4, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{sample.nx}x{sample.ny}x{sample.nz} slab of the workload, {S} fields, 4 steps, "
                         f"{el:.1f} s (C restatement, OpenMP)"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "scheme": "MPDATA order 2 + FCT, relaxation boundary update",
                       "kernel_path": "staged" if args.staged else "fused",
                       "l2": "inputs larger than L2 (12 fields x 42 MB per domain)",
                       "parallelism": f"replicas x{world}"},
            "roofline": rl,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
                    "steps": e2e_steps},
            "gpu_launches": int(alll.value),
            "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    d.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
