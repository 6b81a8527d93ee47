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
# --kernel -> icar_adv_set_path / icar_adv_batch_set_path
KERNEL_PATH = {"two-pass": 0, "single-pass": 2, "single-pass-fast": 3}
UNIT = "cell-species updates/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="full_species",
                   choices=["full_species", "plain_c1", "mid_species", "ensemble", "served", "large", "wind", "mp",
                            "std"])
    p.add_argument("--serve-rate", type=float, default=20.0)
    p.add_argument("--serve-duration", type=float, default=20.0)
    p.add_argument("--serve-steps-scale", type=float, default=0.1)
    p.add_argument("--members", type=int, default=64, help="ensemble size (ensemble workload)")
    p.add_argument("--tile-shape", default="auto", choices=["auto", "0", "1", "2", "3"],
                   help="fused-kernel tile shape 0..3 (8/15/24/31 rows), or auto: chosen by hicar_b200.autotune")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--staged", action="store_true", help="use the staged kernels instead of the fused one")
    p.add_argument("--kernel", default="single-pass-fast", choices=["two-pass", "single-pass", "single-pass-fast"],
                   help="MPDATA kernels: the donor-cell kernel then the fused correction (two-pass), or the "
                        "single-pass kernel with bit-exact or fast arithmetic")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the sub-records of the default line (bit-exact kernels, drift, batched, served)")
    p.add_argument("--drift-steps", type=int, default=200, help="steps of the drift record (blocks of 20)")
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
def cpu_rate(case, threads: int, target_s: float = 10.0, max_steps: int = 200,
             scheme: dict | None = None, min_steps: int = 2) -> tuple[float, float, int]:
    """Cell-species updates/s of the oracle (C restatement, OpenMP) on case:
    whole steps until about target_s seconds of CPU work (at least
    min_steps, at most max_steps).
    scheme: make_opts keywords (default MPDATA order 2 + FCT).
    Returns (rate, seconds, steps)."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from hicar_b200.build import build_oracle
    build_oracle()
    from oracle import oracle as O
    opts = O.make_opts(**(scheme or {}))
    O.advect(case, opts, case.dt)  # warm (page-in, thread pool)
    t0 = time.perf_counter()
    c, steps = case, 0
    while steps < max_steps and (steps < 2 or time.perf_counter() - t0 < target_s or steps < min_steps):
        c.species = O.advect(c, opts, c.dt)
        steps += 1
    dt = time.perf_counter() - t0
    return case.cells() * len(case.species) * steps / dt, dt, steps


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
    this host's cores, on the same whole domain as the GPU arm (one step of
    the 512x512x40 x 12-field workload is about 1.4 s on 16 host threads)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    case, desc = make_case(args.workload, 100)
    sample = case
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from hicar_b200.build import build_oracle
    build_oracle()
    from oracle import oracle as O
    opts = O.make_opts()
    c = sample
    # the same step as the GPU arm: fixed-inflow relaxation update
    # (forcing = initial state, dqdt = 0), then advect
    flt = O.init_relax_filters(c.nx, c.ny, 2)
    forcing = {k: (q.copy(), np.zeros_like(q)) for k, q in c.species.items()}

    def one_step():
        for k, (fh, dq) in forcing.items():
            O.apply_forcing(c.species[k], fh, dq, flt, c.dt)
        c.species = O.advect(c, opts, c.dt)

    # one untimed step pages the arrays in and starts the thread pool; more
    # CPU warm-up would only lengthen the run (1-2 s per step).  The timed
    # steps are whole steps of the whole domain, as many of the requested K
    # as fit in about 150 s, so the run ends within a few minutes.
    tw = time.perf_counter()
    for _ in range(min(args.warmup, 1)):
        one_step()
    t_step = (time.perf_counter() - tw) / max(min(args.warmup, 1), 1)
    n_timed = max(1, min(args.steps, int(150.0 / max(t_step, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(n_timed):
        one_step()
    el = time.perf_counter() - t0
    cs = sample.cells() * len(sample.species)
    val = cs * n_timed / el
    samp = (f"the whole {sample.nx}x{sample.ny}x{sample.nz} domain, {len(sample.species)} fields, every step "
            f"(C restatement with OpenMP over rows in every stage; the reference threads only the FCT sweep)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "warmup_steps_run": min(args.warmup, 1),
        "steps_timed": n_timed, "ms_per_step": el / n_timed * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "scheme": "MPDATA order 2 + FCT, relaxation boundary update",
                   "same_config": True},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": samp},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# --------------------------------------------------------------- GPU arm
def run_b200(args):
    import torch

    from hicar_b200 import _lib as L, replicas as R
    from hicar_b200.advection import Domain, Options, adv_init

    rk = R.from_env()
    world, rank, local = rk.world, rk.rank, rk.local
    torch.cuda.set_device(local)
    R.init(rk, "nccl")
    lib = L.load()
    case, desc = make_case(args.workload, R.replica_seed(100, rk))
    S = len(case.species)
    cells = case.cells()
    opts = Options()
    d = Domain.from_case(case, device=local)
    for k, q in case.species.items():
        d.set_forcing(k, q.copy(), None)            # fixed inflow: forcing = initial state, dqdt = 0
    adv_init(d, opts)
    path = 1 if args.staged else KERNEL_PATH[args.kernel]
    launch = set_launch_shape(d, args) if path == 0 else (
        {"kernel": "staged"} if path == 1 else {"kernel": args.kernel, "tile": "56 x 26 columns per CTA, 16 warps"})
    d.set_path(path)
    # a dedicated stream: the library and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(stream.cuda_stream)), d.handle)
    h = d.handle

    def step():
        L.check(lib.icar_adv_step(h, C.c_double(case.dt), 0), h)

    def barrier():
        R.barrier(rk)

    def timed_steps(n):
        """Device time (ms) of n steps, CUDA events on the library's stream."""
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # ---- resident timed region --------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    L.check(lib.icar_adv_profile(h, 1), h)
    ms = timed_steps(args.steps)
    clk = clocks.stop()
    kms, klaunch, alll, passes = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
    L.check(lib.icar_adv_profile_read(h, C.byref(kms), C.byref(klaunch), C.byref(alll), C.byref(passes)), h)
    cms, claunch = C.c_double(), C.c_int64()
    L.check(lib.icar_adv_profile_read_correction(h, C.byref(cms), C.byref(claunch)), h)
    L.check(lib.icar_adv_profile(h, 0), h)
    L.check(lib.icar_adv_sync(h), h)
    ms_max = R.max_over_ranks(rk, ms)
    value = R.whole_job_rate(cells * S * args.steps, world, ms_max / 1e3)

    # ---- roofline of the dominant kernel and of the whole advect call ---
    from hicar_b200 import roofline
    step_rl = roofline.species_pass(case.nx, case.ny, case.nz, S, kms.value, passes.value)
    if claunch.value > 0 and path >= 2:
        rl = roofline.single_pass_kernel(case.nx, case.ny, case.nz, S, cms.value, claunch.value)
        rl["advect_call"] = step_rl
    elif claunch.value > 0:
        rl = roofline.correction_kernel(case.nx, case.ny, case.nz, S, cms.value, claunch.value)
        rl["advect_call"] = step_rl
    else:                                       # staged path: the whole advect call
        rl = step_rl

    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "quick": True,
                              "ms_per_step": ms_max / args.steps, "roofline": rl}), flush=True)
        d.close()
        R.finalize(rk)
        return

    extras = {}
    if not args.no_extras:
        # ---- the bit-exact kernels on the same workload (same state) ----
        if path != 0:
            d.set_path(0)
            for _ in range(2):
                step()
            ems = R.max_over_ranks(rk, timed_steps(args.steps))
            extras["exact"] = {
                "value": R.whole_job_rate(cells * S * args.steps, world, ems / 1e3), "unit": UNIT,
                "ms_per_step": ems / args.steps, "steps": args.steps,
                "kernel": "two-pass (donor-cell kernel + fused correction), the reference's FP32 arithmetic, "
                          "bit-identical to the oracle"}
            d.set_path(path)
        # ---- drift: the step cost as the fields evolve, from the initial state
        for k, q in case.species.items():
            d.upload(k, q)
        blocks, nb = [], max(1, args.drift_steps // 20)
        for _ in range(nb):
            blocks.append(R.max_over_ranks(rk, timed_steps(20)) / 20)
        extras["drift"] = {"steps": 20 * nb, "block": 20, "ms_per_step_first": blocks[0],
                           "ms_per_step_last": blocks[-1], "ms_per_step_blocks": blocks,
                           "from": "the initial state", "kernel": args.kernel if path >= 2 else "two-pass"}

    # ---- end to end through the C ABI with pinned host buffers ---------
    host = {k: torch.from_numpy(v.copy()).pin_memory() for k, v in case.species.items()}
    ids = {k: L.SPECIES_IDS[k] for k in case.species}
    e2e_steps = max(3, min(args.steps, 20))
    ptrs = (C.c_void_p * S)(*[host[k].data_ptr() for k in d.adv_vars])

    def e2e_step():
        # the whole step from and to page-locked host arrays in one C-ABI call
        L.check(lib.icar_adv_step_host(h, C.c_double(case.dt), 0, ptrs, ptrs), h)

    def e2e_step_per_field():
        for k, tns in host.items():
            L.check(lib.icar_adv_set_field(h, ids[k], C.c_void_p(tns.data_ptr()), None), h)
        step()
        for k, tns in host.items():
            L.check(lib.icar_adv_get_field(h, ids[k], C.c_void_p(tns.data_ptr()), None), h)

    def e2e_time(fn):
        fn()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            fn()
        torch.cuda.synchronize()
        return R.max_over_ranks(rk, time.perf_counter() - t0)

    e2e_s = e2e_time(e2e_step)
    e2e_val = R.whole_job_rate(cells * S * e2e_steps, world, e2e_s)
    e2e_pf = R.whole_job_rate(cells * S * e2e_steps, world, e2e_time(e2e_step_per_field))
    bytes_io = cells * S * 4
    d.close()

    if not args.no_extras and world == 1:
        # ---- the metric's batched and served forms (config 3 and 4) ------
        ens = ensemble_core(args, rk, args.kernel if path >= 2 else "two-pass", want_e2e=False, want_cpu=False)
        ens["workload"] = ENSEMBLE_DESC
        extras["batched"] = ens
        srv = served_core(args, args.kernel if path >= 2 else "two-pass")
        extras["served"] = {"workload": srv["workload"], **srv["report"], "clocks": srv["clocks"]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample = case.copy()
        rate, el, nst = cpu_rate(sample, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"the whole {sample.nx}x{sample.ny}x{sample.nz} domain, {S} fields, {nst} steps, "
                         f"{el:.1f} s (C restatement, OpenMP over all host threads)"}

    if rank == 0:
        arith = ("fast: hardware reciprocal approximation, fused multiply-adds; within the tested tolerance of "
                 "the reference's FP32 results (see icar_adv_set_path)" if path == 3 else
                 "the reference's FP32 arithmetic, bit-identical to the oracle")
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "scheme": "MPDATA order 2 + FCT, relaxation boundary update",
                       "kernel_path": "staged" if args.staged else args.kernel,
                       "arithmetic": arith,
                       "launch_shape": launch,
                       "l2": "inputs larger than L2 (12 fields x 42 MB per domain)",
                       "parallelism": f"replicas x{world}"},
            "roofline": rl,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io,
                    "steps": e2e_steps, "call": "icar_adv_step_host (uploads, step and downloads overlapped by species group)",
                    "per_field_calls_value": e2e_pf},
            "gpu_launches": int(alll.value),
            "clocks": clk,
        }
        out.update(extras)
        print(json.dumps(out), flush=True)
    R.finalize(rk)


def set_launch_shape(d, args) -> dict:
    """Tile shape and species group of the fused kernels for this domain."""
    from hicar_b200 import autotune
    if args.tile_shape == "auto" and not args.staged and args.kernel == "two-pass":
        c = autotune.tune_and_apply(d, fct=True)
        return {"tile_rows": c.rows, "species_group": c.species_group,
                "chosen_by": "autotune: every shape and group timed on a synthetic domain of this grid shape"}
    shape = 1 if args.tile_shape == "auto" else int(args.tile_shape)
    d.set_launch_shape(shape, 0)
    return {"tile_rows": autotune.TILE_ROWS[shape], "species_group": 0, "chosen_by": "--tile-shape"}


# ------------------------------------------------------------ large domain
LARGE_DESC = "large single domain 2048x2048x60, dx 250 m, fractal terrain up to 4000 m, 12 fields, dt 1 s"


def run_large(args):
    """The large single domain, generated on the device.  Every arm starts
    from the same saved initial state: the default launch shape of the
    two-pass kernels, each autotuner candidate, the autotuned shape, and the
    single-pass fast kernel."""
    import torch
    from hicar_b200 import _lib as L, autotune, replicas as R, roofline, synth
    from hicar_b200.advection import Domain, Options

    if not R.from_env().is_root:
        return                                   # a single domain on one GPU: the other ranks have no work
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    nx, ny, nz = 2048, 2048, 60
    fields, dt = synth.device_config5(seed=3, nx=nx, ny=ny, nz=nz, device=local)
    opts = Options()
    d = Domain.create_on_device(fields, nx, ny, nz, 250.0, opts, device=local, forcing=True)
    d._device_fields = None
    del fields
    torch.cuda.empty_cache()
    lib = L.load()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(stream.cuda_stream)), d.handle)
    h = d.handle
    S = len(d.adv_vars)
    cs = nx * ny * nz * S
    # the initial state, restored before every arm so that each is timed on
    # the same fields (the cost of a step depends on the state)
    saved = {}
    for k in d.adv_vars:
        t = torch.empty(nx * ny * nz, dtype=torch.float32, device=f"cuda:{local}")
        d.fetch_device(k, t)
        saved[k] = t
    torch.cuda.synchronize()

    def restore():
        for k, t in saved.items():
            L.check(lib.icar_adv_set_field_device(h, L.SPECIES_IDS[k], C.c_void_p(t.data_ptr())), h)

    def step():
        L.check(lib.icar_adv_step(h, C.c_double(dt), 0), h)

    def timed(steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        L.check(lib.icar_adv_profile(h, 1), h)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        kms, kl, al, ps = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
        L.check(lib.icar_adv_profile_read(h, C.byref(kms), C.byref(kl), C.byref(al), C.byref(ps)), h)
        cms, cl = C.c_double(), C.c_int64()
        L.check(lib.icar_adv_profile_read_correction(h, C.byref(cms), C.byref(cl)), h)
        L.check(lib.icar_adv_profile(h, 0), h)
        return e0.elapsed_time(e1), (kms.value, ps.value, cms.value, cl.value), al.value

    def arm(path, shape=1, group=0, steps=None):
        restore()
        d.set_path(path)
        d.set_launch_shape(shape, group)
        for _ in range(args.warmup):
            step()
        return timed(steps or args.steps)

    ms_plain, _, _ = arm(0, 1, 0)
    measured = {}
    for shape in range(len(autotune.TILE_ROWS)):
        for group in autotune.species_groups(S):
            measured[f"{shape}:{group}"] = arm(0, shape, group, steps=2)[0] / 2
    best = min(measured, key=measured.get)
    shape, group = (int(v) for v in best.split(":"))
    ms_tuned, _, _ = arm(0, shape, group)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    ms, (kms, passes, cms, cl), launches = arm(3)
    clk = clocks.stop()
    rl = roofline.single_pass_kernel(nx, ny, nz, S, cms, cl)
    rl["advect_call"] = roofline.species_pass(nx, ny, nz, S, kms, passes)
    dev_bytes = d.device_bytes()
    d.close()
    del saved
    torch.cuda.empty_cache()
    cpu = None
    if not args.no_cpu_baseline:
        # the oracle for 5 steps on a 512 x 512 domain from the same generator
        # (dx, levels, terrain statistics, winds, 12 fields): the whole
        # domain would need about 40 GB of host memory and minutes per step
        threads = os.cpu_count() or 1
        sample = synth.config5(seed=3, nx=512, ny=512, nz=nz)
        rate, el, nst = cpu_rate(sample, threads, target_s=0.0, max_steps=5, min_steps=5)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{sample.nx}x{sample.ny}x{sample.nz} domain from the same generator, {S} fields, "
                         f"{nst} steps, {el:.1f} s (C restatement, OpenMP over all host threads)"}
    print(json.dumps({
        "metric": METRIC, "value": cs * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (generated on the device)",
        "config": {"workload": LARGE_DESC, "scheme": "MPDATA order 2 + FCT, relaxation boundary update",
                   "kernel": "single-pass-fast",
                   "state": "every arm starts from the same saved initial state",
                   "l2": "inputs larger than L2 (12 fields x 1 GB)"},
        "plain": {"value": cs * args.steps / (ms_plain / 1e3), "ms_per_step": ms_plain / args.steps,
                  "kernel": "two-pass", "launch_shape": {"tile_rows": autotune.TILE_ROWS[1], "species_group": 0}},
        "autotuned": {"value": cs * args.steps / (ms_tuned / 1e3), "ms_per_step": ms_tuned / args.steps,
                      "kernel": "two-pass",
                      "launch_shape": {"tile_rows": autotune.TILE_ROWS[shape], "species_group": group,
                                       "chosen_by": "autotune: every combination timed on this domain, "
                                                    "each from the saved state"}},
        "autotuned_over_plain": ms_plain / ms_tuned,
        "single_pass_over_plain": ms_plain / ms,
        "autotune_ms_per_step": measured,
        "device_bytes": dev_bytes,
        "roofline": rl, "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk}), flush=True)


# ------------------------------------------------------------ wind balance
def run_wind(args):
    """balance_uvw and compute_dt (the per-step wind operations beside
    advection) on the full-species domain, each timed with CUDA events on
    the library's stream, against the HBM roofline of their bytes."""
    import torch
    from hicar_b200 import _lib as L, replicas as R, roofline
    from hicar_b200.advection import Domain, Options, Parameters, adv_init, balance_uvw

    if not R.from_env().is_root:
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    case, desc = make_case("full_species", 100)
    opts = Options(parameters=Parameters(advect_density=True))
    d = Domain.from_case(case, device=local)
    adv_init(d, opts)
    lib = L.load()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(stream.cuda_stream)), d.handle)
    dz = np.ascontiguousarray(case.dz_levels, np.float32)
    dzp = dz.ctypes.data_as(C.POINTER(C.c_float))
    out = C.c_float()

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def dt_device_only():
        # the maxima kernel alone: icar_adv_compute_dt also copies 16 bytes back and waits
        L.check(lib.icar_adv_compute_dt(d.handle, dzp, C.c_float(0.9), 3, 0, C.byref(out)), d.handle)

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    ms_bal = timed(lambda: balance_uvw(d, opts), args.steps)
    t0 = time.perf_counter()
    for _ in range(20):
        dt_device_only()
    ms_dt_host = (time.perf_counter() - t0) / 20 * 1e3
    clk = clocks.stop()
    cells = case.cells()
    peak, kind = roofline.hbm_peak()
    bal_bytes = cells * 32.0                 # u, v, J_u, J_v, rho, dz, J_w read, w written (4 B each)
    dt_bytes = cells * 12.0                  # u, v, w read
    d.close()
    print(json.dumps({
        "metric": "wind balance cells/s", "value": cells / (ms_bal / 1e3), "unit": "cells/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_bal, "higher_is_better": True,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "balance_uvw (advect_density) and compute_dt on the " + desc},
        "roofline": {"kernel": "k_balance_uvw", "bound": "hbm", "achieved": bal_bytes / (ms_bal / 1e3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": bal_bytes / (ms_bal / 1e3) / 1e9 / peak,
                     "traffic": None, "peak_kind": kind, "algorithmic_bytes_per_launch": bal_bytes,
                     "bytes_model": "32 B per cell: seven input fields read and w written once"},
        "compute_dt": {"ms_per_call_host_synchronous": ms_dt_host, "algorithmic_bytes": dt_bytes,
                       "dt_seconds": out.value},
        "clocks": clk}), flush=True)


# ------------------------------------------------------------ microphysics
def run_mp(args):
    """The simple microphysics (mp_simple) on the full-species domain, timed
    with CUDA events on the library's stream, against the HBM roofline of
    its bytes; alone and as the advect -> mp pair with the species resident."""
    import torch
    from hicar_b200 import _lib as L, replicas as R, roofline, synth
    from hicar_b200.advection import Domain, Options, PhysicsOptions, adv_init, kMP_SB04

    if not R.from_env().is_root:
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    case, desc = make_case("full_species", 100)
    synth.add_mp_fields(case)
    opts = Options(physics=PhysicsOptions(microphysics=kMP_SB04))
    d = Domain.from_case(case, device=local)
    adv_init(d, opts)
    lib = L.load()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(stream.cuda_stream)), d.handle)
    h = d.handle

    def mp_call():
        L.check(lib.icar_adv_mp_simple(h, C.c_float(case.dt)), h)

    def pair():
        L.check(lib.icar_adv_advect(h, C.c_float(case.dt)), h)
        mp_call()

    def timed(fn, steps):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    ms_mp = timed(mp_call, args.steps)
    ms_pair = timed(pair, max(3, args.steps // 4))
    clk = clocks.stop()
    L.check(lib.icar_adv_sync(h), h)
    d.close()
    cells = case.cells()
    peak, kind = roofline.hbm_peak()
    mp_bytes = cells * 56.0     # pressure, th, exner, rho, qv, qc, qr, qs, dz read; th, qv, qc, qr, qs written
    print(json.dumps({
        "metric": "simple microphysics cells/s", "value": cells / (ms_mp / 1e3), "unit": "cells/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mp, "higher_is_better": True,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "mp_simple (SB04) on the " + desc + " (qv x1.5, hydrostatic pressure)"},
        "roofline": {"kernel": "k_mp_simple", "bound": "hbm", "achieved": mp_bytes / (ms_mp / 1e3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": mp_bytes / (ms_mp / 1e3) / 1e9 / peak, "traffic": None,
                     "peak_kind": kind, "algorithmic_bytes_per_launch": mp_bytes,
                     "bytes_model": "56 B per cell: nine fields read and five written once"},
        "advect_then_mp_ms": ms_pair, "clocks": clk}), flush=True)


# ------------------------------------------------------------ standard scheme
STD_SCHEME = {"advection": 1, "h_order": 5, "v_order": 3, "flux_corr": 1, "rk3": 1}


def run_std(args):
    """The standard scheme in HICAR's default setting (RK3, 5th-order
    horizontal and 3rd-order vertical fluxes, WRF monotonic flux
    correction) on the full-species domain: the fused kernels and the
    one-kernel-per-stage path, each timed with CUDA events on the library's
    stream, against the HBM roofline of the step's bytes; the oracle on a
    y-slab of the same domain as the CPU baseline."""
    import torch
    from hicar_b200 import _lib as L, replicas as R, roofline
    from hicar_b200.advection import AdvOptions, Domain, Options, PhysicsOptions, TimeOptions, adv_init

    if not R.from_env().is_root:
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    case, desc = make_case("full_species", 100)
    opts = Options(physics=PhysicsOptions(advection=1),
                   adv_options=AdvOptions(h_order=5, v_order=3, flux_corr=1), time_options=TimeOptions(RK3=True))
    S = len(case.species)
    lib = L.load()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    def timed(staged: bool, steps: int):
        d = Domain.from_case(case, device=local)
        adv_init(d, opts)
        if staged:
            d.use_staged_kernels(True)
        h = d.handle
        L.check(lib.icar_adv_set_stream(h, C.c_void_p(stream.cuda_stream)), h)
        for _ in range(args.warmup):
            L.check(lib.icar_adv_advect(h, C.c_float(case.dt)), h)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            L.check(lib.icar_adv_advect(h, C.c_float(case.dt)), h)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        # launch count of one more (profiled) round of steps
        L.check(lib.icar_adv_profile(h, 1), h)
        for _ in range(steps):
            L.check(lib.icar_adv_advect(h, C.c_float(case.dt)), h)
        kms, kl, alll, passes = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
        L.check(lib.icar_adv_profile_read(h, C.byref(kms), C.byref(kl), C.byref(alll), C.byref(passes)), h)
        L.check(lib.icar_adv_profile(h, 0), h)
        d.close()
        return ms, alll.value / steps

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    ms_fused, l_fused = timed(False, args.steps)
    ms_staged, l_staged = timed(True, max(3, args.steps // 4))
    clk = clocks.stop()
    cs = case.cells() * S
    peak, kind = roofline.hbm_peak()
    # three stages: q -> t1 (8 B), (t1, q) -> t2 (12 B), (t2, q) -> q (12 B) per cell-species;
    # per cell: prep reads 9 fields and writes 5 (56 B), each stage reads U_m, V_m, W_m, G, DJR (60 B)
    step_bytes = cs * 32.0 + case.cells() * 116.0
    line = {
        "metric": "standard-scheme cell-species updates/s", "value": cs / (ms_fused / 1e3),
        "unit": "cell-species updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_fused, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "standard scheme (RK3, h_order 5, v_order 3, WRF monotonic flux correction) on the "
                               + desc},
        "roofline": {"kernel": "k_std_prep + 3 x (k_std_ring + k_std_fused) per advect call", "bound": "hbm",
                     "achieved": step_bytes / (ms_fused / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": step_bytes / (ms_fused / 1e3) / 1e9 / peak, "traffic": None, "peak_kind": kind,
                     "algorithmic_bytes_per_launch": step_bytes,
                     "bytes_model": "32 B per cell-species (three RK3 stages) + 116 B per cell (prep, and the "
                                    "Courant and metric fields once per stage)"},
        "staged": {"ms_per_step": ms_staged, "value": cs / (ms_staged / 1e3), "launches_per_step": l_staged},
        "speedup_vs_staged": ms_staged / ms_fused, "gpu_launches_per_step": l_fused, "clocks": clk}
    if not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0))
        sample = cpu_sample(case, 16)
        rate, el, nst = cpu_rate(sample, threads, scheme=STD_SCHEME)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-species updates/s", "cores": threads, "kind": "port",
                                "sample": f"512x16x40 slab of the workload, 12 fields, {nst} steps, {el:.1f} s "
                                          "(C restatement, OpenMP)"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ ensemble
ENSEMBLE_DESC = ("batched uneven ensemble: 64 independent domains, nx,ny ~ U[64,384], nz ~ U[20,50], "
                 "12 fields each, dt 20 s, one graph launch per step vs 64 plain launches")


def _member(args):
    seed, nx, ny, nz = args
    from hicar_b200 import synth
    return synth.ensemble_member(seed, nx, ny, nz)


def make_ensemble(n: int, seed: int):
    """The members of the uneven ensemble, generated in parallel (spawned
    workers, so no CUDA state is inherited)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from hicar_b200 import synth
    shapes = synth.ensemble_shapes(n, seed)
    jobs = [(seed * 1000 + i, nx, ny, nz) for i, (nx, ny, nz) in enumerate(shapes)]
    workers = max(1, min(len(jobs), (os.cpu_count() or 2) - 1))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_member, jobs))


def ensemble_core(args, rk, kernel: str, want_e2e: bool, want_cpu: bool) -> dict:
    """The config-3 ensemble on this rank: plain (one member after another,
    each with its own launches) against batched (one step for every member,
    CUDA graph), both on the chosen kernels.  Returns the measurements."""
    import torch

    from hicar_b200 import _lib as L, replicas as R, roofline
    from hicar_b200.advection import Domain, Options, adv_init
    from hicar_b200.batch import Batch

    world, rank, local = rk.world, rk.rank, rk.local
    cases = make_ensemble(args.members, R.replica_seed(7, rk))
    lib = L.load()
    opts = Options()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    doms = []
    for c in cases:
        d = Domain.from_case(c, device=local)
        for k, q in c.species.items():
            d.set_forcing(k, q, None)           # fixed inflow boundaries
        adv_init(d, opts)
        L.check(lib.icar_adv_set_stream(d.handle, C.c_void_p(stream.cuda_stream)), d.handle)
        d.set_path(KERNEL_PATH[kernel])
        doms.append(d)
    cs_step = sum(c.cells() * len(c.species) for c in cases)

    def timed(fn, steps):
        R.barrier(rk)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        R.barrier(rk)
        return R.max_over_ranks(rk, e0.elapsed_time(e1))

    # ---- plain: one domain per launch sequence, members one after another
    def plain_step():
        for d, c in zip(doms, cases):
            L.check(lib.icar_adv_step(d.handle, C.c_double(c.dt), 0), d.handle)

    for _ in range(2):
        plain_step()
    plain_steps = max(3, args.steps // 4)
    plain_ms = timed(plain_step, plain_steps)
    plain_value = R.whole_job_rate(cs_step * plain_steps, world, plain_ms / 1e3)

    # ---- batched: every member in one graph launch per step
    b = Batch(device=local)
    b.set_stream(stream.cuda_stream)
    b.set_path(KERNEL_PATH[kernel])
    for d, c in zip(doms, cases):
        b.add(d, c.dt)
    shape = 1
    if kernel != "two-pass":
        pass                                    # the single-pass kernel has one tile shape
    elif args.tile_shape == "auto":
        from hicar_b200 import autotune
        shape = autotune.tune_batch(b)
    else:
        shape = int(args.tile_shape)
        b.set_tile_shape(shape)
    for _ in range(args.warmup):
        b.step()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.4)
    b.profile(True)
    ms = timed(b.step, args.steps)
    clk = clocks.stop()
    prof = b.profile_read()
    b.profile(False)
    b.sync()
    value = R.whole_job_rate(cs_step * args.steps, world, ms / 1e3)
    bytes_step = sum(c.cells() * (8 * len(c.species) + 32) for c in cases)
    peak, kind = roofline.hbm_peak()
    step_ms = prof["ms"] / max(prof["steps"], 1)
    achieved = bytes_step / (step_ms / 1e3) / 1e9
    rl = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
          "traffic": None, "peak_kind": kind, "algorithmic_bytes_per_launch": bytes_step, "launch_ms": step_ms,
          "bytes_model": "8 + 32/S B per cell-species; one launch = one batched step (graph)"}
    out = {"value": value, "ms_per_step": ms / args.steps, "steps": args.steps, "cell_species_per_step": cs_step,
           "members": len(cases), "kernel": kernel,
           "tile_shape_rows": [8, 15, 24, 31][shape] if kernel == "two-pass" else 26,
           "plain": {"value": plain_value, "steps": plain_steps, "ms_per_step": plain_ms / plain_steps,
                     "launches_per_step": len(cases) * (3 if kernel != "two-pass" else 4)},
           "batched_over_plain": value / plain_value, "roofline": rl,
           "gpu_launches": int(prof["kernels_per_step"] * prof["steps"]), "clocks": clk}

    if want_e2e:
        # host buffers in and out of every member every step
        host = [{k: torch.from_numpy(v.copy()).pin_memory() for k, v in c.species.items()} for c in cases]

        def e2e_step():
            for d, hb in zip(doms, host):
                for k, tns in hb.items():
                    L.check(lib.icar_adv_set_field(d.handle, L.SPECIES_IDS[k], C.c_void_p(tns.data_ptr()), None),
                            d.handle)
            b.step()
            for d, hb in zip(doms, host):
                for k, tns in hb.items():
                    L.check(lib.icar_adv_get_field(d.handle, L.SPECIES_IDS[k], C.c_void_p(tns.data_ptr()), None),
                            d.handle)

        e2e_step()
        R.barrier(rk)
        torch.cuda.synchronize()
        e2e_steps = 3
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = R.max_over_ranks(rk, time.perf_counter() - t0)
        out["e2e"] = {"value": R.whole_job_rate(cs_step * e2e_steps, world, e2e_s), "unit": UNIT,
                      "h2d_bytes_per_step": cs_step * 4, "d2h_bytes_per_step": cs_step * 4, "steps": e2e_steps}
    if want_cpu and rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        big = max(cases, key=lambda c: c.cells())
        rate, el, nst = cpu_rate(big.copy(), threads)
        out["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"largest member {big.nx}x{big.ny}x{big.nz}, 12 fields, {nst} steps, "
                                         f"{el:.1f} s (C restatement, OpenMP over all host threads)"}
    b.close()
    for d in doms:
        d.close()
    return out


def run_ensemble(args):
    from hicar_b200 import replicas as R
    import torch

    rk = R.from_env()
    torch.cuda.set_device(rk.local)
    R.init(rk, "nccl", timeout_s=600)
    r = ensemble_core(args, rk, args.kernel, want_e2e=not args.quick, want_cpu=not (args.quick or args.no_cpu_baseline))
    if rk.rank == 0:
        if args.quick:
            print(json.dumps({"metric": METRIC, "value": r["value"], "unit": UNIT, "quick": True,
                              "plain_value": r["plain"]["value"], "ms_per_step": r["ms_per_step"],
                              "roofline": r["roofline"]}), flush=True)
        else:
            out = {
                "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": rk.world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": ENSEMBLE_DESC, "members": r["members"],
                           "cell_species_per_step": r["cell_species_per_step"],
                           "scheme": "MPDATA order 2 + FCT, relaxation boundary update", "kernel": r["kernel"],
                           "tile_shape_rows": r["tile_shape_rows"],
                           "l2": "inputs larger than L2 (~6 GB of species per step)",
                           "parallelism": f"replicas x{rk.world}"},
                "plain": r["plain"], "batched_over_plain": r["batched_over_plain"], "roofline": r["roofline"],
                "cpu_baseline": r.get("cpu_baseline"), "e2e": r.get("e2e"), "gpu_launches": r["gpu_launches"],
                "clocks": r["clocks"],
            }
            print(json.dumps(out), flush=True)
    R.finalize(rk)


# -------------------------------------------------------------- served
def served_core(args, kernel: str) -> dict:
    """Poisson arrivals of downscaling requests into the continuous-batching
    server (config 4's size distributions; the arrival window and the step
    counts are scaled by --serve-duration and --serve-steps-scale so a run
    fits in minutes).  Returns the server's report and the workload."""
    import torch
    from hicar_b200.serve import Server, poisson_requests

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    smin, smax = int(round(50 * args.serve_steps_scale)), int(round(500 * args.serve_steps_scale))
    reqs = poisson_requests(args.serve_rate, args.serve_duration, seed=11, steps=(max(1, smin), max(1, smax)))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    srv = Server(device=local, budget_bytes=150e9, keep_results=False, stream=stream.cuda_stream,
                 path=KERNEL_PATH[kernel])
    for r in reqs:
        srv.submit(r)
    clocks = ClockSampler(local)
    clocks.start()
    srv.start_clock()
    srv.run()
    clk = clocks.stop()
    rep = srv.report()
    srv.close()
    desc = (f"served requests: Poisson {args.serve_rate} req/s for {args.serve_duration} s (config 4: 120 s), "
            f"area lognormal median 256^2 (sides 64..1024), nz U[20,60], 12 fields, steps U[{smin},{smax}] "
            f"(config 4: U[50,500], scaled by {args.serve_steps_scale}), HBM admission budget 150 GB, "
            f"kernel {kernel}")
    return {"report": rep, "workload": desc, "clocks": clk}


def run_served(args):
    from hicar_b200 import replicas as R
    if not R.from_env().is_root:
        return                                   # one server on one GPU: the other ranks have no work
    r = served_core(args, args.kernel)
    rep = r["report"]
    print(json.dumps({
        "metric": METRIC + " (served)", "value": rep.get("throughput_cell_species_per_s"), "unit": UNIT,
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": r["workload"]}, "serving": rep, "clocks": r["clocks"]}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "served":
        run_served(args)
    elif args.workload == "large":
        run_large(args)
    elif args.workload == "wind":
        run_wind(args)
    elif args.workload == "mp":
        run_mp(args)
    elif args.workload == "std":
        run_std(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
