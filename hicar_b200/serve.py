"""Served form: a continuous-batching request loop over the batched step.

Requests (a downscaling domain: terrain, initial state and winds, a step
count) arrive over time.  The server admits a request when a slot is free
and its device footprint (icar_adv_footprint) fits the memory budget, keeps
its state resident, and merges every admitted request into the one batched
step (hicar_b200.batch), so requests that arrive while others run join
between steps and their work overlaps on the device.  A finished request is
downloaded and leaves the batch, freeing its slot and memory.  Each
request's result is bit-identical to running it alone (the batch computes
every member exactly as the single-domain path does).

Latency = completion - arrival; its queueing share = (admission - arrival)
/ latency.  Throughput = cell-species updates of all requests / wall time.
"""
from __future__ import annotations

import collections
import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .advection import Domain, Options
from .batch import Batch


@dataclass
class Request:
    rid: int
    nx: int
    ny: int
    nz: int
    steps: int
    seed: int
    arrival: float = 0.0           # seconds on the server clock
    species: tuple = ("qv", "qc", "qr", "qi", "qs", "qg", "nr", "ni", "ns", "ng", "nc", "theta")
    # filled by the server
    admitted: float | None = None
    finished: float | None = None
    result: dict | None = None
    footprint: int = 0
    error: str | None = None       # set when the request failed (it then has no result)

    @property
    def cell_species(self) -> int:
        return self.nx * self.ny * self.nz * len(self.species) * self.steps

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def queueing(self) -> float:
        return self.admitted - self.arrival


@dataclass
class _Live:
    req: Request
    dom: Domain
    remaining: int
    fields: dict = field(default_factory=dict)


def footprint(req: Request, options: Options) -> int:
    """Device bytes a request's domain needs (handle fields + fused scratch + forcing)."""
    lib = L.load()
    desc = L.Desc()
    desc.nx, desc.ny, desc.nz, desc.dx = req.nx, req.ny, req.nz, 4000.0
    desc.n_species = len(req.species)
    for i, n in enumerate(req.species):
        desc.species[i] = L.SPECIES_IDS[n]
    b = C.c_int64()
    opts = options.to_c()
    L.check(lib.icar_adv_footprint(C.byref(desc), C.byref(opts), C.byref(b)))
    P = ((req.nx + 1) + 3) // 4 * 4
    cells = P * req.nz * (req.ny + 1)
    # + the boundary forcing and its tendency per species
    return int(b.value) + 4 * cells * 2 * len(req.species)


class InjectedFault(RuntimeError):
    """A failure raised on the host by the fault hook (tests of the serving loop)."""


class Server:
    """path: MPDATA kernels of the batched step (0 two-pass, 2 single-pass
    bit-exact, 3 single-pass fast; see icar_adv_set_path).  fault_hook(req,
    stage, steps_done), if given, is called on the host when a request is set
    up (stage "setup") and after each of its steps (stage "step"); an
    exception it raises fails that request alone: the request leaves the
    batch with its error recorded, and every other request continues."""

    def __init__(self, device: int = 0, budget_bytes: float = 150e9, max_slots: int = 512,
                 options: Options | None = None, keep_results: bool = True, stream=None, path: int = 0,
                 fault_hook=None):
        self.device = device
        self.budget = int(budget_bytes)
        self.max_slots = max_slots
        self.options = options or Options()
        self.keep_results = keep_results
        self.path = path
        self.fault_hook = fault_hook
        self.failed: list[Request] = []
        import torch
        self.batch = Batch(device)
        self.batch.set_path(path)
        # the batch runs on this stream; completion times come from events on it
        self.stream = torch.cuda.Stream(device) if stream is None else torch.cuda.ExternalStream(stream, device)
        self.batch.set_stream(self.stream.cuda_stream)
        # requests are generated and set up on a stream of their own: set-up
        # waits for its own work, never for the batched steps in flight
        self.setup_stream = torch.cuda.Stream(device)
        self._ev0 = None
        self.queue: collections.deque[Request] = collections.deque()
        self.live: list[_Live] = []
        self.used = 0
        self.done: list[Request] = []
        self.t0 = time.perf_counter()
        self.peak_used = 0
        self.peak_live = 0
        self.steps = 0
        self.graveyard: list = []
        self.flush_every = 16

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, req: Request) -> None:
        req.footprint = footprint(req, self.options)
        if req.footprint > self.budget:
            raise ValueError(f"request {req.rid} needs {req.footprint} bytes, over the whole budget")
        self.queue.append(req)

    # -- admission ----------------------------------------------------------
    def _admit(self) -> None:
        import torch

        from .synth import device_member
        now = self.now()
        while self.queue and self.queue[0].arrival <= now:
            req = self.queue[0]
            if len(self.live) >= self.max_slots or self.used + req.footprint > self.budget:
                break                      # FIFO: wait for a slot / memory to free up
            self.queue.popleft()
            req.admitted = self.now()
            dom = None
            try:
                with torch.cuda.stream(self.setup_stream):
                    fields, dt = device_member(req.nx, req.ny, req.nz, req.seed, device=self.device,
                                               species=req.species)
                    dom = Domain.create_on_device(fields, req.nx, req.ny, req.nz, 4000.0, self.options,
                                                  device=self.device, forcing=True)
                    dom._device_fields = None      # the handle holds its own copies now
                    del fields
                dom.set_path(self.path)
                if self.fault_hook is not None:
                    self.fault_hook(req, "setup", 0)
                self.batch.add(dom, dt)
            except Exception as exc:        # this request fails alone; the server carries on
                if dom is not None:
                    dom.close()
                req.error = f"set-up failed: {exc}"
                req.finished = self.now()
                self.failed.append(req)
                continue
            self.used += req.footprint
            self.live.append(_Live(req, dom, req.steps))
            self.peak_used = max(self.peak_used, self.used)
            self.peak_live = max(self.peak_live, len(self.live))

    def _retire(self, lv: _Live) -> None:
        import torch
        req = lv.req
        if self.keep_results:
            out = {}
            for k in req.species:
                t = torch.empty(req.ny * req.nz * req.nx, dtype=torch.float32, device=f"cuda:{self.device}")
                lv.dom.fetch_device(k, t)
                out[k] = t
            self.batch.sync()
            req.result = {k: t.cpu().numpy().reshape(req.ny, req.nz, req.nx) for k, t in out.items()}
        self.batch.remove(lv.dom)
        # retired domains are destroyed in groups (their memory stays counted
        # until then); destroy returns their memory in stream order
        self.graveyard.append((lv.dom, req.footprint))
        if len(self.graveyard) >= self.flush_every or (self.queue and self.used + self.queue[0].footprint > self.budget):
            self._flush_graveyard()
        req.finished = self.now()
        self.done.append(req)

    def _fail(self, lv: _Live, msg: str) -> None:
        """A request failed between steps: it leaves the batch (no launch of
        it is in flight once the batch stream has drained past its last
        step) and its memory is returned; the batch goes on without it."""
        req = lv.req
        self.batch.remove(lv.dom)
        self.graveyard.append((lv.dom, req.footprint))
        req.error = msg
        req.finished = self.now()
        self.failed.append(req)

    def _flush_graveyard(self) -> None:
        for dom, fp in self.graveyard:
            dom.close()
            self.used -= fp
        self.graveyard.clear()

    # -- loop ---------------------------------------------------------------
    def start_clock(self) -> None:
        """t = 0 of the server clock, matched to an event on the batch stream."""
        import torch
        self.stream.synchronize()
        self._ev0 = torch.cuda.Event(enable_timing=True)
        self._ev0.record(self.stream)
        self._ev0.synchronize()
        self.t0 = time.perf_counter()

    def run(self, max_wall: float | None = None) -> None:
        """Serve until every submitted request is done (or max_wall seconds).
        The host never waits for the device except to download kept results
        and to free retired domains in bulk; a request's completion time is
        read from an event recorded after its last step."""
        import torch
        if self._ev0 is None:
            self.start_clock()
        while self.queue or self.live:
            if max_wall is not None and self.now() > max_wall:
                break
            self._admit()
            if not self.live:
                if self.queue:
                    time.sleep(max(0.0, min(0.01, self.queue[0].arrival - self.now())))
                continue
            self.batch.step()
            self.steps += 1
            finished, broken = [], []
            for lv in self.live:
                lv.remaining -= 1
                if self.fault_hook is not None:
                    try:
                        self.fault_hook(lv.req, "step", lv.req.steps - lv.remaining)
                    except Exception as exc:
                        broken.append((lv, exc))
                        continue
                if lv.remaining == 0:
                    finished.append(lv)
            for lv, exc in broken:
                self.live.remove(lv)
                self._fail(lv, f"failed after {lv.req.steps - lv.remaining} steps: {exc}")
            if finished:
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(self.stream)
                for lv in finished:
                    self.live.remove(lv)
                    lv.req._done_event = ev
                    self._retire(lv)
        self._flush_graveyard()
        for r in self.done:
            ev = getattr(r, "_done_event", None)
            if ev is not None:
                ev.synchronize()
                r.finished = self._ev0.elapsed_time(ev) / 1e3
                r._done_event = None

    def report(self) -> dict:
        done = [r for r in self.done if r.finished is not None]
        if not done:
            return {"requests": 0}
        lat = np.array([r.latency for r in done])
        q = np.array([r.queueing for r in done])
        span = max(r.finished for r in done) - min(r.arrival for r in done)
        work = sum(r.cell_species for r in done)
        return {
            "requests": len(done),
            "failed": len(self.failed),
            "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()),
            "queueing_share": float(q.sum() / lat.sum()),
            "throughput_cell_species_per_s": work / span,
            "wall_s": span,
            "batched_steps": self.steps,
            "peak_in_flight": self.peak_live,
            "peak_bytes": self.peak_used,
        }

    def close(self) -> None:
        for lv in list(self.live):
            self.batch.remove(lv.dom)
            lv.dom.close()
        self.live.clear()
        self.batch.close()


def poisson_requests(rate: float, duration: float, seed: int = 0, steps=(50, 500), median_side: int = 256,
                     side_clip=(64, 1024), nz=(20, 60)) -> list[Request]:
    """Poisson arrivals; area lognormal (median median_side^2, each side
    clipped), nz ~ U[nz], steps ~ U[steps]."""
    rng = np.random.default_rng(seed)
    t, out, rid = 0.0, [], 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t > duration:
            break
        area = float(median_side ** 2 * np.exp(rng.normal(0.0, 0.5)))
        aspect = float(np.exp(rng.normal(0.0, 0.25)))
        nx = int(np.clip(round(np.sqrt(area * aspect)), *side_clip))
        ny = int(np.clip(round(np.sqrt(area / aspect)), *side_clip))
        out.append(Request(rid, nx, ny, int(rng.integers(nz[0], nz[1] + 1)), int(rng.integers(steps[0], steps[1] + 1)),
                           seed * 100000 + rid, arrival=t))
        rid += 1
    return out
