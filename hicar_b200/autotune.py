"""Autotuner for the launch shape of the fused MPDATA kernels.

Two knobs, neither of which changes any result (every combination gives
bit-identical fields; tests/test_autotune_gpu.py checks it):

  tile shape     output rows per tile of the correction kernel (8, 15, 24 or
                 31 rows of 28 columns).  Taller tiles recompute less of the
                 y halo around each tile but need more shared memory per CTA,
                 so fewer CTAs fit on an SM, and waste more rows in the last
                 tile of a column when ny-2 is not a multiple of the height.
  species group  species that one thread of the donor-cell pass takes (0 =
                 all).  All species reuse a cell's winds and metric terms;
                 smaller groups give small domains more blocks.

tune_domain(nx, ny, nz, n_species, fct)
    measures every combination on a synthetic domain of that grid shape,
    generated on the device, each from the same saved initial state, and
    returns the fastest.  Results are cached per
    (GPU name, grid shape, species count, FCT) in memory and in a JSON file
    ($HICAR_B200_AUTOTUNE_CACHE, default ~/.cache/hicar_b200/autotune.json).
shape_costs(fct)
    measures once per GPU the device time of one tile-level of one species
    for every tile shape, on a calibration domain large enough to fill the
    GPU.  choose_batch_shape(members, costs) then picks the tile shape of a
    batch -- one persistent launch over every member's tiles -- as the shape
    with the least predicted time, sum over members of tiles x levels x
    species x cost per tile-level.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import asdict, dataclass
from pathlib import Path

TILE_COLUMNS = 28
TILE_ROWS = (8, 15, 24, 31)          # icar_adv_tile_shapes order
_mem_cache: dict[str, dict] = {}


@dataclass
class Choice:
    tile_shape: int
    species_group: int
    ms_per_advect: float | None = None
    measured: dict | None = None     # "shape:group" -> ms per advect

    @property
    def rows(self) -> int:
        return TILE_ROWS[self.tile_shape]


# ---------------------------------------------------------------- tile geometry
def tiles(nx: int, ny: int, rows: int) -> int:
    """Tiles the correction kernel launches for one species of one level-column:
    tile tx covers output columns [28*tx-2, 28*tx+26), the last one must reach
    nx-2; tile rows cover output rows 1..ny-2."""
    tx = nx // TILE_COLUMNS + 1
    ty = (ny - 2 + rows - 1) // rows
    return tx * ty


def species_groups(n_species: int) -> list[int]:
    """Candidate species groups: all (0), then a few even splits."""
    out = [0]
    for parts in (2, 3, 4, 6):
        g = -(-n_species // parts)
        if 1 <= g < n_species and g not in out:
            out.append(g)
    return out


def choose_batch_shape(members, costs: dict[int, float]) -> int:
    """Tile shape with the least predicted batch time.  members: iterable of
    (nx, ny, nz, n_species); costs: tile shape -> device ms per tile-level of
    one species (shape_costs)."""
    best, best_t = None, None
    for shape, c in sorted(costs.items()):
        rows = TILE_ROWS[shape]
        t = sum(tiles(nx, ny, rows) * nz * s for nx, ny, nz, s in members) * c
        if best_t is None or t < best_t:
            best, best_t = shape, t
    return 1 if best is None else best


# ---------------------------------------------------------------- cache
def _cache_path() -> Path:
    p = os.environ.get("HICAR_B200_AUTOTUNE_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "hicar_b200" / "autotune.json"


def _load_cache() -> dict:
    if not _mem_cache:
        try:
            _mem_cache.update(json.loads(_cache_path().read_text()))
        except (OSError, ValueError):
            pass
    return _mem_cache


def _store(key: str, value: dict) -> None:
    cache = _load_cache()
    cache[key] = value
    try:
        p = _cache_path()
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(".tmp")
        tmp.write_text(json.dumps(cache, indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass                      # a read-only home still tunes, in memory


def _gpu_key(device: int) -> str:
    import torch
    return torch.cuda.get_device_name(device).replace(" ", "_")


# ---------------------------------------------------------------- measurement
def _synthetic_domain(nx, ny, nz, n_species, fct, device, seed=12345):
    from . import synth
    from .advection import AdvOptions, Domain, Options
    names = synth.ALL12[:n_species] if n_species <= len(synth.ALL12) else None
    if names is None:
        raise ValueError(f"at most {len(synth.ALL12)} species can be tuned synthetically")
    fields, dt = synth.device_member(nx, ny, nz, seed, device=device, species=names)
    opts = Options(adv_options=AdvOptions(MPDATA_FCT=bool(fct)))
    dom = Domain.create_on_device(fields, nx, ny, nz, 4000.0, opts, device=device)
    dom._device_fields = None
    return dom, opts, dt


class _SavedState:
    """The species of a domain at one moment, kept on the device, so that
    every candidate is timed from the same state (the cost of a step depends
    on the fields)."""

    def __init__(self, dom):
        import torch
        self.dom = dom
        self.t = {}
        for k in dom.adv_vars:
            t = torch.empty(dom.nx * dom.ny * dom.nz, dtype=torch.float32, device=f"cuda:{dom.device}")
            dom.fetch_device(k, t)
            self.t[k] = t
        dom.sync()

    def restore(self) -> None:
        import ctypes as C
        from . import _lib as L
        lib = L.load()
        for k, t in self.t.items():
            L.check(lib.icar_adv_set_field_device(self.dom.handle, L.SPECIES_IDS[k], C.c_void_p(t.data_ptr())),
                    self.dom.handle)


def _time_advects(dom, opts, dt, shape, group, reps, saved: _SavedState | None = None) -> float:
    import ctypes as C
    from . import _lib as L
    from .advection import advect
    lib = L.load()
    if saved is not None:
        saved.restore()
    dom.set_launch_shape(shape, group)
    advect(dom, opts, dt)                       # warm-up with this shape
    L.check(lib.icar_adv_profile(dom.handle, 1), dom.handle)
    for _ in range(reps):
        advect(dom, opts, dt)
    ms, kl, al, ps = C.c_double(), C.c_int64(), C.c_int64(), C.c_int64()
    L.check(lib.icar_adv_profile_read(dom.handle, C.byref(ms), C.byref(kl), C.byref(al), C.byref(ps)), dom.handle)
    L.check(lib.icar_adv_profile(dom.handle, 0), dom.handle)
    return ms.value / max(ps.value, 1)


def tune_domain(nx: int, ny: int, nz: int, n_species: int, fct: bool = True, device: int = 0, reps: int = 3,
                use_cache: bool = True) -> Choice:
    """Fastest (tile shape, species group) for this grid shape, measured."""
    key = f"domain:{_gpu_key(device)}:{nx}x{ny}x{nz}:S{n_species}:fct{int(bool(fct))}"
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            return Choice(**hit)
    dom, opts, dt = _synthetic_domain(nx, ny, nz, n_species, fct, device)
    measured = {}
    try:
        saved = _SavedState(dom)
        for shape in range(len(TILE_ROWS)):
            for group in species_groups(n_species):
                measured[f"{shape}:{group}"] = _time_advects(dom, opts, dt, shape, group, reps, saved)
    finally:
        dom.close()
    best = min(measured, key=measured.get)
    shape, group = (int(v) for v in best.split(":"))
    choice = Choice(shape, group, measured[best], measured)
    _store(key, asdict(choice))
    return choice


def shape_costs(fct: bool = True, device: int = 0, calib=(256, 256, 40, 12), reps: int = 3,
                use_cache: bool = True) -> dict[int, float]:
    """Device ms per tile-level of one species for every tile shape, measured
    on a calibration domain (the whole fused step per advect, divided by the
    correction kernel's tile-levels)."""
    nx, ny, nz, S = calib
    key = f"costs:{_gpu_key(device)}:{nx}x{ny}x{nz}:S{S}:fct{int(bool(fct))}"
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            return {int(k): v for k, v in hit.items()}
    dom, opts, dt = _synthetic_domain(nx, ny, nz, S, fct, device)
    costs = {}
    try:
        saved = _SavedState(dom)
        for shape, rows in enumerate(TILE_ROWS):
            ms = _time_advects(dom, opts, dt, shape, 0, reps, saved)
            costs[shape] = ms / (tiles(nx, ny, rows) * nz * S)
    finally:
        dom.close()
    _store(key, {str(k): v for k, v in costs.items()})
    return costs


def tune_batch(batch, fct: bool = True, device: int = 0) -> int:
    """Pick and set the tile shape of a hicar_b200.batch.Batch from its
    members' grid shapes (the species group stays 0: the batch's donor-cell
    pass already spans every member)."""
    costs = shape_costs(fct, device)
    members = [(d.nx, d.ny, d.nz, len(d.adv_vars)) for d in batch.members]
    shape = choose_batch_shape(members, costs)
    batch.set_tile_shape(shape)
    return shape


def apply(domain, choice: Choice) -> None:
    domain.set_launch_shape(choice.tile_shape, choice.species_group)


def tune_and_apply(domain, fct: bool = True) -> Choice:
    """Tune for a domain's grid shape (on a synthetic copy, so the domain's
    own state is untouched) and set the result on it."""
    t0 = time.perf_counter()
    c = tune_domain(domain.nx, domain.ny, domain.nz, len(domain.adv_vars), fct, domain.device)
    apply(domain, c)
    c.measured = dict(c.measured or {}, tune_seconds=time.perf_counter() - t0)
    return c
