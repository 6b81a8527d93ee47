"""Host-side mirror of ICAR's ``advection`` module over the C ABI.

Same public names, argument meaning and call order as
src/physics/advection_driver.f90:
    adv_var_request(options)        ->  which variables the scheme needs
    adv_init(domain, options)       ->  create the device-resident domain
    advect(domain, options, dt)     ->  one advection call, species in
                                        adv_vars order
plus the two domain methods that bracket it in a model step
(src/main/time_step.f90:319-389): ``domain.apply_forcing(dt)`` and
``domain.enforce_limits()``.

Options and Domain carry only the fields the advection path reads, named as
in options_t / domain_t.  Arrays are numpy float32 in the Fortran layout
(see hicar_b200.synth).  After adv_init the device copy is authoritative:
``domain.fetch(name)`` brings a field back, ``domain.mark_dirty(name)`` after
a host-side change uploads it again before the next advect (CPU physics
between advection calls).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

kADV_STD = 1
kADV_MPDATA = 2
kFLUXCOR_MONO = 1
kMP_SB04 = 2          # physics%microphysics, icar_constants.f90:393


@dataclass
class AdvOptions:                      # adv_options_type, opt_types.f90:119-127
    boundary_buffer: bool = False
    MPDATA_FCT: bool = True
    mpdata_order: int = 2
    flux_corr: int = 0
    h_order: int = 1
    v_order: int = 1


@dataclass
class PhysicsOptions:
    advection: int = kADV_MPDATA
    microphysics: int = 0


@dataclass
class TimeOptions:
    RK3: bool = False
    cfl_reduction_factor: float = 0.9   # time_options defaults, options_obj.f90 (time_parameters namelist)
    cfl_strictness: int = 3


@dataclass
class Parameters:
    advect_density: bool = False
    debug: bool = False


@dataclass
class Options:
    physics: PhysicsOptions = field(default_factory=PhysicsOptions)
    adv_options: AdvOptions = field(default_factory=AdvOptions)
    time_options: TimeOptions = field(default_factory=TimeOptions)
    parameters: Parameters = field(default_factory=Parameters)
    vars_to_allocate: set = field(default_factory=set)
    vars_to_advect: list = field(default_factory=list)

    def to_c(self) -> L.Opts:
        a = self.adv_options
        return L.Opts(int(self.physics.advection), int(bool(a.MPDATA_FCT)), int(a.mpdata_order), int(a.flux_corr),
                      int(a.h_order), int(a.v_order), int(bool(self.time_options.RK3)),
                      int(bool(self.parameters.advect_density)), int(bool(self.parameters.debug)),
                      int(bool(a.boundary_buffer)))


_METRIC_FIELDS = {
    "u": L.F_U, "v": L.F_V, "w": L.F_W, "density": L.F_DENSITY, "jacobian": L.F_JACOBIAN,
    "jacobian_u": L.F_JACOBIAN_U, "jacobian_v": L.F_JACOBIAN_V, "jacobian_w": L.F_JACOBIAN_W,
    "advection_dz": L.F_ADVECTION_DZ,
    # read only by the simple microphysics (mp)
    "pressure": L.F_PRESSURE, "exner": L.F_EXNER, "dz_mass": L.F_DZ_MASS,
    # kept on the device for restarts only
    "dz_interface": L.F_DZ_INTERFACE,
}


class Domain:
    """The advection-relevant part of domain_t for one image.

    ``adv_vars`` maps species names ('qv', 'theta', 'qc', ...) to arrays in
    the order they are advected (domain_obj.f90:62-89).
    """

    def __init__(self, nx: int, ny: int, nz: int, dx: float, device: int = 0,
                 boundaries=(True, True, True, True)):
        self.nx, self.ny, self.nz, self.dx = int(nx), int(ny), int(nz), float(dx)
        self.ims, self.ime, self.jms, self.jme, self.kms, self.kme = 1, nx, 1, ny, 1, nz
        self.device = device
        self.north_boundary, self.south_boundary, self.east_boundary, self.west_boundary = boundaries
        self.u = self.v = self.w = self.density = None
        self.jacobian = self.jacobian_u = self.jacobian_v = self.jacobian_w = self.advection_dz = None
        self.pressure = self.exner = self.dz_mass = self.dz_interface = None
        self.adv_vars: dict[str, np.ndarray] = {}
        self.forcing: dict[str, tuple[np.ndarray, np.ndarray | None]] = {}
        self._h = None
        self._dirty: set[str] = set()

    @classmethod
    def from_case(cls, case, device: int = 0) -> "Domain":
        d = cls(case.nx, case.ny, case.nz, case.dx, device=device)
        for k in _METRIC_FIELDS:
            a = getattr(case, k, None)
            setattr(d, k, None if a is None else np.ascontiguousarray(a, np.float32))
        d.adv_vars = {k: np.ascontiguousarray(v, np.float32).copy() for k, v in case.species.items()}
        return d

    @classmethod
    def create_on_device(cls, fields: dict, nx: int, ny: int, nz: int, dx: float, options: "Options",
                         device: int = 0, forcing: bool = False) -> "Domain":
        """adv_init from CUDA tensors already in device memory (Fortran layout,
        contiguous): fields holds the nine wind/metric fields and
        fields["species"] the advected ones.  forcing=True fixes every
        species' boundary forcing at its initial value."""
        import torch
        torch.cuda.current_stream(device).synchronize()   # the tensors must be complete before the copies
        d = cls(nx, ny, nz, dx, device=device)
        d._device_fields = fields
        names = list(fields["species"])
        d.adv_vars = {k: None for k in names}
        lib = L.load()
        desc = d._desc(names)
        opts = options.to_c()
        h = C.c_void_p()
        L.check(lib.icar_adv_create(C.byref(desc), C.byref(opts), C.byref(h)))
        d._h = h
        d._options = options
        for k, fid in _METRIC_FIELDS.items():
            if fields.get(k) is None:
                continue                     # the microphysics inputs are optional
            L.check(lib.icar_adv_set_field_device(h, fid, C.c_void_p(fields[k].data_ptr())), h)
        for k in names:
            t = fields["species"][k]
            L.check(lib.icar_adv_set_field_device(h, L.SPECIES_IDS[k], C.c_void_p(t.data_ptr())), h)
            if forcing:
                L.check(lib.icar_adv_set_field_device(h, L.F_FORCING_BASE + L.SPECIES_IDS[k],
                                                      C.c_void_p(t.data_ptr())), h)
        L.check(lib.icar_adv_sync(h), h)
        return d

    def fetch_device(self, name: str, out) -> None:
        """Copy a resident species into a contiguous CUDA tensor (Fortran layout)."""
        L.check(L.load().icar_adv_get_field_device(self.handle, self._field_id(name), C.c_void_p(out.data_ptr())),
                self.handle)

    def _desc(self, names) -> "L.Desc":
        desc = L.Desc()
        desc.nx, desc.ny, desc.nz, desc.dx = self.nx, self.ny, self.nz, self.dx
        if len(names) > L.MAX_SPECIES:
            raise ValueError("too many advected species")
        desc.n_species = len(names)
        for i, n in enumerate(names):
            desc.species[i] = L.SPECIES_IDS[n]
        desc.north_boundary, desc.south_boundary = int(self.north_boundary), int(self.south_boundary)
        desc.east_boundary, desc.west_boundary = int(self.east_boundary), int(self.west_boundary)
        desc.device = self.device
        return desc

    # -- handle plumbing -------------------------------------------------
    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("adv_init(domain, options) has not been called")
        return self._h

    def _field_id(self, name: str) -> int:
        if name in _METRIC_FIELDS:
            return _METRIC_FIELDS[name]
        if name in L.SPECIES_IDS:
            return L.SPECIES_IDS[name]
        if name.startswith("forcing_"):
            return L.F_FORCING_BASE + L.SPECIES_IDS[name[8:]]
        if name.startswith("dqdt_"):
            return L.F_DQDT_BASE + L.SPECIES_IDS[name[5:]]
        if name == "relax_filter":
            return L.F_RELAX_FILTER
        raise KeyError(name)

    def _host_array(self, name: str) -> np.ndarray:
        if name in _METRIC_FIELDS:
            return getattr(self, name)
        if name in self.adv_vars:
            return self.adv_vars[name]
        if name.startswith("forcing_"):
            return self.forcing[name[8:]][0]
        if name.startswith("dqdt_"):
            return self.forcing[name[5:]][1]
        raise KeyError(name)

    def upload(self, name: str, arr: np.ndarray | None = None) -> None:
        a = self._host_array(name) if arr is None else arr
        a = np.ascontiguousarray(a, np.float32)
        L.check(L.load().icar_adv_set_field(self.handle, self._field_id(name), L.f32_ptr(a), None), self.handle)

    def fetch(self, name: str) -> np.ndarray:
        """Copy a resident field back into (and return) its host array."""
        a = self._host_array(name)
        if not a.flags.c_contiguous:
            a = np.ascontiguousarray(a)
        L.check(L.load().icar_adv_get_field(self.handle, self._field_id(name), L.f32_ptr(a), None), self.handle)
        if name in self.adv_vars:
            self.adv_vars[name] = a
        return a

    def _shape_of(self, name: str) -> tuple[int, int, int]:
        if name == "u":
            return (self.ny, self.nz, self.nx + 1)
        if name == "v":
            return (self.ny + 1, self.nz, self.nx)
        return (self.ny, self.nz, self.nx)

    def download(self, names) -> dict[str, np.ndarray]:
        """Copy several resident fields to new host arrays with one wait on
        the device (icar_adv_download); species are also stored back into
        adv_vars."""
        names = list(names)
        ids = (C.c_int32 * max(len(names), 1))(*[self._field_id(n) for n in names])
        out = {n: np.empty(self._shape_of(n), np.float32) for n in names}
        ptrs = (C.c_void_p * max(len(names), 1))(*[out[n].ctypes.data for n in names])
        L.check(L.load().icar_adv_download(self.handle, len(names), ids, ptrs), self.handle)
        for n in names:
            if n in self.adv_vars:
                self.adv_vars[n] = out[n]
        return out

    def upload_many(self, arrays: dict) -> None:
        """Write several fields from host arrays (icar_adv_upload)."""
        names = list(arrays)
        keep = [np.ascontiguousarray(arrays[n], np.float32) for n in names]
        for n, a in zip(names, keep):
            if a.size != int(np.prod(self._shape_of(n))):
                raise ValueError(f"{n}: expected {self._shape_of(n)} values, got {a.shape}")
        ids = (C.c_int32 * max(len(names), 1))(*[self._field_id(n) for n in names])
        ptrs = (C.c_void_p * max(len(names), 1))(*[a.ctypes.data for a in keep])
        L.check(L.load().icar_adv_upload(self.handle, len(names), ids, ptrs), self.handle)

    def restart_vars(self) -> list[str]:
        """The fields options%restart_vars lists for advection
        (adv_std_var_request, advect.f90:95-107)."""
        return restart_vars(self._options)

    def download_restart(self) -> dict[str, np.ndarray]:
        """The advection restart set (u, v, w, dz_interface, qv) in one
        bulk download."""
        return self.download(self.restart_vars())

    def restore_restart(self, arrays: dict) -> None:
        """Write a restart set back (icar_adv_upload)."""
        self.upload_many(arrays)

    def relax_filter(self) -> np.ndarray:
        out = np.zeros((self.ny, self.nx), np.float32)
        L.check(L.load().icar_adv_get_field(self.handle, L.F_RELAX_FILTER, L.f32_ptr(out), None), self.handle)
        return out

    def mark_dirty(self, name: str) -> None:
        self._dirty.add(name)

    def _flush(self) -> None:
        for name in sorted(self._dirty):
            self.upload(name)
        self._dirty.clear()

    def set_forcing(self, name: str, forcing_hi: np.ndarray, dqdt: np.ndarray | None = None) -> None:
        """Boundary forcing of an advected species (forcing_hi and its dqdt)."""
        self.forcing[name] = (np.ascontiguousarray(forcing_hi, np.float32).copy(),
                              None if dqdt is None else np.ascontiguousarray(dqdt, np.float32).copy())
        if self._h is not None:
            self.upload("forcing_" + name)
            if dqdt is not None:
                self.upload("dqdt_" + name)

    # -- domain methods used around advect ---------------------------------
    def apply_forcing(self, dt_seconds: float) -> None:
        self._flush()
        L.check(L.load().icar_adv_apply_forcing(self.handle, C.c_double(dt_seconds)), self.handle)

    def enforce_limits(self) -> None:
        self._flush()
        L.check(L.load().icar_adv_enforce_limits(self.handle), self.handle)

    def sync(self) -> None:
        L.check(L.load().icar_adv_sync(self.handle), self.handle)

    def wait(self, timeout_s: float) -> bool:
        """Bounded wait for the handle's queued work: True when it is done,
        False when timeout_s passed first (the work stays queued)."""
        code = L.load().icar_adv_sync_timeout(self.handle, C.c_double(timeout_s))
        if code == L.TIMEOUT:
            return False
        L.check(code, self.handle)
        return True

    def device_bytes(self) -> int:
        b = C.c_int64(0)
        L.check(L.load().icar_adv_device_bytes(self.handle, C.byref(b)), self.handle)
        return int(b.value)

    def set_launch_shape(self, tile_shape: int | None = None, species_group: int | None = None) -> None:
        """Tile shape of the fused correction kernel (0..3 = 8/15/24/31 rows
        per tile) and species per thread of its donor-cell pass (0 = all);
        see hicar_b200.autotune.  Results do not depend on either."""
        lib = L.load()
        if tile_shape is not None:
            L.check(lib.icar_adv_set_tile_shape(self.handle, int(tile_shape)), self.handle)
        if species_group is not None:
            L.check(lib.icar_adv_set_species_group(self.handle, int(species_group)), self.handle)

    def use_staged_kernels(self, staged: bool = True) -> None:
        L.check(L.load().icar_adv_set_path(self.handle, 1 if staged else 0), self.handle)

    def use_single_pass(self, fast: bool = False) -> None:
        """MPDATA order 2 through the single-pass kernel (donor-cell pass,
        pseudo-velocities, limiter and corrective pass in one launch): bit-exact
        arithmetic, or fast=True for the fast-arithmetic variant."""
        L.check(L.load().icar_adv_set_path(self.handle, 3 if fast else 2), self.handle)

    def set_path(self, path: int) -> None:
        L.check(L.load().icar_adv_set_path(self.handle, int(path)), self.handle)

    def close(self) -> None:
        if self._h is not None:
            L.load().icar_adv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def adv_var_request(options: Options) -> None:
    """advection_driver.f90:46-57 -> adv_std_var_request (advect.f90:94-108)."""
    lib = L.load()
    alloc = (C.c_int32 * 8)()
    adv = (C.c_int32 * 8)()
    na, nv = C.c_int32(8), C.c_int32(8)
    opts = options.to_c()
    L.check(lib.icar_adv_var_request(C.byref(opts), alloc, C.byref(na), adv, C.byref(nv)))
    options.vars_to_allocate |= {int(alloc[i]) for i in range(na.value)}
    for i in range(nv.value):
        if int(adv[i]) not in options.vars_to_advect:
            options.vars_to_advect.append(int(adv[i]))


def restart_vars(options: Options) -> list[str]:
    """Names of the fields options%restart_vars lists for advection, in the
    reference's order (adv_std_var_request, advect.f90:95-107)."""
    n = C.c_int32(8)
    ids = (C.c_int32 * 8)()
    opts = options.to_c()
    L.check(L.load().icar_adv_restart_vars(C.byref(opts), ids, C.byref(n)))
    names = []
    for i in range(n.value):
        fid = int(ids[i])
        names.append(next((k for k, v in _METRIC_FIELDS.items() if v == fid), None) or L.SPECIES_NAMES[fid])
    return names


def adv_init(domain: Domain, options: Options) -> None:
    """advection_driver.f90:26-44: allocate the device-resident domain and
    upload every field the path reads."""
    lib = L.load()
    if domain._h is not None:
        domain.close()
    names = list(domain.adv_vars)
    desc = domain._desc(names)
    opts = options.to_c()
    h = C.c_void_p()
    L.check(lib.icar_adv_create(C.byref(desc), C.byref(opts), C.byref(h)))
    domain._h = h
    domain._options = options
    for k in _METRIC_FIELDS:
        if getattr(domain, k) is not None:
            domain.upload(k)
    for k in names:
        domain.upload(k)
    for k, (fh, dq) in domain.forcing.items():
        domain.upload("forcing_" + k)
        if dq is not None:
            domain.upload("dqdt_" + k)
    domain._dirty.clear()


def advect(domain: Domain, options: Options, dt: float) -> None:
    """advection_driver.f90:59-126: one advection call (asynchronous on the
    device; fetch() or sync() to wait)."""
    domain._flush()
    L.check(L.load().icar_adv_advect(domain.handle, C.c_float(dt)), domain.handle)


def balance_uvw(domain: Domain, options: Options) -> None:
    """wind.f90:88-164: rebuild the resident w from the horizontal
    divergence of u and v (density weighted with advect_density, the setting
    the handle was created with).  Asynchronous; fetch("w") to read it."""
    domain._flush()
    L.check(L.load().icar_adv_balance_uvw(domain.handle), domain.handle)


def compute_dt(domain: Domain, options: Options, dz_levels, use_density: bool = False) -> float:
    """time_step.f90:51-168: the largest stable time step (seconds) for the
    resident winds, options.time_options.cfl_reduction_factor and
    cfl_strictness, and the 1-D dz_levels.  Raises IcarAdvError
    (CFL_VIOLATION) when it is below 0.1 s, where the reference stops."""
    domain._flush()
    dz = np.ascontiguousarray(dz_levels, np.float32)
    if dz.size != domain.nz:
        raise ValueError("dz_levels must have nz entries")
    out = C.c_float()
    t = options.time_options
    L.check(L.load().icar_adv_compute_dt(domain.handle, dz.ctypes.data_as(C.POINTER(C.c_float)),
                                         C.c_float(t.cfl_reduction_factor), int(t.cfl_strictness),
                                         int(bool(use_density)), C.byref(out)), domain.handle)
    return float(out.value)


def mp(domain: Domain, options: Options, dt: float) -> None:
    """mp_driver.f90:813 mp(domain, options, dt) for physics%microphysics =
    kMP_SB04 (mp_simple): theta, qv, qc, qr, qs must be advected species of
    the domain and pressure, exner, density and dz_mass set.  Asynchronous;
    the accumulated rain and snow are read with precipitation()."""
    if options.physics.microphysics != kMP_SB04:
        raise NotImplementedError("only the simple microphysics (kMP_SB04) runs on the device")
    domain._flush()
    L.check(L.load().icar_adv_mp_simple(domain.handle, C.c_float(dt)), domain.handle)


def precipitation(domain: Domain) -> tuple[np.ndarray, np.ndarray]:
    """The real64 accumulated_precipitation and accumulated_snowfall (ny, nx)
    the microphysics has added up on the device."""
    rain = np.zeros((domain.ny, domain.nx), np.float64)
    snow = np.zeros((domain.ny, domain.nx), np.float64)
    L.check(L.load().icar_adv_get_precipitation(domain.handle, rain.ctypes.data_as(C.c_void_p),
                                                snow.ctypes.data_as(C.c_void_p)), domain.handle)
    return rain, snow


def step(domain: Domain, options: Options, dt_seconds: float, enforce_limits: bool = False) -> None:
    """apply_forcing -> advect -> (enforce_limits), time_step.f90:319-389."""
    domain._flush()
    L.check(L.load().icar_adv_step(domain.handle, C.c_double(dt_seconds), int(enforce_limits)), domain.handle)


def step_host(domain: Domain, options: Options, dt_seconds: float, q_in: dict, q_out: dict | None = None,
              enforce_limits: bool = False) -> dict:
    """One step for species held in host memory (icar_adv_step_host): the
    arrays of q_in (every advected species, by name) go to the device, the
    step runs, and the results come back into q_out (new arrays when None;
    q_out may be q_in).  Uploads, the step and downloads overlap by species
    group when the arrays are page-locked (e.g. torch pinned tensors'
    numpy views)."""
    domain._flush()
    names = list(domain.adv_vars)
    missing = [n for n in names if n not in q_in]
    if missing:
        raise KeyError(f"q_in lacks {missing}")
    shape = (domain.ny, domain.nz, domain.nx)
    ins = []
    for n in names:
        a = q_in[n]
        if a.dtype != np.float32 or not a.flags.c_contiguous or a.shape != shape:
            raise ValueError(f"{n}: need a C-contiguous float32 array of shape {shape}")
        ins.append(a)
    if q_out is None:
        q_out = {n: np.empty(shape, np.float32) for n in names}
    outs = []
    for n in names:
        a = q_out[n]
        if a.dtype != np.float32 or not a.flags.c_contiguous or a.shape != shape or not a.flags.writeable:
            raise ValueError(f"{n}: q_out needs a writeable C-contiguous float32 array of shape {shape}")
        outs.append(a)
    k = max(len(names), 1)
    pin = (C.c_void_p * k)(*[a.ctypes.data for a in ins])
    pout = (C.c_void_p * k)(*[a.ctypes.data for a in outs])
    L.check(L.load().icar_adv_step_host(domain.handle, C.c_double(dt_seconds), int(enforce_limits), pin, pout),
            domain.handle)
    return q_out
