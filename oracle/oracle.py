"""ctypes access to the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke()
and by bench.py's CPU-baseline and reference legs, only as the checker or the
timed CPU baseline.  The product (hicar_b200, libicar_adv.so) never imports
it.  See icar_adv_oracle.c for the reference files each routine restates.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class OracleOpts(C.Structure):
    _fields_ = [("advection", C.c_int), ("mpdata_fct", C.c_int), ("mpdata_order", C.c_int),
                ("flux_corr", C.c_int), ("h_order", C.c_int), ("v_order", C.c_int), ("rk3", C.c_int),
                ("advect_density", C.c_int), ("halo", C.c_int)]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            import subprocess
            subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
        _lib = C.CDLL(str(LIB))
    return _lib


def halo_size(advection: int, h_order: int = 1, v_order: int = 1, flux_corr: int = 0) -> int:
    """grid%halo_size as read_domain_shape derives it (domain_obj.f90:2979-2986)."""
    adv_order = max(h_order, v_order)
    if flux_corr == 1:
        adv_order += 2
    if advection == 2:
        adv_order = 4
    return (adv_order + 1) // 2


def make_opts(advection=2, mpdata_fct=1, mpdata_order=2, flux_corr=0, h_order=1, v_order=1, rk3=0,
              advect_density=0) -> OracleOpts:
    return OracleOpts(advection, mpdata_fct, mpdata_order, flux_corr, h_order, v_order, rk3, advect_density,
                      halo_size(advection, h_order, v_order, flux_corr))


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def _sfx(dtype) -> str:
    return "_f64" if np.dtype(dtype) == np.float64 else "_f32"


def advect(case, opts: OracleOpts, dt: float, dtype=np.float32, species=None) -> dict:
    """advect(domain, options, dt) on copies of case's species; returns them."""
    lib = load()
    t = np.dtype(dtype)
    ct = C.c_double if t == np.float64 else C.c_float
    fn = getattr(lib, "advect" + _sfx(t))
    names = list(species if species is not None else case.species.keys())
    arrs = [np.ascontiguousarray(case.species[n], dtype=t).copy() for n in names]
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    f = {k: np.ascontiguousarray(getattr(case, k), dtype=t)
         for k in ("u", "v", "w", "density", "jacobian", "jacobian_u", "jacobian_v", "jacobian_w", "advection_dz")}
    fn.restype = None
    fn(C.byref(opts), C.c_int(case.nx), C.c_int(case.ny), C.c_int(case.nz), ct(case.dx), ct(dt),
       _p(f["u"]), _p(f["v"]), _p(f["w"]), _p(f["density"]), _p(f["jacobian"]), _p(f["jacobian_u"]),
       _p(f["jacobian_v"]), _p(f["jacobian_w"]), _p(f["advection_dz"]), C.c_int(len(arrs)), ptrs)
    return dict(zip(names, arrs))


def run_steps(case, opts: OracleOpts, dt: float, nsteps: int, dtype=np.float32, forcing=None,
              filter2d=None, wrap_y=False) -> dict:
    """nsteps of [apply_forcing ->] advect on a copy of the case's species.
    forcing: dict name -> (forcing_hi, dqdt) arrays; wrap_y copies rows
    ny-2 -> 0 and 1 -> ny-1 after each step (periodic test)."""
    c = case.copy()
    t = np.dtype(dtype)
    c.species = {k: v.astype(t) for k, v in c.species.items()}
    fo = {k: (a.astype(t).copy(), b.astype(t).copy()) for k, (a, b) in (forcing or {}).items()}
    for _ in range(nsteps):
        if fo:
            for name, (fh, dq) in fo.items():
                apply_forcing(c.species[name], fh, dq, filter2d, dt)
        c.species = advect(c, opts, dt, dtype=t)
        if wrap_y:
            for q in c.species.values():
                q[0] = q[c.ny - 2]
                q[c.ny - 1] = q[1]
    return c.species


def apply_forcing(q: np.ndarray, forcing: np.ndarray, dqdt: np.ndarray, filter2d: np.ndarray, dt: float) -> None:
    """In place, on arrays of q's dtype; filter2d is float32 (ny, nx)."""
    lib = load()
    ny, nz, nx = q.shape
    fn = getattr(lib, "apply_forcing" + _sfx(q.dtype))
    fn.restype = None
    flt = np.ascontiguousarray(filter2d, dtype=q.dtype)
    fn(C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(flt), C.c_double(dt), _p(q), _p(forcing), _p(dqdt))


def init_relax_filters(nx: int, ny: int, hs: int, north=1, south=1, east=1, west=1) -> np.ndarray:
    lib = load()
    out = np.zeros((ny, nx), np.float32)
    lib.init_relax_filters.restype = None
    lib.init_relax_filters(C.c_int(nx), C.c_int(ny), C.c_int(hs), C.c_int(north), C.c_int(south), C.c_int(east),
                           C.c_int(west), _p(out))
    return out


def enforce_limits(q: np.ndarray) -> None:
    lib = load()
    fn = getattr(lib, "enforce_limits" + _sfx(q.dtype))
    fn.restype = None
    fn(C.c_size_t(q.size), _p(q))


def mpdata_compute_wind(case, dt: float, advect_density: int = 0, dtype=np.float32):
    lib = load()
    t = np.dtype(dtype)
    ct = C.c_double if t == np.float64 else C.c_float
    nx, ny, nz = case.nx, case.ny, case.nz
    Um = np.zeros((ny, nz, nx + 1), t)
    Vm = np.zeros((ny + 1, nz, nx), t)
    Wm = np.zeros((ny, nz, nx), t)
    a = {k: np.ascontiguousarray(getattr(case, k), dtype=t)
         for k in ("u", "v", "w", "density", "jacobian_u", "jacobian_v", "jacobian_w")}
    fn = getattr(lib, "mpdata_compute_wind" + _sfx(t))
    fn.restype = None
    fn(C.c_int(nx), C.c_int(ny), C.c_int(nz), ct(case.dx), ct(dt), C.c_int(advect_density), _p(a["u"]), _p(a["v"]),
       _p(a["w"]), _p(a["density"]), _p(a["jacobian_u"]), _p(a["jacobian_v"]), _p(a["jacobian_w"]), _p(Um), _p(Vm),
       _p(Wm))
    return Um, Vm, Wm


def upwind_advection(qin, U, V, W, rho, dz, jaco):
    lib = load()
    ny, nz, nx = qin.shape
    out = np.empty_like(qin)
    fn = getattr(lib, "upwind_advection" + _sfx(qin.dtype))
    fn.restype = None
    fn(C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(qin), _p(U), _p(V), _p(W), _p(rho), _p(out), _p(dz), _p(jaco))
    return out


def mpdata_fluxes(q, U, V, wdz, G):
    lib = load()
    ny, nz, nx = q.shape
    u2 = np.zeros((ny, nz, nx + 1), q.dtype)
    v2 = np.zeros((ny + 1, nz, nx), q.dtype)
    w2 = np.zeros((ny, nz, nx), q.dtype)
    fn = getattr(lib, "mpdata_fluxes" + _sfx(q.dtype))
    fn.restype = None
    fn(C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(q), _p(U), _p(V), _p(wdz), _p(u2), _p(v2), _p(w2), _p(G))
    return u2, v2, w2


def flux_limiter(q, q2, u2, v2, w2):
    lib = load()
    ny, nz, nx = q.shape
    fn = getattr(lib, "flux_limiter" + _sfx(q.dtype))
    fn.restype = None
    fn(C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(q), _p(q2), _p(u2), _p(v2), _p(w2))


def balance_uvw(case, hs: int, advect_density: int = 1, dtype=np.float32) -> np.ndarray:
    """balance_uvw (wind.f90:88-164): w rebuilt from the horizontal
    divergence of u, v; returns the new w (the case is not modified)."""
    lib = load()
    t = np.dtype(dtype)
    ct = C.c_double if t == np.float64 else C.c_float
    f = {k: np.ascontiguousarray(getattr(case, k), dtype=t)
         for k in ("u", "v", "density", "jacobian_u", "jacobian_v", "jacobian_w", "advection_dz")}
    w = np.ascontiguousarray(case.w, dtype=t).copy()
    fn = getattr(lib, "balance_uvw" + _sfx(t))
    fn.restype = None
    fn(C.c_int(case.nx), C.c_int(case.ny), C.c_int(case.nz), C.c_int(hs), ct(case.dx), C.c_int(advect_density),
       _p(f["u"]), _p(f["v"]), _p(w), _p(f["density"]), _p(f["advection_dz"]), _p(f["jacobian_u"]),
       _p(f["jacobian_v"]), _p(f["jacobian_w"]))
    return w


def compute_dt(case, hs: int, dz_levels, cfl: float, strictness: int, use_density: int = 0,
               dtype=np.float32) -> tuple[float, bool]:
    """compute_dt (time_step.f90:51-168) on the case's winds; returns
    (dt, too_small) where too_small is the reference's dt < 0.1 stop."""
    lib = load()
    t = np.dtype(dtype)
    ct = C.c_double if t == np.float64 else C.c_float
    u, v, w = (np.ascontiguousarray(getattr(case, k), dtype=t) for k in ("u", "v", "w"))
    dz = np.ascontiguousarray(dz_levels, dtype=t)
    fn = getattr(lib, "compute_dt" + _sfx(t))
    fn.restype = ct
    small = C.c_int(0)
    dt = fn(C.c_int(case.nx), C.c_int(case.ny), C.c_int(case.nz), C.c_int(hs), ct(case.dx), _p(u), _p(v), _p(w),
            _p(dz), ct(cfl), C.c_int(strictness), C.c_int(use_density), C.byref(small))
    return float(dt), bool(small.value)


def mp_simple(fields: dict, dt: float, hs: int, acc_rain=None, acc_snow=None, dtype=np.float32):
    """mp_simple_driver (mp_simple.f90:595-646) on copies of the fields
    (Fortran layout (ny, nz, nx)): pressure, th, pii, rho, qv, qc, qr, qs, dz.
    Returns (updated dict of th, qv, qc, qr, qs, acc_rain, acc_snow, stop)."""
    lib = load()
    t = np.dtype(dtype)
    ct = C.c_double if t == np.float64 else C.c_float
    ny, nz, nx = fields["th"].shape
    f = {k: np.ascontiguousarray(fields[k], dtype=t).copy() for k in ("pressure", "th", "pii", "rho", "qv", "qc",
                                                                     "qr", "qs", "dz")}
    ar = np.zeros((ny, nx)) if acc_rain is None else np.ascontiguousarray(acc_rain, np.float64).copy()
    asn = np.zeros((ny, nx)) if acc_snow is None else np.ascontiguousarray(acc_snow, np.float64).copy()
    fn = getattr(lib, "mp_simple_driver" + _sfx(t))
    fn.restype = C.c_int
    stop = fn(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(hs), ct(dt), _p(f["pressure"]), _p(f["th"]),
              _p(f["pii"]), _p(f["rho"]), _p(f["qv"]), _p(f["qc"]), _p(f["qr"]), _p(f["qs"]), _p(ar), _p(asn),
              _p(f["dz"]))
    out = {k: f[k] for k in ("th", "qv", "qc", "qr", "qs")}
    out.update(acc_rain=ar, acc_snow=asn, stop=bool(stop))
    return out
