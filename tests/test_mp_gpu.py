"""Simple microphysics (SB04, mp_simple.f90) on the GPU against the CPU
oracle, through the C ABI.  Both evaluate exp in the saturation mixing
ratio as the correctly rounded single-precision value, so the fields agree
cell for cell; the path's stated tolerance (max relative error <= 1e-5 per
call, <= 1e-4 after repeated advect -> mp steps, floor 1e-6 * max|q|) is
asserted as well, and the real64 precipitation accumulations to the same
bounds."""
import ctypes as C

import numpy as np
import pytest

from hicar_b200 import _lib as L, synth
from hicar_b200.advection import Domain, Options, PhysicsOptions, adv_init, advect, kMP_SB04, mp, precipitation

pytestmark = pytest.mark.gpu

FIELDS = ("theta", "qv", "qc", "qr", "qs")


def rel_err(a, ref):
    ref = ref.astype(np.float64)
    scale = max(float(np.abs(ref).max()), 1e-30)
    return float((np.abs(a.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-6 * scale)).max())


def mp_case(seed=3, nx=61, ny=47, nz=20, moist=1.6):
    c = synth.add_mp_fields(synth.config2(seed=seed, nx=nx, ny=ny, nz=nz), moist=moist)
    c.species = {k: c.species[k] for k in FIELDS}
    return c


def oracle_mp(O, c, dt, rain=None, snow=None):
    f = {"pressure": c.pressure, "th": c.species["theta"], "pii": c.exner, "rho": c.density, "qv": c.species["qv"],
         "qc": c.species["qc"], "qr": c.species["qr"], "qs": c.species["qs"], "dz": c.dz_mass}
    out = O.mp_simple(f, dt, 2, rain, snow)
    sp = {"theta": out["th"], "qv": out["qv"], "qc": out["qc"], "qr": out["qr"], "qs": out["qs"]}
    return sp, out["acc_rain"], out["acc_snow"], out["stop"]


OPTS = Options(physics=PhysicsOptions(microphysics=kMP_SB04))


@pytest.mark.parametrize("shape", [(61, 47, 20), (33, 29, 9), (128, 100, 40)])
def test_mp_simple_matches_oracle(oracle_lib, shape):
    O = oracle_lib
    c = mp_case(*(11, *shape))
    ref, rain, snow, stop = oracle_mp(O, c, 20.0)
    d = Domain.from_case(c)
    adv_init(d, OPTS)
    mp(d, OPTS, 20.0)
    got = {k: d.fetch(k).copy() for k in FIELDS}
    grain, gsnow = precipitation(d)
    d.close()
    for k in FIELDS:
        assert rel_err(got[k], ref[k]) <= 1e-5, k
        assert np.array_equal(got[k], ref[k]), (k, int((got[k] != ref[k]).sum()))
    assert rel_err(grain, rain) <= 1e-5 and rel_err(gsnow, snow) <= 1e-5
    assert np.array_equal(grain, rain) and np.array_equal(gsnow, snow)
    if shape[2] >= 20:
        assert rain.sum() > 0          # the deeper cases exercise sedimentation


@pytest.mark.parametrize("layout", ["thin", "mixed"])
def test_mp_simple_several_substeps(oracle_lib, layout):
    """Thin levels make the sedimentation take several CFL substeps: those
    columns run the separate passes, the rest the single fused march; with
    "mixed" both kinds sit side by side in every CTA row."""
    O = oracle_lib
    c = mp_case(seed=13, nx=61, ny=47, nz=20)
    dzm = c.dz_mass.copy()
    if layout == "thin":
        dzm *= np.float32(0.05)                       # rain and snow both need several substeps
    else:
        dzm[:, :, ::3] *= np.float32(0.1)            # every third column: rain in several substeps
    c.dz_mass = dzm.astype(np.float32)
    ref, rain, snow, stop = oracle_mp(O, c, 20.0)
    d = Domain.from_case(c)
    adv_init(d, OPTS)
    mp(d, OPTS, 20.0)
    got = {k: d.fetch(k).copy() for k in FIELDS}
    grain, gsnow = precipitation(d)
    d.close()
    for k in FIELDS:
        assert np.array_equal(got[k], ref[k]), (k, int((got[k] != ref[k]).sum()))
    assert np.array_equal(grain, rain) and np.array_equal(gsnow, snow)
    assert rain.sum() > 0


def test_advect_and_mp_steps(oracle_lib):
    """The resident species go through advect -> mp -> advect -> ... on the
    device without a host round trip; five steps stay within 1e-4 of the
    oracle and the accumulations add up across calls."""
    O = oracle_lib
    c = mp_case(seed=4, nx=70, ny=52, nz=16)
    d = Domain.from_case(c)
    adv_init(d, OPTS)
    oc = c.copy()
    rain = snow = None
    ao = O.make_opts()
    for _ in range(5):
        advect(d, OPTS, c.dt)
        mp(d, OPTS, c.dt)
        oc.species = O.advect(oc, ao, oc.dt)
        oc.species, rain, snow, _ = oracle_mp(O, oc, oc.dt, rain, snow)
    got = {k: d.fetch(k).copy() for k in FIELDS}
    grain, gsnow = precipitation(d)
    d.close()
    for k in FIELDS:
        assert rel_err(got[k], oc.species[k]) <= 1e-4, k
        assert np.array_equal(got[k], oc.species[k]), k
    assert rel_err(grain, rain) <= 1e-4 and rel_err(gsnow, snow) <= 1e-4
    assert np.array_equal(grain, rain) and np.array_equal(gsnow, snow)


def test_precipitation_set_and_accumulate(oracle_lib):
    O = oracle_lib
    c = mp_case(seed=6, nx=40, ny=40, nz=12)
    rng = np.random.default_rng(0)
    r0 = rng.random((c.ny, c.nx))
    s0 = rng.random((c.ny, c.nx)) * 0.1
    d = Domain.from_case(c)
    adv_init(d, OPTS)
    lib = L.load()
    L.check(lib.icar_adv_set_precipitation(d.handle, r0.ctypes.data_as(C.c_void_p), s0.ctypes.data_as(C.c_void_p)),
            d.handle)
    mp(d, OPTS, 20.0)
    grain, gsnow = precipitation(d)
    d.close()
    _, rain, snow, _ = oracle_mp(O, c, 20.0, r0, s0)
    assert rel_err(grain, rain) <= 1e-5 and rel_err(gsnow, snow) <= 1e-5


def test_mp_needs_its_fields():
    c = mp_case(seed=7, nx=30, ny=30, nz=8)
    c.pressure = None
    d = Domain.from_case(c)
    adv_init(d, OPTS)
    with pytest.raises(L.IcarAdvError) as e:
        mp(d, OPTS, 20.0)
    assert e.value.code == L.NOT_READY
    d.close()
    c2 = mp_case(seed=7, nx=30, ny=30, nz=8)
    c2.species = {k: c2.species[k] for k in ("theta", "qv", "qc")}
    d = Domain.from_case(c2)
    adv_init(d, OPTS)
    with pytest.raises(L.IcarAdvError) as e:
        mp(d, OPTS, 20.0)
    assert e.value.code == L.BAD_ARG
    d.close()
