"""Wind balance and the stable time step on the GPU (balance_uvw,
wind.f90:88-164; compute_dt, time_step.f90:51-168) against the CPU oracle,
through the C ABI: bit-exact like the advection parity tests."""
import numpy as np
import pytest

from hicar_b200 import _lib as L, synth
from hicar_b200.advection import (AdvOptions, Domain, Options, Parameters, PhysicsOptions, TimeOptions, adv_init,
                                  advect, balance_uvw, compute_dt)

pytestmark = pytest.mark.gpu

# (options, halo): MPDATA -> halo 2; standard upwind -> 1; standard 5th order -> 3
LAYOUTS = [
    (lambda den: Options(parameters=Parameters(advect_density=den)), 2),
    (lambda den: Options(physics=PhysicsOptions(advection=1), parameters=Parameters(advect_density=den)), 1),
    (lambda den: Options(physics=PhysicsOptions(advection=1), adv_options=AdvOptions(h_order=5, v_order=5),
                         parameters=Parameters(advect_density=den)), 3),
]


@pytest.mark.parametrize("layout", range(len(LAYOUTS)))
@pytest.mark.parametrize("den", [False, True])
@pytest.mark.parametrize("shape", [(61, 47, 9), (29, 33, 5), (128, 96, 20)])
def test_balance_uvw_matches_oracle(oracle_lib, layout, den, shape):
    O = oracle_lib
    make, hs = LAYOUTS[layout]
    opts = make(den)
    nx, ny, nz = shape
    case = synth.config2(seed=nx + ny, nx=nx, ny=ny, nz=nz)
    case.w = (case.w * np.float32(1.7) + np.float32(0.01)).astype(np.float32)   # w that needs balancing
    ref = O.balance_uvw(case, hs, int(den))
    d = Domain.from_case(case)
    adv_init(d, opts)
    balance_uvw(d, opts)
    got = d.fetch("w")
    d.close()
    assert np.array_equal(got, ref)


def test_advect_after_balance_uses_the_new_w(oracle_lib):
    """balance_uvw then advect (time_step.f90:324, 373) equals the oracle on
    the balanced w, cell for cell."""
    O = oracle_lib
    case = synth.config2(seed=3, nx=70, ny=54, nz=12)
    opts = Options(parameters=Parameters(advect_density=True))
    d = Domain.from_case(case)
    adv_init(d, opts)
    balance_uvw(d, opts)
    advect(d, opts, case.dt)
    got = {k: d.fetch(k).copy() for k in case.species}
    d.close()
    c2 = case.copy()
    c2.w = O.balance_uvw(case, 2, 1)
    ref = O.advect(c2, O.make_opts(advect_density=1), c2.dt)
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k


@pytest.mark.parametrize("strictness", [1, 2, 3, 4, 5])
def test_compute_dt_matches_oracle(oracle_lib, strictness):
    O = oracle_lib
    case = synth.config2(seed=11, nx=90, ny=70, nz=15)
    dz = np.asarray(case.dz_levels, np.float32)
    opts = Options(time_options=TimeOptions(cfl_reduction_factor=0.9, cfl_strictness=strictness))
    ref, small = O.compute_dt(case, 2, dz, 0.9, strictness)
    d = Domain.from_case(case)
    adv_init(d, opts)
    if small:
        with pytest.raises(L.IcarAdvError) as e:
            compute_dt(d, opts, dz)
        assert e.value.code == L.CFL_VIOLATION
    else:
        assert compute_dt(d, opts, dz) == ref
    d.close()


def test_compute_dt_after_balance(oracle_lib):
    """The time step of the balanced winds (the balanced w enters the per-cell
    vertical rate)."""
    O = oracle_lib
    case = synth.config2(seed=12, nx=64, ny=64, nz=16)
    dz = np.asarray(case.dz_levels, np.float32)
    opts = Options(parameters=Parameters(advect_density=True))
    d = Domain.from_case(case)
    adv_init(d, opts)
    balance_uvw(d, opts)
    got = compute_dt(d, opts, dz)
    d.close()
    c2 = case.copy()
    c2.w = O.balance_uvw(case, 2, 1)
    ref, small = O.compute_dt(c2, 2, dz, 0.9, 3)
    assert not small and got == ref
