"""Fused standard-scheme kernels (k_std_stage / k_std_corr: flux3 and the
update, with WRF_flux_corr, in one z-marching launch per adv_std_advect3d
call) against the CPU oracle and the one-kernel-per-stage path, through the
C ABI.  Bit-exact, like the other parity tests: the fused kernels evaluate
every reference expression in the same order."""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import AdvOptions, Options, Parameters, PhysicsOptions, TimeOptions

from tests.test_parity_gpu import assert_exact, gpu_run

pytestmark = pytest.mark.gpu

ORDERS = [(h, v) for h in (1, 3, 5) for v in (1, 3, 5)]


def std_options(h, v, fc, rk3, den=False) -> Options:
    return Options(physics=PhysicsOptions(advection=1),
                   adv_options=AdvOptions(flux_corr=fc, h_order=h, v_order=v),
                   time_options=TimeOptions(RK3=bool(rk3)), parameters=Parameters(advect_density=den))


@pytest.mark.parametrize("h,v", ORDERS)
@pytest.mark.parametrize("fc,rk3", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_every_order_and_switch(oracle_lib, h, v, fc, rk3):
    """All 9 order pairs x flux correction x RK3 on a shape that leaves
    partial tiles in x and y."""
    O = oracle_lib
    case = synth.config2(seed=h * 10 + v, nx=45, ny=37, nz=11)
    case.species = {k: case.species[k] for k in ("qv", "qc", "qr")}
    o = O.make_opts(advection=1, h_order=h, v_order=v, flux_corr=fc, rk3=rk3)
    ref = O.run_steps(case, o, case.dt, 2)
    assert_exact(gpu_run(case, std_options(h, v, fc, rk3), 2), ref, label=f"h{h} v{v} fc{fc} rk3{rk3} ")


@pytest.mark.parametrize("fc,rk3", [(1, 1), (0, 0)])
def test_advect_density(oracle_lib, fc, rk3):
    O = oracle_lib
    case = synth.config2(seed=21, nx=70, ny=52, nz=14)
    case.species = {k: case.species[k] for k in ("qv", "theta", "ni")}
    o = O.make_opts(advection=1, h_order=5, v_order=3, flux_corr=fc, rk3=rk3, advect_density=1)
    ref = O.run_steps(case, o, case.dt, 3)
    assert_exact(gpu_run(case, std_options(5, 3, fc, rk3, den=True), 3), ref)


@pytest.mark.parametrize("shape", [(9, 9, 4), (10, 13, 4), (33, 9, 6), (9, 41, 5)])
def test_small_and_thin_domains(oracle_lib, shape):
    """Domains just above twice the halo, one-tile grids, shallow columns."""
    O = oracle_lib
    nx, ny, nz = shape
    case = synth.config1(seed=nx + ny + nz, nx=nx, ny=ny, nz=nz)
    o = O.make_opts(advection=1, h_order=5, v_order=5, flux_corr=1, rk3=1)
    ref = O.run_steps(case, o, case.dt, 2)
    assert_exact(gpu_run(case, std_options(5, 5, 1, 1), 2), ref)


def test_full_species_matches_staged_path():
    """256x256x40 with 12 fields, the HICAR default (RK3, 5th/3rd order, WRF
    monotonic correction): fused kernels equal the staged kernels cell for cell."""
    case = synth.config2(seed=31, nx=256, ny=256, nz=40)
    opts = std_options(5, 3, 1, 1)
    fused = gpu_run(case, opts, 3)
    staged = gpu_run(case, opts, 3, staged=True)
    for k in case.species:
        assert np.array_equal(fused[k], staged[k]), k


def test_many_steps_with_forcing(oracle_lib):
    """apply_forcing -> advect for 20 steps on the standard scheme."""
    O = oracle_lib
    case = synth.config2(seed=41, nx=48, ny=44, nz=10)
    case.species = {k: case.species[k] for k in ("qv", "qc")}
    rng = np.random.default_rng(3)
    forcing = {k: (case.species[k] * np.float32(1.05), (rng.standard_normal(case.species[k].shape) * 1e-7).astype(np.float32))
               for k in case.species}
    o = O.make_opts(advection=1, h_order=3, v_order=3, flux_corr=1, rk3=1)
    flt = O.init_relax_filters(case.nx, case.ny, o.halo)
    ref = O.run_steps(case, o, case.dt, 20, forcing=forcing, filter2d=flt)
    assert_exact(gpu_run(case, std_options(3, 3, 1, 1), 20, forcing=forcing), ref)
