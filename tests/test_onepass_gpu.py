"""Single-pass MPDATA kernel (donor-cell pass, pseudo-velocities, FCT
limiter and corrective pass in one launch per advect call).

The bit-exact variant must equal the FP32 oracle cell for cell on every case
the two-kernel path is held to: ragged shapes at every tile offset, FCT on
and off, the golden fixtures, extreme magnitudes, several steps.  The
fast-arithmetic variant is checked against the same oracle within a stated
tolerance (see test_onepass_fast_gpu.py).
"""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import Domain, Options, AdvOptions, adv_init, advect, step

pytestmark = pytest.mark.gpu

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def run(case, nsteps, fct=1, fast=False, forcing=None):
    opts = Options(adv_options=AdvOptions(MPDATA_FCT=bool(fct)))
    d = Domain.from_case(case)
    for k, (fh, dq) in (forcing or {}).items():
        d.set_forcing(k, fh, dq)
    adv_init(d, opts)
    d.use_single_pass(fast=fast)
    for _ in range(nsteps):
        if forcing:
            step(d, opts, case.dt)
        else:
            advect(d, opts, case.dt)
    out = {k: d.fetch(k).copy() for k in case.species}
    d.sync()
    d.close()
    return out


def assert_same(out, ref, label=""):
    for k in ref:
        nd = int((out[k] != ref[k]).sum())
        if nd:
            bad = np.argwhere(out[k] != ref[k])
            j, kk, i = bad[0]
            raise AssertionError(f"{label}{k}: {nd} cells differ from the FP32 oracle; first at (j={j}, k={kk}, "
                                 f"i={i}): {out[k][j, kk, i]!r} vs {ref[k][j, kk, i]!r}")


@pytest.mark.parametrize("nx,ny,nz", [(3, 3, 3), (30, 18, 3), (29, 17, 5), (57, 33, 7), (100, 70, 41),
                                      (31, 200, 4), (113, 53, 9), (56, 26, 6), (57, 27, 6)])
def test_exact_single_pass_matches_oracle_on_ragged_shapes(oracle_lib, nx, ny, nz):
    O = oracle_lib
    case = synth.config2(seed=nx + ny + nz, nx=nx, ny=ny, nz=nz)
    case.species = {k: case.species[k] for k in ("qv", "qc", "nr", "theta")}
    for fct in (1, 0):
        ref = O.run_steps(case, O.make_opts(mpdata_fct=fct), case.dt, 3)
        assert_same(run(case, 3, fct=fct), ref, label=f"{nx}x{ny}x{nz} fct={fct} ")


def test_exact_single_pass_golden_fixtures(oracle_lib):
    from tests.golden import make_golden as G
    for name, (case, o, nsteps) in G.cases(oracle_lib).items():
        if o.advection != 2 or o.mpdata_order != 2 or o.rk3:
            continue
        ref = dict(np.load(GOLDEN / f"{name}.npz"))
        assert_same(run(case, nsteps, fct=o.mpdata_fct), ref, label=f"{name} ")


def test_exact_single_pass_config2_reduced(oracle_lib):
    O = oracle_lib
    case = synth.config2(seed=5, nx=96, ny=80, nz=24)
    ref = O.run_steps(case, O.make_opts(), case.dt, 5)
    assert_same(run(case, 5), ref)


@pytest.mark.parametrize("scale", [1e-28, 1e-36, 1e30, 1.0])
def test_exact_single_pass_extreme_magnitudes(oracle_lib, scale):
    O = oracle_lib
    case = synth.config2(seed=44, nx=61, ny=47, nz=9)
    case.species = {k: case.species[k] for k in ("qv", "qc", "nr", "theta")}
    rng = np.random.default_rng(3)
    for k, q in case.species.items():
        if scale == 1.0:
            tiny = rng.random(q.shape) < 0.3
            case.species[k] = np.where(tiny, np.float32(1e-33) * rng.random(q.shape).astype(np.float32), q)
        else:
            case.species[k] = (q * np.float32(scale)).astype(np.float32)
    for fct in (1, 0):
        ref = O.run_steps(case, O.make_opts(mpdata_fct=fct), case.dt, 3)
        assert_same(run(case, 3, fct=fct), ref, label=f"scale={scale} fct={fct} ")


def test_exact_single_pass_with_boundary_forcing(oracle_lib):
    O = oracle_lib
    case = synth.config1(seed=8, nx=64, ny=48, nz=12)
    rng = np.random.default_rng(1)
    fh = (case.species["qv"] * 1.1).astype(np.float32)
    dq = (rng.standard_normal(fh.shape) * 1e-7).astype(np.float32)
    flt = O.init_relax_filters(case.nx, case.ny, 2)
    ref = O.run_steps(case, O.make_opts(), case.dt, 10, forcing={"qv": (fh, dq)}, filter2d=flt)
    assert_same(run(case, 10, forcing={"qv": (fh, dq)}), ref)
