"""GPU parity: the sm_100a kernels against the CPU oracle, through the C ABI.

Every kernel evaluates the reference's FP32 expressions in the same order
without fused multiply-adds, so the bar is bit-exact equality with the FP32
oracle (np.array_equal); the error against the FP64 oracle is reported as
well.  The path's stated tolerance (max relative error <= 1e-5 per step,
<= 1e-4 after 100 steps) is asserted too, so a deliberate relaxation of the
arithmetic would still be judged against it.
"""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import Domain, Options, AdvOptions, PhysicsOptions, TimeOptions, adv_init, advect, step

pytestmark = pytest.mark.gpu

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def rel_err(a, ref):
    """max |a-ref| / max(|ref|, floor), floor = 1e-6 * max|ref| (zeros are common)."""
    ref = ref.astype(np.float64)
    scale = max(float(np.abs(ref).max()), 1e-30)
    den = np.maximum(np.abs(ref), 1e-6 * scale)
    return float((np.abs(a.astype(np.float64) - ref) / den).max())


def options_from(o) -> Options:
    return Options(physics=PhysicsOptions(advection=o.advection),
                   adv_options=AdvOptions(MPDATA_FCT=bool(o.mpdata_fct), mpdata_order=o.mpdata_order,
                                          flux_corr=o.flux_corr, h_order=o.h_order, v_order=o.v_order),
                   time_options=TimeOptions(RK3=bool(o.rk3)))


def gpu_run(case, opts: Options, nsteps: int, staged=False, forcing=None, fetch_each=False):
    d = Domain.from_case(case)
    for k, (fh, dq) in (forcing or {}).items():
        d.set_forcing(k, fh, dq)
    adv_init(d, opts)
    if staged:
        d.use_staged_kernels(True)
    for _ in range(nsteps):
        if forcing:
            step(d, opts, case.dt)
        else:
            advect(d, opts, case.dt)
    out = {k: d.fetch(k).copy() for k in case.species}
    d.close()
    return out


def assert_exact(out, ref, tol=1e-5, label=""):
    for k in ref:
        e = rel_err(out[k], ref[k])
        assert e <= tol, f"{label}{k}: rel err {e:.3e} > {tol}"
        nd = int((out[k] != ref[k]).sum())
        assert nd == 0, f"{label}{k}: {nd} cells differ from the FP32 oracle (max rel err {e:.3e})"


def test_golden_fixtures_gpu(oracle_lib):
    from tests.golden import make_golden as G
    for name, (case, o, nsteps) in G.cases(oracle_lib).items():
        ref = dict(np.load(GOLDEN / f"{name}.npz"))
        for staged in (False, True):
            out = gpu_run(case, options_from(o), nsteps, staged=staged)
            assert_exact(out, ref, label=f"{name} staged={staged} ")


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-5), (100, 1e-4)])
def test_config1_mpdata(oracle_lib, nsteps, tol):
    """Config 1 (128x128x20, qv, MPDATA order 2 + FCT, dt 20 s)."""
    O = oracle_lib
    case = synth.config1(seed=11)
    ref = O.run_steps(case, O.make_opts(), case.dt, nsteps)
    out = gpu_run(case, Options(), nsteps)
    assert_exact(out, ref, tol)
    ref64 = O.run_steps(case, O.make_opts(), case.dt, nsteps, dtype=np.float64)
    e64 = rel_err(out["qv"], ref64["qv"])
    print(f"config1 {nsteps} steps: error vs FP64 oracle {e64:.3e}")
    assert e64 < tol


def test_config2_reduced_12_species(oracle_lib):
    O = oracle_lib
    case = synth.config2(seed=5, nx=96, ny=80, nz=24)
    ref = O.run_steps(case, O.make_opts(), case.dt, 5)
    assert_exact(gpu_run(case, Options(), 5), ref)
    assert_exact(gpu_run(case, Options(), 5, staged=True), ref)


def test_config2_full_size_one_step(oracle_lib):
    """512x512x40 with 12 fields, one step, cell for cell against the oracle."""
    O = oracle_lib
    case = synth.config2(seed=2)
    ref = O.run_steps(case, O.make_opts(), case.dt, 1)
    assert_exact(gpu_run(case, Options(), 1), ref)


@pytest.mark.parametrize("h,v,fc,rk3", [(1, 1, 0, 0), (3, 3, 0, 0), (5, 5, 0, 0), (5, 3, 1, 0), (1, 1, 1, 0),
                                        (3, 3, 1, 1), (5, 5, 0, 1)])
def test_standard_scheme(oracle_lib, h, v, fc, rk3):
    O = oracle_lib
    case = synth.config2(seed=9, nx=64, ny=56, nz=16)
    case.species = {k: case.species[k] for k in ("qv", "qc", "theta")}
    o = O.make_opts(advection=1, h_order=h, v_order=v, flux_corr=fc, rk3=rk3)
    ref = O.run_steps(case, o, case.dt, 3)
    assert_exact(gpu_run(case, options_from(o), 3), ref, label=f"std h{h} v{v} fc{fc} rk3{rk3} ")


@pytest.mark.parametrize("fct,order", [(0, 2), (1, 1), (1, 3)])
def test_mpdata_switches(oracle_lib, fct, order):
    O = oracle_lib
    case = synth.config2(seed=4, nx=48, ny=40, nz=12)
    o = O.make_opts(mpdata_fct=fct, mpdata_order=order)
    ref = O.run_steps(case, o, case.dt, 3)
    assert_exact(gpu_run(case, options_from(o), 3), ref)


def test_mpdata_rk3_is_a_noop(oracle_lib):
    case = synth.config1(seed=3, nx=32, ny=32, nz=8)
    opts = Options(time_options=TimeOptions(RK3=True))
    out = gpu_run(case, opts, 2)
    assert np.array_equal(out["qv"], case.species["qv"])


def test_boundary_forcing_step(oracle_lib):
    """apply_forcing (relaxation zone, real64 dt) followed by advect, 20 steps,
    with a drifting forcing field."""
    O = oracle_lib
    case = synth.config1(seed=8, nx=64, ny=48, nz=12)
    rng = np.random.default_rng(1)
    fh = (case.species["qv"] * 1.1).astype(np.float32)
    dq = (rng.standard_normal(fh.shape) * 1e-7).astype(np.float32)
    flt = O.init_relax_filters(case.nx, case.ny, 2)
    ref = O.run_steps(case, O.make_opts(), case.dt, 20, forcing={"qv": (fh, dq)}, filter2d=flt)
    out = gpu_run(case, Options(), 20, forcing={"qv": (fh, dq)})
    assert_exact(out, ref)


def test_boundary_forcing_several_species(oracle_lib):
    """One apply_forcing launch covers every forced species, each with its own
    forcing and tendency; one species is left unforced."""
    O = oracle_lib
    case = synth.config2(seed=4, nx=48, ny=40, nz=10)
    rng = np.random.default_rng(2)
    forcing = {}
    for n, k in enumerate(case.species):
        if k == "qr":
            continue
        q = case.species[k]
        fh = (q * np.float32(1.0 + 0.02 * (n + 1))).astype(np.float32)
        dq = (rng.standard_normal(q.shape) * 1e-6 * float(np.abs(q).max())).astype(np.float32)
        forcing[k] = (fh, dq)
    flt = O.init_relax_filters(case.nx, case.ny, 2)
    ref = O.run_steps(case, O.make_opts(), case.dt, 6, forcing=forcing, filter2d=flt)
    out = gpu_run(case, Options(), 6, forcing=forcing)
    assert_exact(out, ref)


def test_relax_filter_matches_oracle(oracle_lib):
    case = synth.config1(seed=1, nx=50, ny=40, nz=6)
    d = Domain.from_case(case)
    adv_init(d, Options())
    assert np.array_equal(d.relax_filter(), oracle_lib.init_relax_filters(50, 40, 2))
    d.close()


def test_enforce_limits_gpu(oracle_lib):
    case = synth.config1(seed=2, nx=40, ny=30, nz=6)
    rng = np.random.default_rng(0)
    case.species["qv"] = rng.standard_normal(case.species["qv"].shape).astype(np.float32)
    d = Domain.from_case(case)
    adv_init(d, Options())
    d.enforce_limits()
    q = d.fetch("qv")
    ref = case.species["qv"].copy()
    oracle_lib.enforce_limits(ref)
    assert np.array_equal(q, ref)
    d.close()


def test_positivity_where_reference_guarantees_it(oracle_lib):
    """Donor cell (order 1) keeps non-negative fields non-negative, exactly;
    with FCT the GPU is negative only where the oracle is."""
    O = oracle_lib
    case = synth.config2(seed=6, nx=64, ny=48, nz=16)
    case.species = {k: case.species[k] for k in ("qc", "qr", "nr")}
    out1 = gpu_run(case, options_from(O.make_opts(mpdata_order=1)), 5)
    for q in out1.values():
        assert (q >= 0).all()
    ref = O.run_steps(case, O.make_opts(), case.dt, 5)
    out2 = gpu_run(case, Options(), 5)
    for k in ref:
        assert np.array_equal(out2[k] < 0, ref[k] < 0)


def test_closed_domain_mass_gpu(oracle_lib):
    case = synth.config1(nx=64, ny=64, nz=16)
    y, z, x = np.meshgrid(np.arange(case.ny), np.arange(case.nz), np.arange(case.nx), indexing="ij")
    case.species = {"qv": np.exp(-(((x - 24) / 5.0) ** 2 + ((y - 32) / 5.0) ** 2 + ((z - 6) / 1.5) ** 2)).astype(np.float32)}
    m = lambda q: float((q.astype(np.float64) * case.jacobian * case.density * case.advection_dz).sum())
    out = gpu_run(case, Options(), 50)
    assert abs(m(out["qv"]) - m(case.species["qv"])) / m(case.species["qv"]) < 2e-6


@pytest.mark.parametrize("nx,ny,nz", [(3, 3, 3), (30, 18, 3), (29, 17, 5), (57, 33, 7), (100, 70, 41), (31, 200, 4)])
def test_fused_matches_oracle_on_ragged_shapes(oracle_lib, nx, ny, nz):
    """Tile edges of the fused kernel (28-column tiles) at every offset,
    the smallest legal domain and short/tall columns."""
    O = oracle_lib
    case = synth.config2(seed=nx + ny + nz, nx=nx, ny=ny, nz=nz)
    case.species = {k: case.species[k] for k in ("qv", "qc", "nr", "theta")}
    for fct in (1, 0):
        o = O.make_opts(mpdata_fct=fct)
        ref = O.run_steps(case, o, case.dt, 3)
        assert_exact(gpu_run(case, options_from(o), 3), ref, label=f"{nx}x{ny}x{nz} fct={fct} ")


def test_fused_and_staged_agree_over_many_steps(oracle_lib):
    case = synth.config2(seed=21, nx=90, ny=75, nz=20)
    a = gpu_run(case, Options(), 40)
    b = gpu_run(case, Options(), 40, staged=True)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("scale", [1e-28, 1e-36, 1e30, 1.0])
def test_fused_exact_at_extreme_magnitudes(oracle_lib, scale):
    """Fields scaled to the edges of the FP32 range: subnormal values and
    quotients (1e-28, 1e-36), values near the overflow threshold (1e30),
    and tiny values (below 1e-33) mixed into ordinary ones.  The fused
    kernel still equals the oracle cell for cell."""
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
        o = O.make_opts(mpdata_fct=fct)
        ref = O.run_steps(case, o, case.dt, 3)
        assert_exact(gpu_run(case, options_from(o), 3), ref, label=f"scale={scale} fct={fct} ")
