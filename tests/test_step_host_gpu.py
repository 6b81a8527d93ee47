"""icar_adv_step_host: one step for species held in host memory (upload ->
apply_forcing -> advect -> enforce_limits -> download, pipelined by species
group on the fused kernels) equals the same step done with per-field
set_field / icar_adv_step / get_field, bit for bit, through the C ABI."""
import ctypes as C

import numpy as np
import pytest
import torch

from hicar_b200 import _lib as L, synth
from hicar_b200.advection import (AdvOptions, Domain, Options, PhysicsOptions, TimeOptions, adv_init, step,
                                  step_host)

pytestmark = pytest.mark.gpu

SCHEMES = {
    "mpdata": Options(),
    "mpdata_staged": Options(),
    "std_rk3_wrf": Options(physics=PhysicsOptions(advection=1), adv_options=AdvOptions(h_order=5, v_order=3, flux_corr=1),
                           time_options=TimeOptions(RK3=True)),
    "std_plain": Options(physics=PhysicsOptions(advection=1), adv_options=AdvOptions(h_order=3, v_order=3)),
}


def forced_domain(case, opts, staged):
    d = Domain.from_case(case)
    rng = np.random.default_rng(7)
    for k in ("qv", "qc"):
        d.set_forcing(k, (case.species[k] * np.float32(1.03)).astype(np.float32),
                      (rng.standard_normal(case.species[k].shape) * 1e-8).astype(np.float32))
    adv_init(d, opts)
    if staged:
        d.use_staged_kernels(True)
    return d


def pinned_like(a: np.ndarray) -> np.ndarray:
    t = torch.empty(a.shape, dtype=torch.float32).pin_memory()
    v = t.numpy()
    v[...] = a
    return v


@pytest.mark.parametrize("scheme", list(SCHEMES))
@pytest.mark.parametrize("pinned", [True, False])
def test_step_host_equals_set_step_get(scheme, pinned):
    opts = SCHEMES[scheme]
    case = synth.config2(seed=12, nx=90, ny=70, nz=16)
    staged = scheme.endswith("staged")
    ref = forced_domain(case, opts, staged)
    got = forced_domain(case, opts, staged)
    host = {k: (pinned_like(v) if pinned else v.copy()) for k, v in case.species.items()}
    for n in range(4):
        enforce = n % 2 == 1
        # reference: per-field uploads, the step, per-field downloads
        for k, a in host.items():
            ref.upload(k, a)
        step(ref, opts, case.dt, enforce_limits=enforce)
        want = {k: ref.fetch(k).copy() for k in host}
        # pipelined host step, results written back in place
        step_host(got, opts, case.dt, host, host, enforce_limits=enforce)
        for k in host:
            assert np.array_equal(host[k], want[k]), f"{scheme} step {n} {k}"
        # perturb the host state as CPU physics would between calls
        for k in host:
            host[k] *= np.float32(0.999)
    ref.close()
    got.close()


def test_step_host_rejects_bad_arguments():
    case = synth.config1(seed=3, nx=32, ny=28, nz=8)
    d = Domain.from_case(case)
    adv_init(d, Options())
    lib = L.load()
    assert lib.icar_adv_step_host(d.handle, C.c_double(1.0), 0, None, None) == L.BAD_ARG
    arr = (C.c_void_p * 1)(None)
    assert lib.icar_adv_step_host(d.handle, C.c_double(1.0), 0, arr, arr) == L.BAD_ARG
    buf = case.species["qv"].copy()
    ok = (C.c_void_p * 1)(buf.ctypes.data)
    assert lib.icar_adv_step_host(d.handle, C.c_double(float("nan")), 0, ok, ok) == L.BAD_ARG
    assert lib.icar_adv_step_host(None, C.c_double(1.0), 0, ok, ok) == L.BAD_ARG
    with pytest.raises(ValueError):
        step_host(d, Options(), 1.0, {"qv": np.zeros((3, 3, 3), np.float32)})
    d.close()


def test_bounded_wait_reports_timeout_then_completes(oracle_lib):
    """icar_adv_sync_timeout: with 30 steps of a 256x256x40 x 12-field
    domain queued (tens of milliseconds of device work), a zero timeout
    returns ICAR_ADV_TIMEOUT and leaves the work queued; a generous one then
    returns OK, and the result equals the same steps waited for with
    icar_adv_sync.  Nothing on the device is made to hang: the work simply
    has not finished when the first wait gives up."""
    from hicar_b200 import synth
    from hicar_b200.advection import Domain, Options, adv_init, advect
    case = synth.config2(seed=12, nx=256, ny=256, nz=40)
    opts = Options()
    outs = []
    for bounded in (True, False):
        d = Domain.from_case(case)
        adv_init(d, opts)
        d.sync()
        for _ in range(30):
            advect(d, opts, case.dt)
        if bounded:
            assert d.wait(0.0) is False
            assert d.wait(120.0) is True
        else:
            d.sync()
        outs.append({k: d.fetch(k).copy() for k in ("qv", "theta")})
        d.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k])
