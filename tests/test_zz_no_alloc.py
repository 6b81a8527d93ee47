"""icar_adv_advect_noalloc: the MPDATA step for callers that cannot allocate
device memory (a host framework's pool owns every allocation, or the call
sits in a region where cudaMalloc would synchronise or break a capture).

The test owns all inputs and outputs (allocated here with torch, in the
library's pitched device layout) and calls the entry point through the C
ABI twice in a row, feeding the first output back in, and checks each
result against the handle API (icar_adv_create / icar_adv_advect) on the
same case, to the same standard as the other parity tests: bit-exact, and
within 1e-5 relative error.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from hicar_b200 import _lib as L, synth
from hicar_b200.advection import Domain, Options, AdvOptions, adv_init, advect

pytestmark = pytest.mark.gpu


def pitched(torch, arr: np.ndarray, nx_eff: int, P: int):
    """Copy a (rows, nz, nx_eff) Fortran-layout array into a pitched device buffer."""
    rows, nz, _ = arr.shape
    host = np.zeros((rows, nz, P), np.float32)
    host[:, :, :nx_eff] = arr
    return torch.from_numpy(host.reshape(-1)).cuda()


def unpitch(t, rows: int, nz: int, nx: int, P: int) -> np.ndarray:
    return t.cpu().numpy().reshape(rows, nz, P)[:, :, :nx].copy()


def rel_err(a, ref):
    ref = ref.astype(np.float64)
    scale = max(float(np.abs(ref).max()), 1e-30)
    return float((np.abs(a.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-6 * scale)).max())


@pytest.mark.parametrize("fct", [1, 0])
def test_noalloc_matches_handle_api_on_two_calls(fct):
    import torch
    lib = L.load()
    case = synth.config2(seed=31, nx=61, ny=47, nz=14)
    case.species = {k: case.species[k] for k in ("qv", "qc", "nr", "theta")}
    nx, ny, nz = case.nx, case.ny, case.nz
    P = ((nx + 1) + 3) // 4 * 4
    torch.cuda.set_device(0)
    dev = {
        "u": pitched(torch, case.u, nx + 1, P), "v": pitched(torch, case.v, nx, P),
        "w": pitched(torch, case.w, nx, P), "density": pitched(torch, case.density, nx, P),
        "jacobian": pitched(torch, case.jacobian, nx, P), "jacobian_u": pitched(torch, case.jacobian_u, nx + 1, P),
        "jacobian_v": pitched(torch, case.jacobian_v, nx, P), "jacobian_w": pitched(torch, case.jacobian_w, nx, P),
        "advection_dz": pitched(torch, case.advection_dz, nx, P),
    }
    names = list(case.species)
    bufs = [{k: pitched(torch, case.species[k], nx, P) for k in names},
            {k: torch.zeros(P * nz * ny, dtype=torch.float32, device="cuda") for k in names}]
    stream = torch.cuda.current_stream()

    def call(src, dst):
        a = L.NoallocArgs()
        a.nx, a.ny, a.nz, a.dx, a.dt = nx, ny, nz, case.dx, case.dt
        a.mpdata_fct, a.advect_density, a.n_species = fct, 0, len(names)
        for f, t in dev.items():
            setattr(a, f, C.c_void_p(t.data_ptr()))
        for s, k in enumerate(names):
            a.q_in[s] = src[k].data_ptr()
            a.q_out[s] = dst[k].data_ptr()
        a.stream = stream.cuda_stream
        rc = lib.icar_adv_advect_noalloc(C.byref(a))
        assert rc == L.OK, lib.icar_adv_last_error(None)

    # the existing entry point on the same case, one step at a time
    opts = Options(adv_options=AdvOptions(MPDATA_FCT=bool(fct)))
    d = Domain.from_case(case)
    adv_init(d, opts)
    for n in range(2):
        call(bufs[n % 2], bufs[(n + 1) % 2])
        torch.cuda.synchronize()
        advect(d, opts, case.dt)
        for k in names:
            got = unpitch(bufs[(n + 1) % 2][k], ny, nz, nx, P)
            ref = d.fetch(k)
            assert rel_err(got, ref) <= 1e-5, (n, k)
            assert np.array_equal(got, ref), (n, k)
    d.close()


def test_noalloc_rejects_domains_beyond_the_static_scratch():
    import torch
    lib = L.load()
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    a = L.NoallocArgs()
    a.nx, a.ny, a.nz, a.dx, a.dt, a.mpdata_fct, a.n_species = 512, 512, 40, 1000.0, 4.0, 1, 1
    for f in ("u", "v", "w", "density", "jacobian", "jacobian_u", "jacobian_v", "jacobian_w", "advection_dz"):
        setattr(a, f, C.c_void_p(buf.data_ptr()))
    a.q_in[0] = buf.data_ptr()
    a.q_out[0] = buf.data_ptr() + 16
    rc = lib.icar_adv_advect_noalloc(C.byref(a))
    assert rc == L.BAD_ARG
    msg = lib.icar_adv_last_error(None).decode()
    assert "static scratch holds" in msg and "512x512x40" in msg
