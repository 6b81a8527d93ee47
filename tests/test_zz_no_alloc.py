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


def pitched(torch, arr: np.ndarray, nx_eff: int, P: int, pad: float = 0.0):
    """Copy a (rows, nz, nx_eff) Fortran-layout array into a pitched device
    buffer whose padding columns [nx_eff, P) hold `pad`."""
    rows, nz, _ = arr.shape
    host = np.full((rows, nz, P), pad, np.float32)
    host[:, :, :nx_eff] = arr
    return torch.from_numpy(host.reshape(-1)).cuda()


def unpitch(t, rows: int, nz: int, nx: int, P: int) -> np.ndarray:
    return t.cpu().numpy().reshape(rows, nz, P)[:, :, :nx].copy()


def rel_err(a, ref):
    ref = ref.astype(np.float64)
    scale = max(float(np.abs(ref).max()), 1e-30)
    return float((np.abs(a.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-6 * scale)).max())


@pytest.mark.parametrize("fct,pad", [(1, 0.0), (0, 0.0), (1, float("nan")), (1, 1e30)])
def test_noalloc_matches_handle_api_on_two_calls(fct, pad):
    """pad fills the padding columns of every input and of the outputs: the
    header promises that input padding is ignored and output padding left
    untouched, so NaN or 1e30 there must change nothing."""
    import torch
    lib = L.load()
    case = synth.config2(seed=31, nx=61, ny=47, nz=14)
    case.species = {k: case.species[k] for k in ("qv", "qc", "nr", "theta")}
    nx, ny, nz = case.nx, case.ny, case.nz
    P = ((nx + 1) + 3) // 4 * 4
    torch.cuda.set_device(0)
    dev = {
        "u": pitched(torch, case.u, nx + 1, P, pad), "v": pitched(torch, case.v, nx, P, pad),
        "w": pitched(torch, case.w, nx, P, pad), "density": pitched(torch, case.density, nx, P, pad),
        "jacobian": pitched(torch, case.jacobian, nx, P, pad),
        "jacobian_u": pitched(torch, case.jacobian_u, nx + 1, P, pad),
        "jacobian_v": pitched(torch, case.jacobian_v, nx, P, pad),
        "jacobian_w": pitched(torch, case.jacobian_w, nx, P, pad),
        "advection_dz": pitched(torch, case.advection_dz, nx, P, pad),
    }
    names = list(case.species)
    bufs = [{k: pitched(torch, case.species[k], nx, P, pad) for k in names},
            {k: torch.full((P * nz * ny,), pad, dtype=torch.float32, device="cuda") for k in names}]
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
            full = bufs[(n + 1) % 2][k].cpu().numpy().reshape(ny, nz, P)
            got = full[:, :, :nx].copy()
            ref = d.fetch(k)
            assert rel_err(got, ref) <= 1e-5, (n, k)
            assert np.array_equal(got, ref), (n, k)
            padding = full[:, :, nx:]
            assert np.array_equal(padding, np.full_like(padding, pad), equal_nan=True), (n, k, "padding changed")
    d.close()


def _args_for(L, buf, nx=32, ny=24, nz=8):
    a = L.NoallocArgs()
    a.nx, a.ny, a.nz, a.dx, a.dt, a.mpdata_fct, a.n_species = nx, ny, nz, 1000.0, 4.0, 1, 1
    return a


def test_noalloc_rejects_misaligned_and_overlapping_arrays():
    """Checks made on the host before any launch: a q_in that is not 16-byte
    aligned, an output that overlaps an input, and two outputs that overlap
    all get BAD_ARG with a message."""
    import torch
    lib = L.load()
    nx, ny, nz = 32, 24, 8
    P = ((nx + 1) + 3) // 4 * 4
    n = P * nz * (ny + 1)
    fields = {f: torch.zeros(n, dtype=torch.float32, device="cuda")
              for f in ("u", "v", "w", "density", "jacobian", "jacobian_u", "jacobian_v", "jacobian_w",
                        "advection_dz")}
    qa = torch.zeros(3 * n, dtype=torch.float32, device="cuda")

    def run(q_in, q_out, n_species=1):
        a = _args_for(L, None, nx, ny, nz)
        a.n_species = n_species
        for f, t in fields.items():
            setattr(a, f, C.c_void_p(t.data_ptr()))
        for s in range(n_species):
            a.q_in[s] = q_in[s]
            a.q_out[s] = q_out[s]
        return lib.icar_adv_advect_noalloc(C.byref(a)), lib.icar_adv_last_error(None).decode()

    base = qa.data_ptr()
    rc, msg = run([base + 4], [base + n * 4])
    assert rc == L.BAD_ARG and "16-byte aligned" in msg
    rc, msg = run([base], [base + 16 * 4])                      # q_out inside q_in
    assert rc == L.BAD_ARG and "overlaps q_in[0]" in msg
    rc, msg = run([base, base + n * 4], [base + 2 * n * 4, base + 2 * n * 4 + 64], n_species=2)
    assert rc == L.BAD_ARG and "overlaps q_out" in msg
    rc, msg = run([base, base + n * 4], [base + 2 * n * 4, base], n_species=2)  # output of 1 = input of 0
    assert rc == L.BAD_ARG and "overlaps q_in[0]" in msg
    rc, msg = run([base], [fields["u"].data_ptr()])
    assert rc == L.BAD_ARG and "overlaps u" in msg


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
