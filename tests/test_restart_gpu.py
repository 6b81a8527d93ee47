"""Restart download and upload through the C ABI (row: device download into
the options%restart_vars set, adv_std_var_request, advect.f90:95-107).

icar_adv_download copies several resident fields in one call with one wait
on the device; icar_adv_upload writes them back.  A run that is stopped,
downloaded, and resumed on a fresh handle from the downloaded fields must
continue bit for bit like the uninterrupted run."""
import ctypes as C

import numpy as np
import pytest

from hicar_b200 import _lib as L, synth
from hicar_b200.advection import Domain, Options, adv_init, advect

pytestmark = pytest.mark.gpu


def restart_case(seed=5, nx=61, ny=47, nz=12):
    c = synth.config2(seed=seed, nx=nx, ny=ny, nz=nz)
    d = Domain.from_case(c)
    # dz_interface is only carried for the restart: any (nx, nz, ny) field
    d.dz_interface = (c.advection_dz * np.float32(1.01)).astype(np.float32)
    return c, d


def test_download_restart_equals_per_field_fetch():
    c, d = restart_case()
    opts = Options()
    adv_init(d, opts)
    for _ in range(3):
        advect(d, opts, c.dt)
    assert d.restart_vars() == ["u", "v", "w", "dz_interface", "qv"]
    got = d.download_restart()
    assert got["u"].shape == (c.ny, c.nz, c.nx + 1) and got["v"].shape == (c.ny + 1, c.nz, c.nx)
    for name in ("u", "v", "w"):
        assert np.array_equal(got[name], getattr(c, name)), name
    assert np.array_equal(got["dz_interface"], d.dz_interface)
    per_field = d.fetch("qv").copy()
    assert np.array_equal(got["qv"], per_field)
    assert not np.array_equal(got["qv"], c.species["qv"])     # it did advance
    d.close()


def test_resume_from_downloaded_fields_is_bit_exact():
    c, a = restart_case(seed=8)
    opts = Options()
    adv_init(a, opts)
    for _ in range(6):
        advect(a, opts, c.dt)
    ref = a.download(list(c.species))
    a.close()

    _, b = restart_case(seed=8)
    adv_init(b, opts)
    for _ in range(3):
        advect(b, opts, c.dt)
    saved = b.download(b.restart_vars() + [k for k in c.species if k != "qv"])
    b.close()

    _, r = restart_case(seed=8)
    r.dz_interface = None
    adv_init(r, opts)
    r.restore_restart(saved)
    got_dzi = r.download(["dz_interface"])["dz_interface"]
    assert np.array_equal(got_dzi, saved["dz_interface"])
    for _ in range(3):
        advect(r, opts, c.dt)
    got = r.download(list(c.species))
    r.close()
    for k in c.species:
        assert np.array_equal(got[k], ref[k]), k


def test_bulk_calls_validate_their_arguments():
    c, d = restart_case(nx=29, ny=33, nz=5)
    opts = Options()
    adv_init(d, opts)
    lib = L.load()
    assert d.download([]) == {}
    ids = (C.c_int32 * 1)(9999)
    buf = np.zeros(8, np.float32)
    ptrs = (C.c_void_p * 1)(buf.ctypes.data)
    assert lib.icar_adv_download(d.handle, 1, ids, ptrs) == L.BAD_ARG
    ptrs0 = (C.c_void_p * 1)(None)
    ids[0] = L.F_QV
    assert lib.icar_adv_download(d.handle, 1, ids, ptrs0) == L.BAD_ARG
    assert lib.icar_adv_download(d.handle, -1, ids, ptrs) == L.BAD_ARG
    with pytest.raises(ValueError):
        d.upload_many({"u": np.zeros((c.ny, c.nz, c.nx), np.float32)})
    d.close()
