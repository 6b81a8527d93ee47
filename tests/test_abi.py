"""C ABI: the library loads, exports every entry point of include/icar_adv.h,
and its host-only calls behave (no device work; runs without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "icar_adv.h"


def _header_functions():
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(icar_adv_\w+)\s*\(", txt)))


def test_library_exports_every_header_symbol(cuda_lib):
    lib = cuda_lib.load()
    declared = _header_functions()
    assert len(declared) >= 18
    for name in declared:
        assert hasattr(lib, name), name
    # the Python binding covers the same set (plus the internal path selector)
    assert set(declared) <= set(cuda_lib.exported_symbols())


def test_abi_version_and_defaults(cuda_lib):
    lib = cuda_lib.load()
    assert lib.icar_adv_abi_version() == 1
    o = cuda_lib.Opts()
    assert lib.icar_adv_default_opts(C.byref(o)) == 0
    # adv_parameters_namelist defaults (options_obj.f90:1576-1582)
    assert (o.advection, o.mpdata_fct, o.mpdata_order, o.flux_corr, o.h_order, o.v_order) == (2, 1, 2, 0, 1, 1)


@pytest.mark.parametrize("adv,h,v,fc,expect", [(2, 1, 1, 0, 2), (1, 1, 1, 0, 1), (1, 3, 3, 0, 2),
                                               (1, 5, 3, 0, 3), (1, 1, 1, 1, 2), (1, 5, 5, 1, 4)])
def test_halo_size_matches_reference(cuda_lib, adv, h, v, fc, expect):
    lib = cuda_lib.load()
    o = cuda_lib.Opts(adv, 1, 2, fc, h, v, 0, 0, 0, 0)
    assert lib.icar_adv_halo_size(C.byref(o)) == expect


def test_var_request(cuda_lib):
    from hicar_b200 import Options, adv_var_request
    opts = Options()
    adv_var_request(opts)
    assert opts.vars_to_advect == [cuda_lib.F_QV, cuda_lib.F_THETA]
    assert {cuda_lib.F_U, cuda_lib.F_V, cuda_lib.F_W, cuda_lib.F_QV} <= opts.vars_to_allocate


def test_footprint_and_validation(cuda_lib):
    lib = cuda_lib.load()
    d = cuda_lib.Desc()
    d.nx, d.ny, d.nz, d.dx, d.n_species = 64, 48, 20, 1000.0, 2
    d.species[0], d.species[1] = cuda_lib.F_QV, cuda_lib.F_QC
    o = cuda_lib.Opts()
    lib.icar_adv_default_opts(C.byref(o))
    b = C.c_int64()
    assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == 0
    assert b.value > 4 * 64 * 48 * 20 * 10
    d.nz = 2
    assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == cuda_lib.BAD_ARG
    assert b"too small" in lib.icar_adv_last_error(None)
    d.nz = 20
    d.species[1] = cuda_lib.F_QV
    assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == cuda_lib.BAD_ARG
    o.advection = 1
    o.h_order = 4
    d.species[1] = cuda_lib.F_QC
    assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == cuda_lib.BAD_ARG


def test_null_handle_is_an_error_not_a_crash(cuda_lib):
    lib = cuda_lib.load()
    assert lib.icar_adv_advect(None, C.c_float(1.0)) == cuda_lib.BAD_ARG
    assert lib.icar_adv_sync(None) == cuda_lib.BAD_ARG
    assert lib.icar_adv_destroy(None) == 0


def test_restart_vars_match_reference_request(cuda_lib):
    """adv_std_var_request (advect.f90:95-107) asks for u, v, w,
    dz_interface and water_vapor as restart variables, for both schemes."""
    from hicar_b200 import Options, kADV_STD, restart_vars
    lib = cuda_lib.load()
    assert restart_vars(Options()) == ["u", "v", "w", "dz_interface", "qv"]
    o = Options()
    o.adv_options.advection = kADV_STD
    assert restart_vars(o) == ["u", "v", "w", "dz_interface", "qv"]
    n = C.c_int32(0)
    assert lib.icar_adv_restart_vars(None, None, C.byref(n)) == 0 and n.value == 5
    ids = (C.c_int32 * 4)()
    n = C.c_int32(4)
    assert lib.icar_adv_restart_vars(None, ids, C.byref(n)) == cuda_lib.BAD_ARG
    assert lib.icar_adv_download(None, 0, None, None) == cuda_lib.BAD_ARG
    assert lib.icar_adv_upload(None, 0, None, None) == cuda_lib.BAD_ARG


def test_c_consumer_compiles_links_and_runs(cuda_lib, tmp_path):
    """The header compiles as strict C99 and a C program linked to the
    library runs its host-only entry points (tests/c_consumer.c), as a
    Fortran shim bound through ISO_C_BINDING would call them."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    so = Path(cuda_lib.LIB_PATH)
    exe = tmp_path / "c_consumer"
    cmd = [gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "c_consumer.c"), "-o", str(exe), str(so), f"-Wl,-rpath,{so.parent}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout, r.stderr)


def test_standard_scheme_needs_an_updated_column_and_row(cuda_lib):
    """The standard scheme updates its..ite x jts..jte, the domain less its
    halo on each side; a domain with no such cell is refused (BAD_ARG)."""
    lib = cuda_lib.load()
    o = cuda_lib.Opts()
    lib.icar_adv_default_opts(C.byref(o))
    o.advection, o.h_order, o.v_order, o.flux_corr = 1, 5, 3, 1
    hs = lib.icar_adv_halo_size(C.byref(o))
    assert hs == 4
    d = cuda_lib.Desc()
    d.nx, d.ny, d.nz, d.dx, d.n_species = 2 * hs + 1, 2 * hs + 1, 3, 1000.0, 1
    d.species[0] = cuda_lib.F_QV
    b = C.c_int64()
    assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == 0
    for nx, ny in [(2 * hs, 2 * hs + 1), (2 * hs + 1, 2 * hs)]:
        d.nx, d.ny = nx, ny
        assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == cuda_lib.BAD_ARG
        assert b"twice the halo" in lib.icar_adv_last_error(None)
    o.advection = 2                                  # MPDATA takes any extent >= 3
    d.nx, d.ny = 3, 3
    assert lib.icar_adv_footprint(C.byref(d), C.byref(o), C.byref(b)) == 0
