"""Smallest domains the boundary accepts and ragged ones just above them,
where one tile covers the whole domain and most cells lie in the boundary
ring: every extent >= 3 for MPDATA; for the standard scheme nx, ny >=
2*halo + 1, so that one column and one row are updated.  Fused and staged
kernels against the FP32 oracle, cell for cell, for MPDATA (order 2, FCT),
the HICAR default standard scheme (RK3, h_order 5, v_order 3, WRF
correction) and a third-order standard scheme."""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import Domain, adv_init, advect

from tests.test_parity_gpu import assert_exact, options_from

pytestmark = pytest.mark.gpu

MPDATA_SHAPES = [(3, 3, 3), (4, 3, 5), (3, 7, 4), (7, 4, 3), (5, 6, 3), (9, 8, 3)]
STD_SCHEMES = {
    "std_h5v3_wrf_rk3": dict(advection=1, h_order=5, v_order=3, flux_corr=1, rk3=1),
    "std_h3v3": dict(advection=1, h_order=3, v_order=3),
}


def _std_shapes():
    """Per standard scheme: the smallest accepted extents m = 2*halo + 1 (one
    updated column and row) and ragged ones just above."""
    from oracle import oracle as O
    out = []
    for name, kw in STD_SCHEMES.items():
        m = 2 * O.halo_size(1, kw["h_order"], kw["v_order"], kw.get("flux_corr", 0)) + 1
        for shape in [(m, m, 3), (m + 1, m, 5), (m, m + 3, 4), (m + 2, m + 1, 3)]:
            out.append((name, shape))
    return out


CASES = [("mpdata", s) for s in MPDATA_SHAPES] + _std_shapes()


def _run(oracle_lib, scheme_kw, shape):
    O = oracle_lib
    nx, ny, nz = shape
    case = synth.config2(seed=7, nx=nx, ny=ny, nz=nz)
    o = O.make_opts(**scheme_kw)
    ref = O.run_steps(case, o, case.dt, 3)
    for staged in (False, True):
        d = Domain.from_case(case)
        adv_init(d, options_from(o))
        if staged:
            d.use_staged_kernels(True)
        for _ in range(3):
            advect(d, options_from(o), case.dt)
        out = {k: d.fetch(k).copy() for k in case.species}
        d.close()
        assert all(np.isfinite(v).all() for v in out.values())
        assert_exact(out, ref, label=f"{scheme_kw} {shape} staged={staged} ")


@pytest.mark.parametrize("scheme,shape", CASES, ids=[f"{n}-{'x'.join(map(str, s))}" for n, s in CASES])
def test_tiny_and_ragged_domains(oracle_lib, scheme, shape):
    _run(oracle_lib, STD_SCHEMES.get(scheme, {}), shape)
