"""Differential test of the two CPU restatements of MPDATA (no GPU).

The C oracle (oracle/icar_adv_oracle.c) and the CUDA kernels were written
from one reading of src/physics/adv_mpdata.f90.  oracle/mpdata_numpy.py is a
second, independent transliteration of the same Fortran array statements
(numpy, slice for slice, no shared code).  No Fortran compiler exists on
either machine, so agreement of the two restatements is the available guard
against a shared misreading.  Both round every operation to single
precision in the Fortran order, so they must agree bit for bit, stage by
stage and over whole steps.
"""
import numpy as np
import pytest

from hicar_b200 import synth
from oracle import mpdata_numpy as M


def _small(seed, nx=13, ny=11, nz=7, species=("qv", "qc", "nr", "theta")):
    c = synth.config2(seed=seed, nx=nx, ny=ny, nz=nz)
    c.species = {k: c.species[k] for k in species}
    return c


def _F(a, lb=(1, 1, 1)):
    return M.F(np.ascontiguousarray(a, dtype=np.float32).copy(), lb)


def _same(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    nd = int((a != b).sum())
    assert nd == 0, f"{what}: {nd} of {a.size} values differ (max |d| {np.abs(a.astype(float) - b).max():.3e})"


@pytest.mark.parametrize("advect_density", [0, 1])
def test_compute_wind_matches(oracle_lib, advect_density):
    O = oracle_lib
    c = _small(3)
    Um, Vm, Wm = O.mpdata_compute_wind(c, c.dt, advect_density)
    b = M.Bounds(c.nx, c.ny, c.nz)
    um, vm, wm = M.mpdata_compute_wind(b, _F(c.u), _F(c.v), _F(c.w), _F(c.density), _F(c.jacobian_u),
                                       _F(c.jacobian_v), _F(c.jacobian_w), c.dx, c.dt, bool(advect_density))
    _same(um.a, Um[:, :, 1:c.nx], "U_m")
    _same(vm.a, Vm[1:c.ny], "V_m")
    _same(wm.a, Wm, "W_m")


def test_stages_match(oracle_lib):
    """upwind_advection, mpdata_fluxes and flux_limiter one by one on the
    same inputs (the stage entry points of the C oracle)."""
    O = oracle_lib
    c = _small(5, nx=15, ny=12, nz=8)
    b = M.Bounds(c.nx, c.ny, c.nz)
    Um, Vm, Wm = O.mpdata_compute_wind(c, c.dt, 0)
    um, vm, wm = M.mpdata_compute_wind(b, _F(c.u), _F(c.v), _F(c.w), _F(c.density), _F(c.jacobian_u),
                                       _F(c.jacobian_v), _F(c.jacobian_w), c.dx, c.dt, False)
    rho, jac, dz = (np.ascontiguousarray(getattr(c, k), np.float32) for k in ("density", "jacobian", "advection_dz"))
    for name, q in c.species.items():
        q = np.ascontiguousarray(q, np.float32)
        # pass 1
        q2_c = O.upwind_advection(q, Um, Vm, Wm, rho, dz, jac)
        q2_n = M.F(np.zeros_like(q))
        M.upwind_advection(b, _F(q), um, vm, wm, _F(rho), q2_n, _F(dz), _F(jac))
        _same(q2_n.a, q2_c, f"{name} upwind_advection")
        # pseudo-velocities from q2 with W_m/dz and G = J*rho
        wdz = (Wm / dz).astype(np.float32)
        G = (jac * rho).astype(np.float32)
        u2_c, v2_c, w2_c = O.mpdata_fluxes(q2_c, Um, Vm, wdz, G)
        u2 = M.F(np.zeros((c.ny, c.nz, c.nx - 1), np.float32), (2, 1, 1))
        v2 = M.F(np.zeros((c.ny - 1, c.nz, c.nx), np.float32), (1, 1, 2))
        w2 = M.F(np.zeros((c.ny, c.nz, c.nx), np.float32))
        M.mpdata_fluxes(b, q2_n, um, vm, M.F(wm.a / dz), u2, v2, w2, M.F(G))
        _same(u2.a, u2_c[:, :, 1:c.nx], f"{name} u2")
        _same(v2.a, v2_c[1:c.ny], f"{name} v2")
        _same(w2.a, w2_c, f"{name} w2")
        # FCT on the scaled pseudo-velocities
        for a in (u2_c, v2_c):
            a *= np.float32(0.5)
        w2_c[...] = w2_c * np.float32(0.5) * dz
        u2.a[...] = u2.a * np.float32(0.5)
        v2.a[...] = v2.a * np.float32(0.5)
        w2.a[...] = w2.a * np.float32(0.5) * dz
        O.flux_limiter(q, q2_c, u2_c, v2_c, w2_c)
        M.flux_limiter(b, _F(q), q2_n, u2, v2, w2)
        _same(u2.a, u2_c[:, :, 1:c.nx], f"{name} limited u2")
        _same(v2.a, v2_c[1:c.ny], f"{name} limited v2")
        _same(w2.a, w2_c, f"{name} limited w2")


@pytest.mark.parametrize("order,fct,density", [(2, True, 0), (2, False, 0), (1, True, 0), (3, True, 0),
                                               (2, True, 1)])
def test_whole_steps_match(oracle_lib, order, fct, density):
    """advect() over three steps, every switch of mpdata_advect3d."""
    O = oracle_lib
    c = _small(7 + order, nx=14, ny=12, nz=9)
    opts = O.make_opts(mpdata_order=order, mpdata_fct=int(fct), advect_density=density)
    ref = c.copy()
    got = c.copy()
    for n in range(3):
        ref.species = O.advect(ref, opts, ref.dt)
        got.species = M.advect(got, got.dt, mpdata_order=order, mpdata_fct=fct, advect_density=bool(density))
        for k in ref.species:
            _same(got.species[k], ref.species[k], f"step {n + 1} {k} order={order} fct={fct} density={density}")


def test_config1_shape_matches(oracle_lib):
    """A config-1 style domain (ridge, one tracer) at reduced size, two steps."""
    O = oracle_lib
    c = synth.config1(seed=2, nx=24, ny=20, nz=10)
    ref = O.run_steps(c, O.make_opts(), c.dt, 2)
    got = c.copy()
    for _ in range(2):
        got.species = M.advect(got, got.dt)
    _same(got.species["qv"], ref["qv"], "config1 qv")
