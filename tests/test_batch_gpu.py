"""Batched form: every member advanced inside a batch matches the same
domain advanced alone and the CPU oracle, cell for cell."""
import numpy as np
import pytest

from hicar_b200 import synth
from hicar_b200.advection import Domain, Options, AdvOptions, adv_init, step
from hicar_b200.batch import Batch

pytestmark = pytest.mark.gpu


def make_members(shapes, seed0=0, forcing_every=2):
    cases, doms = [], []
    for n, (nx, ny, nz) in enumerate(shapes):
        c = synth.ensemble_member(seed0 + n, nx, ny, nz)
        c.species = {k: c.species[k] for k in ("qv", "qc", "nr", "theta")}
        cases.append(c)
    return cases


def run_alone(case, nsteps, forcing=None, opts=None):
    opts = opts or Options()
    d = Domain.from_case(case)
    if forcing is not None:
        for k in case.species:
            d.set_forcing(k, forcing[k][0], forcing[k][1])
    adv_init(d, opts)
    for _ in range(nsteps):
        step(d, opts, case.dt)
    out = {k: d.fetch(k).copy() for k in case.species}
    d.close()
    return out


def forcing_for(case, seed):
    rng = np.random.default_rng(seed)
    return {k: ((v * 1.05).astype(np.float32), (rng.standard_normal(v.shape) * 1e-9).astype(np.float32))
            for k, v in case.species.items()}


@pytest.mark.parametrize("shape_id", [0, 1, 2, 3])
def test_batch_matches_alone_and_oracle(oracle_lib, shape_id):
    shapes = [(40, 36, 12), (67, 30, 20), (29, 45, 9), (100, 64, 7), (33, 33, 25)]
    cases = make_members(shapes, seed0=10)
    forc = [forcing_for(c, i) if i % 2 == 0 else None for i, c in enumerate(cases)]
    b = Batch()
    b.set_tile_shape(shape_id)
    doms = []
    for c, f in zip(cases, forc):
        d = Domain.from_case(c)
        if f is not None:
            for k in c.species:
                d.set_forcing(k, f[k][0], f[k][1])
        adv_init(d, Options())
        b.add(d, c.dt)
        doms.append(d)
    nsteps = 5
    for _ in range(nsteps):
        b.step()
    b.sync()
    O = oracle_lib
    for c, d, f in zip(cases, doms, forc):
        got = {k: d.fetch(k).copy() for k in c.species}
        alone = run_alone(c, nsteps, forcing=f)
        for k in c.species:
            assert np.array_equal(got[k], alone[k]), (c.nx, c.ny, c.nz, k)
        if f is None:
            ref = O.run_steps(c, O.make_opts(), c.dt, nsteps)
        else:
            flt = O.init_relax_filters(c.nx, c.ny, 2)
            ref = O.run_steps(c, O.make_opts(), c.dt, nsteps, forcing=f, filter2d=flt)
        for k in c.species:
            assert np.array_equal(got[k], ref[k]), ("oracle", c.nx, c.ny, c.nz, k)
    b.close()
    for d in doms:
        d.close()


def test_batch_membership_changes_and_per_member_dt(oracle_lib):
    """Members join and leave between steps; each keeps its own dt; a
    member's result is the same alone and in the mix."""
    shapes = [(50, 40, 10), (30, 60, 14), (45, 45, 8)]
    cases = make_members(shapes, seed0=40)
    cases[1].dt = 10.0
    b = Batch()
    doms = [Domain.from_case(c) for c in cases]
    for d in doms:
        adv_init(d, Options())
    b.add(doms[0], cases[0].dt)
    b.add(doms[1], cases[1].dt)
    b.step()
    b.step()
    b.add(doms[2], cases[2].dt)      # joins after two steps
    b.step()
    b.remove(doms[0])                # leaves after three steps
    b.step()
    b.step()
    b.sync()
    O = oracle_lib
    expect_steps = [3, 5, 3]
    for c, d, n in zip(cases, doms, expect_steps):
        ref = O.run_steps(c, O.make_opts(), c.dt, n)
        for k in c.species:
            assert np.array_equal(d.fetch(k), ref[k]), (c.nx, k, n)
    # a removed member can be stepped on its own again
    step(doms[0], Options(), cases[0].dt)
    ref = O.run_steps(cases[0], O.make_opts(), cases[0].dt, 4)
    assert np.array_equal(doms[0].fetch("qv"), ref["qv"])
    b.close()
    for d in doms:
        d.close()


def test_batch_rejects_ineligible_members():
    c = make_members([(30, 30, 6)])[0]
    d = Domain.from_case(c)
    adv_init(d, Options(adv_options=AdvOptions(mpdata_order=3)))
    b = Batch()
    with pytest.raises(Exception):
        b.add(d, c.dt)
    b.close()
    d.close()


@pytest.mark.parametrize("path", [2, 3])
def test_batch_single_pass_kernel(oracle_lib, path):
    """The batched step on the single-pass kernel (a persistent launch over
    every member's 56 x 26 tiles): bit-identical to the oracle and to each
    member stepped alone with the bit-exact arithmetic (path 2); within the
    fast variant's tolerance with fast arithmetic (path 3), and still
    identical to the same member stepped alone on the same kernel."""
    shapes = [(40, 36, 12), (67, 30, 20), (129, 61, 9), (100, 64, 7), (33, 33, 25)]
    cases = make_members(shapes, seed0=60)
    forc = [forcing_for(c, i) if i % 2 == 0 else None for i, c in enumerate(cases)]
    b = Batch()
    b.set_path(path)
    doms = []
    for c, f in zip(cases, forc):
        d = Domain.from_case(c)
        if f is not None:
            for k in c.species:
                d.set_forcing(k, f[k][0], f[k][1])
        adv_init(d, Options())
        b.add(d, c.dt)
        doms.append(d)
    nsteps = 5
    for _ in range(nsteps):
        b.step()
    b.sync()
    O = oracle_lib
    for c, d, f in zip(cases, doms, forc):
        got = {k: d.fetch(k).copy() for k in c.species}
        # the same member alone on the same kernel
        a = Domain.from_case(c)
        if f is not None:
            for k in c.species:
                a.set_forcing(k, f[k][0], f[k][1])
        adv_init(a, Options())
        a.set_path(path)
        for _ in range(nsteps):
            step(a, Options(), c.dt)
        alone = {k: a.fetch(k).copy() for k in c.species}
        a.close()
        for k in c.species:
            assert np.array_equal(got[k], alone[k]), ("alone", path, c.nx, c.ny, c.nz, k)
        if f is None:
            ref = O.run_steps(c, O.make_opts(), c.dt, nsteps)
        else:
            flt = O.init_relax_filters(c.nx, c.ny, 2)
            ref = O.run_steps(c, O.make_opts(), c.dt, nsteps, forcing=f, filter2d=flt)
        for k in c.species:
            if path == 2:
                assert np.array_equal(got[k], ref[k]), ("oracle", c.nx, c.ny, c.nz, k)
            else:
                scale = float(np.abs(ref[k]).max()) or 1.0
                assert float(np.abs(got[k].astype(np.float64) - ref[k]).max()) / scale <= 1e-5, (c.nx, k)
    b.close()
    for d in doms:
        d.close()
