"""Launch shapes on the GPU: every tile shape and species group gives the
same fields bit for bit (plain and batched), and the autotuner measures
every combination and returns the fastest."""
import numpy as np
import pytest

from hicar_b200 import autotune as A, synth
from hicar_b200.advection import AdvOptions, Domain, Options, adv_init, advect
from hicar_b200.batch import Batch

pytestmark = pytest.mark.gpu


def _run(case, opts, shape, group, steps=3):
    d = Domain.from_case(case)
    adv_init(d, opts)
    d.set_launch_shape(shape, group)
    for _ in range(steps):
        advect(d, opts, case.dt)
    out = {k: d.fetch(k).copy() for k in case.species}
    d.close()
    return out


@pytest.mark.parametrize("fct", [True, False])
def test_every_launch_shape_gives_identical_fields(fct):
    case = synth.config2(seed=7, nx=61, ny=45, nz=11)
    case.species = {k: case.species[k] for k in ("qv", "qc", "qr", "nr", "theta")}
    opts = Options(adv_options=AdvOptions(MPDATA_FCT=fct))
    ref = _run(case, opts, 1, 0)
    for shape in range(len(A.TILE_ROWS)):
        for group in (0, 1, 2, 3):
            got = _run(case, opts, shape, group)
            for k in ref:
                assert np.array_equal(got[k], ref[k]), (shape, group, k)


def test_batch_species_group_and_shape_give_identical_fields():
    cases = [synth.ensemble_member(100 + i, nx, ny, nz) for i, (nx, ny, nz) in
             enumerate([(40, 33, 9), (70, 29, 12), (33, 61, 7)])]
    opts = Options()
    ref = []
    for c in cases:
        ref.append(_run(c, opts, 1, 0, steps=2))
    for shape, group in ((0, 5), (3, 1), (2, 0)):
        b = Batch(0)
        doms = []
        for c in cases:
            d = Domain.from_case(c)
            adv_init(d, opts)
            b.add(d, c.dt)
            doms.append(d)
        b.set_tile_shape(shape)
        b.set_species_group(group)
        for _ in range(2):
            b.step()
        b.sync()
        for c, d, r in zip(cases, doms, ref):
            b.remove(d)
            for k in c.species:
                assert np.array_equal(d.fetch(k), r[k]), (shape, group, k)
            d.close()
        b.close()


def test_tune_domain_measures_every_combination(tmp_path, monkeypatch):
    monkeypatch.setenv("HICAR_B200_AUTOTUNE_CACHE", str(tmp_path / "t.json"))
    monkeypatch.setattr(A, "_mem_cache", {})
    c = A.tune_domain(96, 80, 20, 12, fct=True, reps=1)
    assert len(c.measured) == len(A.TILE_ROWS) * len(A.species_groups(12))
    assert c.ms_per_advect == min(c.measured.values()) > 0
    again = A.tune_domain(96, 80, 20, 12, fct=True, reps=1)      # from the cache
    assert (again.tile_shape, again.species_group) == (c.tile_shape, c.species_group)
    costs = A.shape_costs(True, calib=(96, 80, 20, 12), reps=1)
    assert set(costs) == set(range(len(A.TILE_ROWS))) and all(v > 0 for v in costs.values())
