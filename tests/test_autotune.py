"""Autotuner host logic (no GPU): tile geometry, candidate groups, the
batch-shape model and the result cache."""
import json

import pytest

from hicar_b200 import autotune as A


def test_tiles_match_the_kernel_tiling():
    # 28-column tiles starting at output column -2; the last must reach nx-2
    for nx in (3, 27, 28, 29, 55, 56, 57, 512):
        tx = nx // 28 + 1
        assert 28 * (tx - 1) - 2 <= nx - 2 <= 28 * tx - 2 + 27
    assert A.tiles(512, 512, 16) == (512 // 28 + 1) * ((510 + 15) // 16)
    assert A.tiles(64, 10, 8) == 3 * 1


def test_species_groups_are_distinct_and_cover():
    assert A.species_groups(12) == [0, 6, 4, 3, 2]
    assert A.species_groups(1) == [0]
    for s in range(1, 33):
        gs = A.species_groups(s)
        assert gs[0] == 0 and len(set(gs)) == len(gs)
        assert all(1 <= g < s for g in gs[1:])


def test_batch_shape_model_prefers_less_waste():
    # cost per tile-level = rows + a fixed halo share: taller tiles are cheaper
    # per row unless their last tile is mostly empty
    costs = {s: r + 4.0 for s, r in enumerate(A.TILE_ROWS)}
    assert A.choose_batch_shape([(64, 10, 20, 12)], costs) == 0       # 8 interior rows: one 8-row tile
    assert A.choose_batch_shape([(64, 33, 20, 12)], costs) == 3       # 31 rows: one 31-row tile, no waste
    assert A.choose_batch_shape([(64, 10, 20, 12)] * 3 + [(64, 33, 20, 12)], costs) == 0
    # a shape that is cheaper per row wins when waste is equal
    costs2 = {0: 8.0, 1: 14.0, 2: 24.0, 3: 32.0}
    assert A.choose_batch_shape([(300, 258, 40, 12)], costs2) == 1


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("HICAR_B200_AUTOTUNE_CACHE", str(path))
    monkeypatch.setattr(A, "_mem_cache", {})
    A._store("domain:X:1x2x3:S4:fct1", {"tile_shape": 2, "species_group": 0, "ms_per_advect": 1.5, "measured": {}})
    assert json.loads(path.read_text())["domain:X:1x2x3:S4:fct1"]["tile_shape"] == 2
    monkeypatch.setattr(A, "_mem_cache", {})
    assert A._load_cache()["domain:X:1x2x3:S4:fct1"]["ms_per_advect"] == 1.5
    c = A.Choice(**A._load_cache()["domain:X:1x2x3:S4:fct1"])
    assert c.rows == 24
