"""Roofline bookkeeping of the bench line, on the CPU: the bytes models, the
peak taken from the measured peaks file, and achieved = algorithmic bytes
per launch / mean launch time."""
import json

import pytest

from hicar_b200 import roofline as RL


def test_bytes_models():
    assert RL.bytes_per_cell_species(12) == pytest.approx(8 + 32 / 12)
    assert RL.bytes_per_cell_species(1) == 40.0


def test_peak_is_the_measured_copy_bandwidth():
    peak, kind = RL.hbm_peak()
    measured = json.loads((RL.ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
    assert kind == "measured" and peak == measured


def test_advect_call_entry():
    nx, ny, nz, S = 512, 512, 40, 12
    r = RL.species_pass(nx, ny, nz, S, total_ms=70.0, passes=10)
    per = nx * ny * nz * (8 * S + 32)
    assert r["algorithmic_bytes_per_launch"] == pytest.approx(per)
    assert r["launch_ms"] == pytest.approx(7.0)
    assert r["achieved"] == pytest.approx(per / 7e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert RL.species_pass(nx, ny, nz, S, 0.0, 0)["achieved"] is None


def test_correction_kernel_entry():
    nx, ny, nz, S = 512, 512, 40, 12
    r = RL.correction_kernel(nx, ny, nz, S, total_ms=62.7, launches=10)
    per = nx * ny * nz * (12 * S + 24)
    assert r["algorithmic_bytes_per_launch"] == pytest.approx(per)
    assert r["achieved"] == pytest.approx(per / 6.27e-3 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    # the ncu traffic per cell-species, scaled to the launch; close to the model
    assert r["traffic"] == pytest.approx(nx * ny * nz * S * RL.CORR_DRAM_BYTES_PER_CS)
    assert abs(r["traffic"] / per - 1) < 0.02
