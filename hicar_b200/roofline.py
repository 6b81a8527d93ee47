"""HBM roofline bookkeeping for the advection kernels.

Algorithmic bytes of one MPDATA step (the bytes model): every species is
read and written once (8 B per cell-species) and the eight species-
independent fields (u, v, w, density, jacobian, jacobian_u/_v/_w) are read
once per step (32 B per cell), shared by the S species:
    8 + 32/S bytes per cell-species  (10.67 B at S=12, 40 B at S=1).
One advect call (all S species) therefore moves cells * (8*S + 32)
algorithmic bytes.  advection_dz is one value per level and is not counted.

The single-pass kernel (k_mpdata_onepass) reads each species once and
writes it once (8 B per cell-species) and reads seven species-independent
fields once (U_m, V_m, W_m/dz and J*rho through TMA, W_m, dz*J*rho and dz by
plain loads: 28 B per cell):
    8 + 28/S bytes per cell-species  (10.33 B at S=12).

The dominant kernel of the two-kernel form, the fused correction kernel (k_mp_corr),
reads q0 and q1 and writes the new state of every species (12 B per
cell-species) and reads six species-independent fields once (U_m, V_m,
W_m/dz, J*rho, dz*J*rho and dz: 24 B per cell):
    12 + 24/S bytes per cell-species  (14 B at S=12).
"""
from __future__ import annotations

import json
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
FALLBACK_HBM_GBS = 6650.0


def hbm_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def bytes_per_cell_species(S: int) -> float:
    return 8.0 + 32.0 / S


def species_pass(nx: int, ny: int, nz: int, S: int, total_ms: float, passes: int, traffic=None) -> dict:
    """Roofline entry for the advection kernels of one advect call (all S
    species), timed with CUDA events on the launching stream."""
    peak, kind = hbm_peak()
    per_pass = nx * ny * nz * S * bytes_per_cell_species(S)
    if passes <= 0 or total_ms <= 0:
        achieved = None
    else:
        achieved = per_pass / (total_ms / passes / 1e3) / 1e9
    return {
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None, "traffic": traffic,
        "peak_kind": kind, "algorithmic_bytes_per_launch": per_pass,
        "launch_ms": (total_ms / passes) if passes else None,
        "bytes_model": "8 + 32/S B per cell-species; one launch = the kernels of one advect call",
    }


# DRAM bytes (read + write) per cell-species of one k_mp_corr launch, from
# an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of a
# 256x256x40, 12-species launch with tile shape 1 and FCT on.
CORR_DRAM_BYTES_PER_CS = 13.87


def correction_kernel(nx: int, ny: int, nz: int, S: int, total_ms: float, launches: int) -> dict:
    """Roofline entry for the fused correction kernel alone, timed with CUDA
    events around its launches on the launching stream."""
    peak, kind = hbm_peak()
    cells = nx * ny * nz
    per_launch = cells * (12.0 * S + 24.0)
    achieved = per_launch / (total_ms / launches / 1e3) / 1e9 if launches > 0 and total_ms > 0 else None
    traffic = cells * S * CORR_DRAM_BYTES_PER_CS if CORR_DRAM_BYTES_PER_CS else None
    return {
        "kernel": "k_mp_corr (pseudo-velocities + FCT + corrective pass, all species)",
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None, "traffic": traffic,
        "peak_kind": kind, "algorithmic_bytes_per_launch": per_launch,
        "launch_ms": (total_ms / launches) if launches else None,
        "bytes_model": "12 + 24/S B per cell-species; one launch = all species of one advect call",
        "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per cell-species of a "
                           "256x256x40x12 launch, scaled to this launch by cell-species")
        if CORR_DRAM_BYTES_PER_CS else None,
    }


# DRAM bytes (read + write) per cell-species of one k_mpdata_onepass launch
# (fast variant, FCT on), from an ncu capture of the 512x512x40, 12-species
# bench launch: 955.92 MB read + 483.57 MB written for 125.8 M cell-species.
ONEPASS_DRAM_BYTES_PER_CS = (955.918592e6 + 483.570688e6) / (512 * 512 * 40 * 12)


def single_pass_kernel(nx: int, ny: int, nz: int, S: int, total_ms: float, launches: int) -> dict:
    """Roofline entry for the single-pass kernel alone (all S species of one
    advect call per launch), timed with CUDA events around its launches."""
    peak, kind = hbm_peak()
    cells = nx * ny * nz
    per_launch = cells * (8.0 * S + 28.0)
    achieved = per_launch / (total_ms / launches / 1e3) / 1e9 if launches > 0 and total_ms > 0 else None
    return {
        "kernel": "k_mpdata_onepass (donor-cell pass, pseudo-velocities, FCT and corrective pass, all species)",
        "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": (achieved / peak) if achieved else None, "traffic": cells * S * ONEPASS_DRAM_BYTES_PER_CS,
        "peak_kind": kind, "algorithmic_bytes_per_launch": per_launch,
        "launch_ms": (total_ms / launches) if launches else None,
        "bytes_model": "8 + 28/S B per cell-species; one launch = all species of one advect call",
        "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per cell-species of a "
                           "512x512x40x12 launch, scaled to this launch by cell-species"),
    }
