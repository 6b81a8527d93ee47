"""The constant-divisor quotients the standard-scheme kernels use for the
/12 and /60 of flux3 (hicar_b200/csrc/const_div.h): the constants against
exact rational arithmetic, and the quotient against IEEE division for every
non-negative float (exhaustive, a few seconds on a few cores)."""
import re
import shutil
import subprocess
from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
HDR = HERE.parent / "hicar_b200" / "csrc" / "const_div.h"


def header_constants() -> dict:
    vals = {}
    for name, lit in re.findall(r"#define (ICAR_\w+) (-?0x[0-9a-fp.+-]+)", HDR.read_text()):
        vals[name] = float.fromhex(lit)
    return vals


@pytest.mark.parametrize("d", [12, 60])
def test_constant_is_the_double_nearest_the_reciprocal(d):
    r = header_constants()[f"ICAR_RCP{d}_D"]
    exact = Fraction(1, d)
    below, above = np.nextafter(r, -np.inf), np.nextafter(r, np.inf)
    assert abs(Fraction(r) - exact) < abs(Fraction(float(below)) - exact)
    assert abs(Fraction(r) - exact) < abs(Fraction(float(above)) - exact)


def test_quotient_is_correctly_rounded_for_every_float(tmp_path):
    cc = shutil.which("cc") or shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = tmp_path / "const_div_check"
    subprocess.run([cc, "-O2", "-ffp-contract=off", "-fopenmp", str(HERE / "const_div_check.c"), "-o", str(exe)],
                   check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=900)
    print(res.stdout)
    assert res.returncode == 0, res.stdout
    assert res.stdout.count("mismatches=0") == 2
