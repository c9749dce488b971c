"""The slabs' d/h in f32 by the product form (div_by_step) gives division's bits: checked here on
the host for common grid steps over a strided sample of all floats and every tiny one (where the
remainder underflows and the form must hand over to division). The engine itself checks every
finite float on the device for each grid step it is given before using the form."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def check_program():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "check")
        subprocess.run(["g++", "-O2", "-std=c++17", "-mfma", "-ffp-contract=off",
                        "-I", "/usr/local/cuda/include",
                        "-I", os.path.join(ROOT, "photonoxide_b200", "csrc"),
                        os.path.join(ROOT, "tests", "division_check.cpp"), "-o", exe], check=True)
        yield exe


@pytest.mark.parametrize("h", ["0.02", "0.05", "0.01", "0.04", "0.03", "0.013"])
def test_product_form_gives_division_bits(check_program, h):
    bad, total = map(int, subprocess.run([check_program, h, "251"], check=True, capture_output=True,
                                         text=True).stdout.split())
    assert total > 100_000_000 and bad == 0, f"{bad} of {total} differ"
