"""The engine's portable exp and sincos (host and device, photonoxide_b200/csrc/portable.h) give
the bits of the oracle's restatement of the reference's (oracle/refmath.h), which the canary hash
pins to photonoxide's own: so source waveforms and transform phases are the reference's bits."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_portable_math_matches_the_oracle_bitwise():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "check")
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                        "-I", os.path.join(ROOT, "photonoxide_b200", "csrc"),
                        "-I", os.path.join(ROOT, "oracle"),
                        os.path.join(ROOT, "tests", "portable_check.cpp"), "-o", exe], check=True)
        bad, total = map(int, subprocess.run([exe], check=True, capture_output=True,
                                             text=True).stdout.split())
    assert total > 0 and bad == 0, f"{bad} of {total} differ"
