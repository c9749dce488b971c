"""The reference's own bit canary for its portable maths (src/portable/tests.rs:345-556): the hash
of each function's bits over a fixed grid of 620 arguments, taken on Windows x86-64 with libm
0.2.16 and the same on every IEEE system. The engine's portable maths
(photonoxide_b200/csrc/portable.h: the source waveforms' exp and sincos, the CPML grading's ln and
pow) and the oracle's restatement (oracle/refmath.h) must both give the reference's hashes: that
pins them to photonoxide's bits over the whole grid, special values and subnormals included.
(sincos takes the C library's sin and cos beyond 2^20 pi/2, which the FDTD path never reaches; on
this grid's three such arguments, 1e22 and the largest doubles, those agree too.)"""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# GRID_HASHES of src/portable/tests.rs:514-556, the functions the FDTD path calls
REFERENCE = {
    "exp": 0x413fbc04627e9685,
    "ln": 0x0bf1e9d3216efc53,
    "sin_cos.0": 0xda525217fa01fbf0,
    "sin_cos.1": 0xda5c8775269b6b93,
    "powf": 0x9133a6eca7e0bb06,
}


def test_grid_hashes_are_the_references():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "grid")
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off",
                        "-I", os.path.join(ROOT, "photonoxide_b200", "csrc"),
                        "-I", os.path.join(ROOT, "oracle"),
                        os.path.join(ROOT, "tests", "portable_grid.cpp"), "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        who, name, value = line.split()
        got[(who, name)] = int(value, 16)
    for who in ("engine", "oracle"):
        for name, want in REFERENCE.items():
            assert got[(who, name)] == want, f"{who} {name}: {got[(who, name)]:#018x} != {want:#018x}"
