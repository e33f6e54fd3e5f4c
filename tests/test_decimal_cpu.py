"""The device Matrix Market reader's decimal conversion (csrc/decimal.cuh),
compiled for the host, against the C library's strtod -- the conversion that
scanf("%lf") in the reference's reader performs: random doubles printed at
3-40 digits, random digit strings over the whole exponent range, exact
midpoints between neighbouring doubles and strings a hair either side (the
big-integer pass), fixed edge cases; all bit-identical.  No GPU needed."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_decimal_matches_strtod(tmp_path):
    exe = str(tmp_path / "decimal_test")
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "sparseops_b200", "csrc"), "-o", exe,
                    os.path.join(ROOT, "tests", "cpp", "decimal_test.cpp")], check=True)
    r = subprocess.run([exe, "60000"], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
