"""The C++ drop-in header (include/spops_b200/SpOps.h): a caller of the
reference's SpOps.h API compiles against it and links the library.

CPU: the test program (tests/cpp/shim_test.cpp, every format, conversion,
delete_host_matrix and the LeSpGEMM preprocessing calls) compiles with
-Wall -Wextra -Werror and links.  GPU: it runs and checks every SpMV against
a plain CPU loop (1e-12 FP64, 1e-5 FP32) and the conversions' layouts."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "sparseops_b200")


def _build(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("no g++")
    exe = str(tmp_path / "shim_test")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include", "spops_b200"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "shim_test.cpp"), "-L", LIBDIR, "-lsparseops_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_header_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_header_program_runs(tmp_path, cuda):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "shim OK" in r.stdout, r.stdout[-4000:] + r.stderr[-2000:]
