"""The C ABI library loads on a machine without a GPU and exports every entry
point the public header declares; the ctypes table covers all of them.  Also
checks the status codes and refusals that need no device."""
import ctypes as C
import os
import re

import pytest

from sparseops_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sparseops_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:spops_status_t|const char\s*\*|int)\s+(spops_\w+)\s*\(", src, flags=re.M)
    assert len(names) > 40
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing


def test_ctypes_table_matches_header():
    declared = set(_declared())
    bound = set(_lib.exported_symbols())
    assert declared == bound, (declared - bound, bound - declared)


def test_abi_version_and_status_strings():
    L = _lib.lib()
    assert L.spops_abi_version() >= 1
    for s in range(0, 7):
        assert L.spops_status_string(s)


def test_null_arguments_are_refused_without_a_device():
    """Argument checks run before any CUDA call."""
    L = _lib.lib()
    assert L.spops_matrix_info(None, None) == 1  # SPOPS_ERR_INVALID
    assert L.spops_destroy(None) in (0, 1)
    assert L.spops_matrix_destroy(None) == 0
    assert L.spops_pairs_destroy(None) == 0
    assert L.spops_batch_destroy(None) == 0
    with pytest.raises(_lib.SpOpsError) as e:
        _lib.call("spops_csr_spmv_noalloc", _lib.i64(-1), _lib.i64(1), _lib.i64(0), None, None, None, C.c_int(0),
                  C.c_int(1), _lib.dbl(1.0), None, _lib.dbl(0.0), None, None)
    assert e.value.status == 1
