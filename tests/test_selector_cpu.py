"""The learned format selector's committed model (csrc/selector_tree.h,
fitted by sparseops_b200/selector.py on the measurements in
sparseops_b200/selector_data.json): the library's choice from stored
features (spops_select_format_from_features, host only) equals the tree
walked here, for every measured matrix, and the held-out figures written in
the header are what the committed data and tree give."""
import json
import os
import re

import numpy as np
import pytest

from sparseops_b200 import selector
from sparseops_b200.formats import select_format_from_features

DATA = os.path.join(os.path.dirname(selector.__file__), "selector_data.json")


@pytest.fixture(scope="module")
def data():
    if not os.path.exists(DATA):
        pytest.skip("no selector measurements committed")
    with open(DATA) as fh:
        return json.load(fh)["rows"]


def test_library_choice_equals_tree(data):
    code_name = {v[0]: k for k, v in selector.CANDIDATES.items()}
    for r in data:
        f = r["features"]
        want = code_name[selector.predict_table(selector.derived(f))]
        if want == "dia" and not selector.dia_allowed(f):
            want = "csr"  # the library never returns DIA where its diagonals do not allow it
        got = select_format_from_features(f)
        assert got["format"] == want, r["name"]
        if want in ("sell_c_sigma", "sell_c_R"):
            assert got["params"]["chunk"] == 32 and got["params"]["layout"] == 1


def test_header_figures_match_the_data(data):
    with open(selector.TREE_HEADER) as fh:
        text = fh.read()
    m = re.search(r"on the\s+(\d+) held-out ones it picks the\s*//\s*timed choice for (\d+)", text)
    if m is None:
        pytest.skip("tree not fitted")
    held = [r for k, r in enumerate(data) if k % 3 == 2]
    code_name = {v[0]: k for k, v in selector.CANDIDATES.items()}
    agree = sum(code_name[selector.predict_table(selector.derived(r["features"]))] == min(r["ms"], key=r["ms"].get)
                for r in held)
    assert int(m.group(1)) == len(held) and int(m.group(2)) == agree
