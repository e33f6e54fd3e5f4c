"""The learned format selector on the device (spops_select_format mode 2):
its choice for matrices outside the training corpus equals the choice from
the same features on the host, and SpOps_auto in that format gives the
oracle's y (componentwise 1e-12)."""
import math

import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu


def _cases():
    yield "powerlaw", synth.powerlaw(200000, mu=math.log(9.0), sigma=1.0, seed=99)
    yield "laplacian", synth.laplacian_2d(300)
    yield "banded", synth.banded_random(150000, 12.0, 32, seed=77)


@pytest.mark.parametrize("name", ["powerlaw", "laplacian", "banded"])
def test_learned_choice_runs_and_matches_host(cuda, orc, name):
    import torch
    from sparseops_b200 import CSR_Matrix, SpOps_auto, matrix_features, select_format
    from sparseops_b200.formats import select_format_from_features
    rp, ci, v = next(c for n, c in _cases() if n == name)
    n = len(rp) - 1
    d = torch.device("cuda")
    A = CSR_Matrix(n, n, torch.from_numpy(rp).to(d), torch.from_numpy(ci).to(d), torch.from_numpy(v).to(d))
    choice = select_format(A, learned=True)
    assert choice["format"] == select_format_from_features(matrix_features(A))["format"]
    x = synth.uniform(n, 3)
    y = torch.zeros(n, dtype=torch.float64, device=d)
    SpOps_auto(1.0, A, torch.from_numpy(x).to(d), 0.0, y, learned=True)
    assert A._auto[1]["format"] == choice["format"]
    torch.cuda.synchronize()
    ref = orc.spmv_csr(rp, ci, v, x)
    den = np.maximum(orc.absdot(rp, ci, v, x), 1e-300)
    assert (np.abs(y.cpu().numpy() - ref) / den).max() <= 1e-12
