"""The GPU path against the golden fixtures tests/golden/*.npz, which were
generated from the reference's own C (src/c/so3_core.c compiled unmodified,
tests/golden/gen_golden.py): inverse of the stored flmn against the stored
samples, forward of the stored samples against the stored coefficients.
This pins the GPU to the reference directly, not through the oracle's
restatement.  Tolerance: 1e-12 normwise relative error."""
import glob
import json
import os

import numpy as np
import pytest

import so3_b200 as so3
from tests.helpers import params, rel_err, rel_err_elem

pytestmark = pytest.mark.gpu

TOL = 1e-12
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = sorted(glob.glob(os.path.join(HERE, "case*.npz")))


def test_fixtures_present():
    assert len(FILES) == 7


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f) for f in FILES])
def test_gpu_matches_reference_fixture(path):
    d = np.load(path)
    c = json.loads(str(d["config"]))
    p = params(c["L"], c["N"], L0=c["L0"], reality=c["reality"], sampling=c["sampling"], order=c["order"],
               storage=c["storage"], mode=c["mode"], method=c["method"])
    f = so3.inverse(d["flmn"], p)
    assert rel_err(f, d["f"]) < TOL
    assert rel_err_elem(f, d["f"]) < 1e-9
    back = so3.forward(d["f"], p)
    assert rel_err(back, d["flmn_back"]) < TOL
    assert rel_err_elem(back, d["flmn_back"]) < 1e-9
