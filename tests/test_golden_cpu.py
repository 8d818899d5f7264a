"""The oracle against the committed golden fixtures (tests/golden, made by
tests/golden/make_golden.py): FormH and FormJ bit for bit (CSR SHA-256,
NumH, numzero, Hmin), Dinit's term list, and the Davidson levels."""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from conftest import get_system, oracle_h

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _sha(rowptr, col, val):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, np.int64).tobytes())
    h.update(np.ascontiguousarray(col, np.int32).tobytes())
    h.update(np.ascontiguousarray(val, np.float64).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", ["tiny", "cfg1", "small3"])
def test_oracle_matches_golden(name):
    g = np.load(os.path.join(GOLD, f"{name}.npz"))
    s = get_system(name)
    (rp, col, val, nz, hmin, pairs), (jr, jc, jv) = oracle_h(name)
    assert rp[-1] == g["numh"] and nz == g["numzero"] and hmin == g["hmin"]
    assert _sha(rp, col, val) == str(g["h_sha"])
    assert _sha(jr, jc, jv) == str(g["j_sha"])
    if name == "tiny":
        assert np.array_equal(rp, g["h_rowptr"]) and np.array_equal(col, g["h_col"])
        assert np.array_equal(val.view(np.int64), g["h_val"].view(np.int64))
    assert O.j_terms(s.basis, s.configs, s.mj) == g["jterms"].tolist()
    p = dict(s.params)
    if int(g["n_it"]) > 0:
        p.update(N_it=int(g["n_it"]), admix_crit=0.0)
    res = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    assert res["iterations"] == int(g["iterations"])
    assert np.max(np.abs(res["Tk"] - g["tk"])) <= 1e-10
    assert np.allclose(res["Tj"], g["tj"], atol=1e-8)
