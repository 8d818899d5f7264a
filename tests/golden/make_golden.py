"""Regenerate the golden fixtures of this directory.

The reference (Fortran pconf) cannot be built or run here, so these
fixtures are not its outputs: they record the oracle's results on the seeded
synthetic systems (the oracle restates the reference's FormH/Hmltn/Gint and
Diag4), so that the oracle, the host enumeration and the CUDA path are held
to the same numbers from one version to the next.

    python tests/golden/make_golden.py      # rewrites tests/golden/*.npz

Each fixture holds, for one system: NumH, numzero and Hmin of FormH, the
SHA-256 of its CSR (rowptr int64, 1-based col int32, val float64, in that
order), the J^2 CSR's SHA-256, Dinit's term list Jt, and the Davidson levels
(Tk, Tj) of the system's default parameters (Kv = 4, admix_crit 1e-6) after
the iterations stated in the file.  The tiny system also keeps its full H
CSR.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from pci_b200 import system as S  # noqa: E402

# (system, Davidson iterations recorded; None = run to convergence)
SYSTEMS = [("tiny", None), ("cfg1", None), ("small3", 25)]


def csr_sha(rowptr, col, val):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, np.int64).tobytes())
    h.update(np.ascontiguousarray(col, np.int32).tobytes())
    h.update(np.ascontiguousarray(val, np.float64).tobytes())
    return h.hexdigest()


def golden(name, n_it):
    s = S.make_system(**S.CONFIGS[name]())
    o = O.Oracle(s)
    (rp, col, val, nz, hmin, pairs) = o.form_h()
    jr, jc, jv = o.form_j()
    p = dict(s.params)
    if n_it is not None:
        p.update(N_it=n_it, admix_crit=0.0)
    res = O.diag4(s.nd, (rp, col, val), hmin, (jr, jc, jv), p, s.ndc)
    out = dict(numh=np.int64(rp[-1]), numzero=np.int64(nz), hmin=np.float64(hmin),
               h_sha=np.array(csr_sha(rp, col, val)), j_sha=np.array(csr_sha(jr, jc, jv)),
               jterms=np.array(O.j_terms(s.basis, s.configs, s.mj), np.int32),
               tk=res["Tk"], tj=res["Tj"], iterations=np.int32(res["iterations"]),
               n_it=np.int32(-1 if n_it is None else n_it))
    if name == "tiny":
        out.update(h_rowptr=rp, h_col=col, h_val=val)
    return out


def main():
    O.build()
    for name, n_it in SYSTEMS:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **golden(name, n_it))
        print("wrote", name)


if __name__ == "__main__":
    main()
