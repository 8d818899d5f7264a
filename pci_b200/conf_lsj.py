"""conf_lsj's level table (PrintLSJ, src/conf_lsj.f90:958-1093): for each
level its J, L and S (pci_gpu_lsj, the same formulas as pconf's lsj), the
non-relativistic g-factor, the energy with the Gj J^2 shift taken off, the
energy above the core and the interval from the lowest level in cm^-1, and
the weight of every configuration in every level.  Host formatting of
numbers the device has produced, as in the reference's master rank.
"""
from __future__ import annotations

import numpy as np

# the Rydberg constant in cm^-1 the reference uses (src/params.f90:18)
DPRY = 109737.315709


def lande_g(J, L, S):
    """g = (3 J(J+1) - L(L+1) + S(S+1)) / (2 J(J+1)), PrintLSJ's g-factor
    (conf_lsj.f90:1029); J = 0 gives nan."""
    J, L, S = (np.asarray(v, np.float64) for v in (J, L, S))
    jj = J * (J + 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        return (3 * jj - L * (L + 1) + S * (S + 1)) / (2 * jj)


def config_weights(X, ndc):
    """W[ic, n]: the sum of squared coefficients of level n over the
    determinants of configuration ic (conf_lsj.f90:1041-1059)."""
    X = np.asarray(X, np.float64)
    if X.ndim == 1:
        X = X[:, None]
    ends = np.concatenate([[0], np.cumsum(np.asarray(ndc, np.int64))])
    if ends[-1] != X.shape[0]:
        raise ValueError("the configurations' determinants differ from the vectors' length")
    sq = np.vstack([np.zeros((1, X.shape[1])), np.cumsum(X * X, axis=0)])
    return sq[ends[1:]] - sq[ends[:-1]]


def level_table(E, J, L, S, gj=0.0, ecore=0.0):
    """PrintLSJ's rows (conf_lsj.f90:1014-1035): per level n, (n, J, L, S, g,
    E, E - Ecore, DEL) with E the stored energy plus 4 Gj J(J+1) and DEL =
    (E_1 - E_n) * 2 Ry in cm^-1; energies in the reference's sign convention
    (the engine's eigenvalues of H with the sign flipped)."""
    E = np.asarray(E, np.float64)
    J = np.asarray(J, np.float64)
    et = E + 4.0 * gj * J * (J + 1.0)
    g = lande_g(J, L, S)
    rows = []
    for n in range(len(E)):
        rows.append((n + 1, float(J[n]), float(L[n]), float(S[n]), float(g[n]), float(et[n]),
                     float(et[n] - ecore), float((et[0] - et[n]) * 2 * DPRY)))
    return rows
