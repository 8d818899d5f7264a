"""conf_pt's host steps around the second-order pass: which part of the CI
space is the zero-order space, the weights of the non-relativistic (NR)
configurations, and the reordered configuration list for the next CI run.

The reference runs them on its master rank around PTE
(src/conf_pt.f90:61-110): Weight_CI before PT_Init, then Weight_PT, Cutoff,
Sort and NewConfList after it.  They are host logic over O(Ncnr) numbers;
the device work they consume is pci_gpu_pt2_groups (each PT NR
configuration's dE and dV).  NR configurations are pci_b200.system.nr_layout's
(NR_Init).  Indices here are 0-based; the reference's are 1-based.

Energies follow the engine's convention (dE negative for a lowest level); the
reference's dE(n,ic) is -dEg[ic, n].
"""
from __future__ import annotations

import numpy as np

# conf_pt.f90:16, the largest zero-order space PT_Init accepts
IPPT = 5000
# the reference's lg e and lg 2 as it writes them (conf_pt.f90:1033, 1062):
# kept so that weights on a cutoff boundary fall on the same side
LG_E = 0.4342945
LG_2 = 0.301029996


def weight_ci(X, ndcnr_ci, nrn_ci, cut0, ippt=IPPT):
    """Weight_CI (src/conf_pt.f90:573-654).  X: the CI vectors over the CI
    space's determinants (nd1 x nlv); ndcnr_ci, nrn_ci: determinants and
    relativistic configurations of each CI NR configuration.

    For each level the NR configurations are taken in order and their weight
    (the sum of squared coefficients) is taken off a running tail starting
    at 1; the zero-order space of that level runs through the NR
    configuration at which the tail first falls below cut0 (and stays below
    ippt determinants).  Nd0 is the largest over the levels.  Returns dict
    nd0, nc0 (relativistic configurations), ncnr0 (NR configurations), wmax
    (the largest tail left out), dvnr (each CI NR configuration's weight
    summed over the levels)."""
    X = np.asarray(X, np.float64)
    if X.ndim == 1:
        X = X[:, None]
    ndcnr_ci = np.asarray(ndcnr_ci, np.int64)
    nrn_ci = np.asarray(nrn_ci, np.int64)
    if int(ndcnr_ci.sum()) > X.shape[0]:
        raise ValueError("the CI NR configurations hold more determinants than the vectors")
    dvnr = np.zeros(len(ndcnr_ci))
    nd0 = nc0 = ncnr0 = 0
    wmax = 0.0
    # the reference's per-level variables persist from one level to the next
    nd0j = nc0j = ncnr0j = 0
    wj0 = 0.0
    for j in range(X.shape[1]):
        b = X[:, j]
        wj = 1.0
        i = ic = 0
        tail = False
        for icnr in range(len(ndcnr_ci)):
            ic += int(nrn_ci[icnr])
            ndk = int(ndcnr_ci[icnr])
            d = float(np.sum(b[i:i + ndk] ** 2))
            i += ndk
            dvnr[icnr] += d
            wj -= d
            if not tail and i < ippt:
                nd0j, nc0j, ncnr0j, wj0 = i, ic, icnr + 1, wj
            tail = wj < cut0
        if wj0 > wmax:
            wmax = wj0
        if nd0 < nd0j:
            nd0, nc0, ncnr0 = nd0j, nc0j, ncnr0j
    return {"nd0": nd0, "nc0": nc0, "ncnr0": ncnr0, "wmax": wmax, "dvnr": dvnr}


def pt_nr_weights(dEg, dVg):
    """PTE's per-NR-configuration summary (src/conf_pt.f90:887-900, 933-949)
    from pci_gpu_pt2_groups' sums of the PT NR configurations: DEnr (the
    largest reference-convention dE over the levels, at least 0), DVnr (dV
    summed over the levels), and the largest weight with its configuration
    (0-based index among the PT NR configurations; -1 when every weight is
    0)."""
    dEg = np.atleast_2d(np.asarray(dEg, np.float64))
    dVg = np.atleast_2d(np.asarray(dVg, np.float64))
    denr = np.maximum(0.0, (-dEg).max(axis=1)) if dEg.size else np.zeros(0)
    dvnr = dVg.sum(axis=1)
    dvnrx, ix = 0.0, -1
    for k, w in enumerate(dvnr):
        if w > dvnrx:
            dvnrx, ix = float(w), k
    return {"denr": denr, "dvnr": dvnr, "dvnrx": dvnrx, "ix": ix}


def weight_pt(dvnr_ci, dvnr_pt, dvnrx):
    """Weight_PT (src/conf_pt.f90:991-1013): how many CI NR configurations
    weigh less than the largest PT weight, and how many PT NR configurations
    weigh more than the smallest CI weight.  Returns (icci, icpt, dvnrn)."""
    dvnrn = 11.0e1
    icci = 0
    for w in dvnr_ci:
        if w < dvnrx:
            icci += 1
        if w < dvnrn:
            dvnrn = float(w)
    icpt = int(sum(1 for w in dvnr_pt if w > dvnrn))
    return icci, icpt, dvnrn


def cutoff(dvnr, nrn, dvnrx, ktf, kvar, ncnr0, ncnrci):
    """Cutoff (src/conf_pt.f90:1015-1091).  dvnr: the weights of all NR
    configurations (CI ones from weight_ci, PT ones from pt_nr_weights);
    the threshold is dvnrx / 2**ktf on a lg scale, and the first nc_0 NR
    configurations are kept whatever their weight (kvar 1: none, 2: the
    zero-order space's ncnr0, 3: the CI space's ncnrci).  Returns dict w
    (Ncnr x 2: lg weight, -99 for 0; 1 kept / 0 dropped), nc_0, ncnew (the
    relativistic configurations kept), ctf (the lg threshold)."""
    dvnr = np.asarray(dvnr, np.float64)
    nrn = np.asarray(nrn, np.int64)
    if dvnrx <= 0.0:
        raise ValueError("cutoff needs a positive largest PT weight")
    w = np.zeros((len(dvnr), 2))
    for k, wx in enumerate(dvnr):
        w[k, 0] = np.log(wx) * LG_E if wx > 0.0 else -99.0
    ctf = np.log(dvnrx) * LG_E - LG_2 * ktf
    nc_0 = {2: ncnr0, 3: ncnrci}.get(kvar, 0)
    ncnew = 0
    for k in range(len(dvnr)):
        if w[k, 0] > ctf or k < nc_0:
            w[k, 1] = 1.0
            ncnew += int(nrn[k])
    return {"w": w, "nc_0": nc_0, "ncnew": ncnew, "ctf": ctf}


def sort_nr(w, nc_0):
    """Sort (src/conf_pt.f90:1093-1128): the NR configurations beyond the
    first nc_0 ordered by lg weight, largest first, by the reference's
    selection sort (for each position the first largest of the rest is
    swapped in, so equal weights may change order).  Returns the new order
    as indices of the old NR configurations."""
    w1 = [float(x) for x in np.asarray(w)[:, 0]]
    order = list(range(len(w1)))
    for ic in range(nc_0, len(w1) - 1):
        x, i1 = -100.0, ic
        for kc in range(ic, len(w1)):
            if w1[kc] > x:
                i1, x = kc, w1[kc]
        if i1 != ic:
            w1[i1], w1[ic] = w1[ic], w1[i1]
            order[i1], order[ic] = order[ic], order[i1]
    return order


def new_conf_list(order, w, nrr, nrn, ndc, nc_0, nc4, maxnd0, ncnrci):
    """NewConfList (src/conf_pt.f90:1130-1264) without the text file: the
    relativistic configurations in their new order (old 0-based indices),
    the new CI space (the configurations before the first dropped NR
    configuration), the new Nc4 (the leading NR configurations that fit in
    maxnd0 determinants, when nc_0 < nc4) and Kl4 (2, start from the stored
    vectors, when the CI space was kept; else 1).  Returns dict conf_order,
    nci, nc4, kl4, weights (each NR configuration's weight in the new
    order, 10**lg as the reference prints it)."""
    w = np.asarray(w, np.float64)
    ndc = np.asarray(ndc, np.int64)
    if nc_0 < nc4:
        kd4 = kc4 = 0
        for k in order:
            kd = int(ndc[nrr[k]:nrr[k] + nrn[k]].sum())
            if kd4 + kd > maxnd0:
                break
            kd4 += kd
            kc4 += int(nrn[k])
        nc4 = kc4 if kc4 > 0 else int(nrn[order[0]])
    kl4 = 2 if nc_0 == ncnrci else 1
    conf_order, nci, inci = [], 0, True
    for k in order:
        if w[k, 1] == 0.0:
            inci = False
        for ic in range(int(nrr[k]), int(nrr[k] + nrn[k])):
            conf_order.append(ic)
            if inci:
                nci += 1
    return {"conf_order": conf_order, "nci": nci, "nc4": int(nc4), "kl4": kl4,
            "weights": [10.0 ** w[k, 0] for k in order]}


def pt_level_table(E, dE, J=None):
    """PTE's result table (src/conf_pt.f90:909-925) in the reference's sign
    convention: per level n, (n, J, Ev0, DEL0, dE(PT2), Ev(PT2), DEL) with
    Ev0 = -E_n (E the engine's eigenvalues of H), dE(PT2) = -dE_n (the
    engine's pt2 result), Ev(PT2) = Ev0 + dE(PT2), and the intervals from
    the first level in cm^-1, DEL0 = (Ev0_1 - Ev0_n) 2 Ry and DEL = DEL0 +
    (dE_1 - dE_n) 2 Ry with the reference's dE."""
    from .conf_lsj import DPRY
    en = -np.asarray(E, np.float64)
    ey = -np.asarray(dE, np.float64)
    J = np.full(len(en), np.nan) if J is None else np.asarray(J, np.float64)
    rows = []
    for n in range(len(en)):
        des0 = (en[0] - en[n]) * 2 * DPRY
        des = des0 + (ey[0] - ey[n]) * 2 * DPRY
        rows.append((n + 1, float(J[n]), float(en[n]), float(des0), float(ey[n]), float(en[n] + ey[n]), float(des)))
    return rows


def save_vectors(path, EnG, Xj, X_ci, Xpt, nd1):
    """SaveVectors (src/conf_pt.f90:954-989): CONF_PT.XIJ, one record per
    level (pci_io's CONF.XIJ layout) holding the CI vector over the first
    nd1 determinants and the first-order coefficients beyond them, the whole
    normalised.  EnG and Xj are the levels' energies and J as the CI run's
    CONF.XIJ holds them (PT_Init adds 4 Gj J(J+1) to EnG and SaveVectors
    takes it off again, so they are written back unchanged); X_ci is nd1 x
    nlv; Xpt the engine's first-order coefficients (pci_gpu_pt2's Xpt, Nd x
    nlv).  The reference's coefficients are x / (En + H_ii) with En = -E
    (conf_pt.f90:865-874), the engine's x / (E - H_ii): the PT part is
    written as -Xpt.  Returns the written vectors (Nd x nlv)."""
    from . import files
    X_ci = np.asarray(X_ci, np.float64)
    if X_ci.ndim == 1:
        X_ci = X_ci[:, None]
    Xpt = np.asarray(Xpt, np.float64)
    if Xpt.ndim == 1:
        Xpt = Xpt[:, None]
    nd, nlv = Xpt.shape
    if X_ci.shape != (nd1, nlv):
        raise ValueError("X_ci must be nd1 x nlv")
    X = np.zeros((nd, nlv))
    X[:nd1] = X_ci
    X[nd1:] = -Xpt[nd1:]
    X /= np.sqrt(np.sum(X * X, axis=0))
    files.write_xij(path, np.asarray(EnG, np.float64)[:nlv], np.asarray(Xj, np.float64)[:nlv], X)
    return X


def select_configurations(layout, ncnrci, ndc, X_ci, dEg, dVg, cut0, ktf=5, kvar=1, nc4=None, maxnd0=3000):
    """conf_pt's selection end to end: Weight_CI on the CI vectors, the PT
    weights from pci_gpu_pt2_groups' sums over the PT NR configurations,
    Weight_PT, Cutoff, Sort and NewConfList.  layout: nr_layout of the whole
    list; ncnrci: how many NR configurations form the CI space.  ktf and
    kvar default to cpt.in's defaults (src/conf_pt.f90:1413-1414)."""
    nrn, nrr, ndcnr = layout["nrn"], layout["nrr"], layout["ndcnr"]
    wci = weight_ci(X_ci, ndcnr[:ncnrci], nrn[:ncnrci], cut0)
    pt = pt_nr_weights(dEg, dVg)
    if len(pt["dvnr"]) != len(nrn) - ncnrci:
        raise ValueError("one dE/dV row per PT NR configuration expected")
    icci, icpt, dvnrn = weight_pt(wci["dvnr"], pt["dvnr"], pt["dvnrx"])
    dvnr = np.concatenate([wci["dvnr"], pt["dvnr"]])
    cut = cutoff(dvnr, nrn, pt["dvnrx"], ktf, kvar, wci["ncnr0"], ncnrci)
    order = sort_nr(cut["w"], cut["nc_0"])
    new = new_conf_list(order, cut["w"], nrr, nrn, ndc, cut["nc_0"],
                        int(nrr[-1] + nrn[-1]) if nc4 is None else nc4, maxnd0, ncnrci)
    if new["nci"] != cut["ncnew"]:
        raise ValueError(f"new CI space {new['nci']} differs from the kept configurations {cut['ncnew']}")
    return {"weight_ci": wci, "pt": pt, "icci": icci, "icpt": icpt, "dvnrn": dvnrn, "cutoff": cut,
            "nr_order": order, **new}
