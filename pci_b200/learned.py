"""Training data and training for the learned Davidson correction.

The batched solver (include/pci_batch.h) records samples while it solves
(``Batch.set_harvest``): for sampled rows n of a block, every unconverged root
j and every iteration k, the entries x_k[n] and r_k[n] of the root's Ritz
vector and residual, its Ritz value theta, residual norm |r| and H_nn.  After
the solve converges, the target of a sample is the entry of x* - x_k, where
x* is the converged vector of the root that x_k is closest to: the exact
expansion vector that would finish the root in one Rayleigh-Ritz step.  The
network sees per row

* the occupation counts of the orbitals (inputs 0 .. nin-4),
* H_nn - theta (input nin-3),
* r_k[n] * s with s = sqrt(Nd) / |r_k| (input nin-2),
* the diagonal correction r_k[n] * s / (theta - H_nn) of the reference's
  Dvdsn (input nin-1; denominator at least 1e-8 in size, clipped to +-1e4),

and predicts (x* - x_k)[n], scaled so its RMS over the sampled rows of that
root and iteration equals that of the diagonal-correction input (signs of x_k
and r_k aligned with x*).  The solver uses
the prediction as the expansion direction of the root (its length does not
matter: corrections are normalised), with the diagonal correction of the
reference's Dvdsn (davidson.f90:436-570) as the fallback of every root whose
residual stops dropping.
"""
from __future__ import annotations

import numpy as np

from .capi import PCI_BATCH_CORR_LEARNED, PCI_BATCH_FP64, Batch, Engine, Mlp

NSCAL = 3
NIN_DEFAULT = 143   # 140 orbitals (the largest basis of the workloads) + 3 scalars


def occupation_counts(sysm, rows, nin=NIN_DEFAULT):
    """Occupation counts of the orbitals for determinant rows (0-based), [n, nin-3]."""
    norb = nin - NSCAL
    if sysm.nsu > norb:
        raise ValueError(f"{sysm.nsu} orbitals exceed the model's {norb} occupation inputs")
    orb = sysm.nh[sysm.iarr[rows] - 1] - 1            # [n, Ne] 0-based orbitals
    out = np.zeros((len(rows), norb), np.float32)
    np.add.at(out, (np.repeat(np.arange(len(rows)), orb.shape[1]), orb.ravel()), 1.0)
    return out


def samples_to_training(sysm, recs, X, nin=NIN_DEFAULT, blk=0):
    """Features [n, nin] and targets [n] from one block's samples and its
    converged vectors X [Nd, nlv] (the solve's own).

    Samples are grouped by (iteration, root); each group's x_k is matched to
    the converged vector it overlaps most on the sampled rows, signs aligned,
    and the targets scaled to unit RMS within the group."""
    recs = recs[recs["blk"] == blk]
    if recs.size == 0:
        return np.zeros((0, nin), np.float32), np.zeros(0, np.float32)
    nd = sysm.nd
    key = recs["iter"].astype(np.int64) * 64 + recs["root"]
    order = np.argsort(key, kind="stable")
    recs = recs[order]
    key = key[order]
    starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
    ends = np.r_[starts[1:], key.size]
    feats, targs = [], []
    occ_all = occupation_counts(sysm, recs["row"], nin)
    for a, b in zip(starts, ends):
        g = recs[a:b]
        rows = g["row"]
        xk = g["x"]
        xs = X[rows]                                    # [m, nlv]
        ov = xs.T @ xk
        jj = int(np.argmax(np.abs(ov)))
        sgn = 1.0 if ov[jj] >= 0 else -1.0
        t = xs[:, jj] - sgn * xk
        rms = np.sqrt(np.mean(t * t))
        if not np.isfinite(rms) or rms <= 0:
            continue
        f = np.empty((b - a, nin), np.float32)
        f[:, :nin - NSCAL] = occ_all[a:b]
        f[:, nin - 3] = g["diag"] - g["theta"]
        rs = sgn * g["r"] * np.sqrt(nd) / g["rnorm"]
        den = g["theta"] - g["diag"]
        den = np.where(np.abs(den) < 1e-8, np.where(den < 0, -1e-8, 1e-8), den)
        f[:, nin - 2] = rs
        d = np.clip(rs / den, -1e4, 1e4)
        f[:, nin - 1] = d
        drms = np.sqrt(np.mean(d * d))
        if not np.isfinite(drms) or drms <= 0:
            continue
        feats.append(f)
        # on the scale of the diagonal-correction input, so the network can keep it
        targs.append((t / rms * drms).astype(np.float32))
    if not feats:
        return np.zeros((0, nin), np.float32), np.zeros(0, np.float32)
    return np.concatenate(feats), np.concatenate(targs)


def harvest(systems, nlv, rows_per_block=2000, nin=NIN_DEFAULT, device=0, max_sub=48, keep=None, tol=1e-8,
            max_it=400, cap_per_block=400_000, seed=0):
    """Solve every system (one batch, FP64 H and FP64 SpMM, diagonal
    correction) while recording samples; training (features, targets) of the
    blocks that converged, and the solve's result."""
    b = Batch(device)
    b.set_value_prec(64)
    for s in systems:
        with Engine(device) as e:
            e.load_system(s)
            e.form_h(64)
            b.add_engine(e)
    b.set_harvest(rows_per_block, cap_per_block * len(systems), seed)
    r = b.davidson(nlv=nlv, max_sub=max_sub, keep=keep, max_it=max_it, tol=tol, precision=PCI_BATCH_FP64)
    recs, count = b.harvest()
    F, T = [], []
    for i, s in enumerate(systems):
        if r["status"][i] != 1:
            continue
        f, t = samples_to_training(s, recs, b.vectors(i), nin, blk=i)
        F.append(f)
        T.append(t)
    b.close()
    F = np.concatenate(F) if F else np.zeros((0, nin), np.float32)
    T = np.concatenate(T) if T else np.zeros(0, np.float32)
    return F, T, dict(result=r, recorded=count)


def train(F, T, nin=NIN_DEFAULT, device=0, epochs=4, batch=4096, lr=1e-3, seed=0, clip=1e3):
    """A fresh model trained on (F, T) on the GPU (targets clipped to +-clip)."""
    m = Mlp(nin, device, seed)
    T = np.clip(T, -clip, clip).astype(np.float32)
    loss = m.train(F, T, epochs=epochs, batch=batch, lr=lr, seed=seed)
    return m, loss


def solve(systems, nlv, model=None, device=0, value_prec=64, **kw):
    """Solve systems in one batch with the diagonal correction (model None) or
    the learned one; returns (result dict, stats)."""
    b = Batch(device)
    b.set_value_prec(value_prec)
    for s in systems:
        with Engine(device) as e:
            e.load_system(s)
            e.form_h(64)
            b.add_engine(e)
    if model is not None:
        b.set_correction_model(model)
        kw["correction"] = PCI_BATCH_CORR_LEARNED
    r = b.davidson(nlv=nlv, **kw)
    st = b.stats()
    b.close()
    return r, st
