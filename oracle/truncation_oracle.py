"""Density-matrix truncation after a sector solve, restated in numpy.

TEST INFRASTRUCTURE (oracle): only tests/ use it, as the checker of
dmrgpp_density_truncate.  It restates the reference's per-patch SVD route:
for every group g of the block being truncated, the stacked matrix M_g of the
sector-vector entries of the patches of g (DensityMatrixSvd.h:285-340,
ParallelPsiSplit::doTask; one column block per patch and target, scaled by
sqrt(weight)) and its singular values (DensityMatrixSvd.h:355-410,
ParallelSvd::doTask: eigs = s^2), here as the eigenvalues of
rho_g = M_g M_g^T; then the kept number of Truncation::computeKeptStates
(Truncation.h:476-512) and the discarded weight of updateKeptStates
(Truncation.h:373-419, sumUpTo).
"""
from __future__ import annotations

import numpy as np


def density_blocks(lsz, rsz, patch_group, group_size, side, psis, weights=None):
    """rho_g for every group (side 0: sum X_p^T X_p, l x l; side 1: sum
    X_p X_p^T, r x r), X_p the r_p x l_p column-major block of each target."""
    lsz = np.asarray(lsz, dtype=np.int64)
    rsz = np.asarray(rsz, dtype=np.int64)
    xs = np.concatenate([[0], np.cumsum(lsz * rsz)])
    psis = [np.asarray(p, dtype=np.float64) for p in psis]
    w = np.ones(len(psis)) if weights is None else np.asarray(weights, dtype=np.float64)
    rho = [np.zeros((int(n), int(n))) for n in group_size]
    for t, psi in enumerate(psis):
        for p in range(len(lsz)):
            X = psi[xs[p]:xs[p + 1]].reshape(int(lsz[p]), int(rsz[p])).T   # r x l
            g = int(patch_group[p])
            rho[g] += w[t] * (X.T @ X if side == 0 else X @ X.T)
    return rho


def compute_kept_states(kept_states, tolerance, m_min, eigs):
    """Truncation.h:476-512; eigs ascending."""
    if tolerance < 0:
        return kept_states
    n = len(eigs)
    start = max(n - kept_states, 0)
    max_to_remove = max(n - m_min, 0)
    total = m_min
    disc = float(np.sum(np.abs(eigs[:start])))
    for i in range(start, max_to_remove):
        disc += abs(eigs[i])
        if disc > tolerance:
            total = n - i
            break
    if total >= kept_states:
        return kept_states
    if total < m_min:
        return m_min
    return total


def truncate(lsz, rsz, patch_group, group_size, side, psis, m, tolerance=-1.0, m_min=0,
             weights=None):
    """Per group: ascending eigenvalues and eigenvectors; kept per group, kept
    total and discarded weight.  States are ranked by eigenvalue, ties by
    group then index (the reference's std::sort leaves ties unspecified)."""
    rho = density_blocks(lsz, rsz, patch_group, group_size, side, psis, weights)
    evals, evecs = [], []
    for r in rho:
        if r.shape[0] == 0:
            evals.append(np.zeros(0))
            evecs.append(np.zeros((0, 0)))
            continue
        w, v = np.linalg.eigh(0.5 * (r + r.T))
        evals.append(w)
        evecs.append(v)
    flat = [(float(w), g, i) for g, ws in enumerate(evals) for i, w in enumerate(ws)]
    order = sorted(range(len(flat)), key=lambda q: (flat[q][0], q))
    eigs = np.array([flat[q][0] for q in order])
    N = len(flat)
    K = min(compute_kept_states(m, tolerance, m_min, eigs), N)
    kept = np.array([int(n) for n in group_size], dtype=np.int64)
    disc = 0.0
    for q in order[:N - K]:
        kept[flat[q][1]] -= 1
        disc += abs(flat[q][0])
    return {"eigenvalues": evals, "vectors": evecs, "kept": kept, "kept_total": K,
            "discarded": disc, "rho": rho}
