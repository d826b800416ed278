"""Density-matrix truncation after a sector solve, restated in numpy.

TEST INFRASTRUCTURE (oracle): only tests/ use it, as the checker of
dmrgpp_density_truncate.  It restates the reference's per-patch SVD route:
for every group g of the block being truncated, the stacked matrix M_g of the
sector-vector entries of the patches of g (DensityMatrixSvd.h:285-340,
ParallelPsiSplit::doTask; one column block per patch and target, scaled by
sqrt(weight)) and its singular values and left singular vectors
(DensityMatrixSvd.h:355-410, ParallelSvd::doTask: eigs = s^2, LAPACK SVD of
M_g); rho_g = M_g M_g^T is also returned; then the kept number of
Truncation::computeKeptStates
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


def stacked_blocks(lsz, rsz, patch_group, group_size, side, psis, weights=None):
    """M_g for every group (DensityMatrixSvd.h:285-340, ParallelPsiSplit): the
    columns of every patch of g and every target, scaled by sqrt(weight); side
    0 stacks X_p^T (l x r_p), side 1 X_p (r x l_p)."""
    lsz = np.asarray(lsz, dtype=np.int64)
    rsz = np.asarray(rsz, dtype=np.int64)
    xs = np.concatenate([[0], np.cumsum(lsz * rsz)])
    psis = [np.asarray(p, dtype=np.float64) for p in psis]
    w = np.ones(len(psis)) if weights is None else np.asarray(weights, dtype=np.float64)
    cols = [[] for _ in group_size]
    for t, psi in enumerate(psis):
        for p in range(len(lsz)):
            X = psi[xs[p]:xs[p + 1]].reshape(int(lsz[p]), int(rsz[p])).T   # r x l
            cols[int(patch_group[p])].append(np.sqrt(w[t]) * (X.T if side == 0 else X))
    return [np.hstack(c) if c else np.zeros((int(n), 0)) for c, n in zip(cols, group_size)]


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
    # the reference's route: svd('A', M_g) (DensityMatrixSvd.h:355-410), the
    # density-matrix eigenvalues the squared singular values, ascending
    for Mg in stacked_blocks(lsz, rsz, patch_group, group_size, side, psis, weights):
        n = Mg.shape[0]
        if n == 0:
            evals.append(np.zeros(0))
            evecs.append(np.zeros((0, 0)))
            continue
        U, sv, _ = np.linalg.svd(Mg, full_matrices=True)
        w = np.zeros(n)
        w[:len(sv)] = sv ** 2
        evals.append(w[::-1].copy())
        evecs.append(U[:, ::-1].copy())
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
