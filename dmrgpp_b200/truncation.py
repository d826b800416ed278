"""Density-matrix truncation after a sector solve (dmrgpp_density_truncate):
the reduced density matrix of the system or environment block, group by
group, from the solved sector vector(s) on the device, its eigenpairs, and
the kept states (the reference's DensityMatrixSvd + Truncation::changeBasis)."""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _capi


def density_truncate(lsz: Sequence[int], rsz: Sequence[int], patch_group: Sequence[int],
                     group_size: Sequence[int], side: int, psi, m: int, tolerance: float = -1.0,
                     m_min: int = 0, weights: Optional[Sequence[float]] = None,
                     vectors: bool = True, stream: Optional[int] = None, device: int = -1) -> dict:
    """psi: torch CUDA float64 tensor of D (one target) or ntargets x D entries,
    patch order.  Returns per group the ascending eigenvalues, the kept
    states per group (each group's largest) and, if vectors, the kept
    eigenvectors (group size x kept, columns in ascending eigenvalue order),
    the kept total and the discarded weight."""
    L = _capi.lib()
    np_ = len(lsz)
    lsz_a = np.ascontiguousarray(lsz, dtype=np.uint64)
    rsz_a = np.ascontiguousarray(rsz, dtype=np.uint64)
    pg = np.ascontiguousarray(patch_group, dtype=np.uint64)
    gs = np.ascontiguousarray(group_size, dtype=np.uint64)
    D = int(np.sum(lsz_a.astype(np.int64) * rsz_a.astype(np.int64)))
    if psi.numel() % D:
        raise ValueError("psi must hold a whole number of sector vectors")
    nt = psi.numel() // D
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    d = _capi.DensityDesc()
    szp = ctypes.POINTER(ctypes.c_size_t)
    d.npatches = np_
    d.left_patch_size = lsz_a.ctypes.data_as(szp)
    d.right_patch_size = rsz_a.ctypes.data_as(szp)
    d.patch_group = pg.ctypes.data_as(szp)
    d.ngroups = len(gs)
    d.group_size = gs.ctypes.data_as(szp)
    d.side = side
    d.ntargets = nt
    d.psi = psi.data_ptr()
    d.weights = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if w is not None else None
    d.stream = stream
    d.device = device
    N = int(gs.sum())
    eig = np.zeros(max(N, 1))
    vec = np.zeros(max(int(np.sum(gs.astype(np.int64) ** 2)), 1)) if vectors else None
    kept = np.zeros(len(gs), dtype=np.uint64)
    kt = ctypes.c_size_t()
    disc = ctypes.c_double()
    dp = ctypes.POINTER(ctypes.c_double)
    rc = L.dmrgpp_density_truncate(ctypes.byref(d), m, tolerance, m_min, eig.ctypes.data_as(dp),
                                   vec.ctypes.data_as(dp) if vectors else None,
                                   kept.ctypes.data_as(szp), ctypes.byref(kt), ctypes.byref(disc))
    _capi.check(rc)
    evals, evecs, e0, v0 = [], [], 0, 0
    for n, k in zip(gs.astype(np.int64), kept.astype(np.int64)):
        evals.append(eig[e0:e0 + n].copy())
        if vectors:   # views into the one packed output buffer
            evecs.append(vec[v0:v0 + n * k].reshape(n, k, order="F"))
        e0 += n
        v0 += n * k
    return {"eigenvalues": evals, "vectors": evecs if vectors else None,
            "kept": kept.astype(np.int64), "kept_total": int(kt.value),
            "discarded": float(disc.value)}


TRUNCATION_PHASES = ("rho", "eigenvalues", "select", "vectors_host", "vectors_device", "total")


def truncation_profile() -> dict:
    """Seconds of the phases of this thread's last density_truncate
    (dmrgpp_density_profile)."""
    n = len(TRUNCATION_PHASES)
    t = (ctypes.c_double * n)()
    _capi.check(_capi.lib().dmrgpp_density_profile(t, n))
    return {k: float(v) for k, v in zip(TRUNCATION_PHASES, t)}
