"""The density-matrix truncation oracle on the CPU: the kept-state rule of
Truncation::computeKeptStates (Truncation.h:476-512) on hand-worked cases,
and the oracle's selection against the DMRG driver's own truncation."""
import os
import subprocess

import numpy as np

from oracle import truncation_oracle as to

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


EIGS = np.array([1e-9, 1e-8, 1e-6, 1e-3, 0.1, 0.898998989])


def test_negative_tolerance_keeps_m():
    assert to.compute_kept_states(4, -1.0, 0, EIGS) == 4


def test_tolerance_exceeded_at_start_keeps_m():
    # removing the two smallest (m = 4) leaves 1.1e-8; the next one passes 1e-7
    assert to.compute_kept_states(4, 1e-7, 0, EIGS) == 4


def test_tolerance_reduces_the_kept_states():
    # m = 5: 1e-9 + 1e-8 + 1e-6 + 1e-3 stays below 1e-2, adding 0.1 does not
    assert to.compute_kept_states(5, 1e-2, 1, EIGS) == 2


def test_m_min_floor():
    # nothing exceeds the tolerance up to n - m_min removals: m_min states kept
    assert to.compute_kept_states(5, 1.0, 3, EIGS) == 3


def test_oracle_selection_matches_the_driver_truncation():
    """Same kept subspace per group as oracle/dmrg_driver.py's truncation of
    the same density matrices (distinct eigenvalues)."""
    from oracle import dmrg_driver as dd
    rng = np.random.default_rng(4)
    lsz, rsz = [5, 7, 3, 6], [4, 6, 8, 2]
    D = int(np.dot(lsz, rsz))
    psi = rng.standard_normal(D)
    psi /= np.linalg.norm(psi)
    out = to.truncate(lsz, rsz, [0, 1, 2, 3], lsz, 0, [psi], m=9)
    assert out["kept_total"] == 9 and int(out["kept"].sum()) == 9
    drv = dd.DMRG.__new__(dd.DMRG)
    drv.m = 9
    blk = dd.Block(qns=[(q,) for q in range(4)], sizes=list(lsz),
                   ops={"H": {(g, g): np.eye(n) for g, n in enumerate(lsz)}})
    new = drv.truncate(blk, {g: r for g, r in enumerate(out["rho"])})
    kept_groups = [g for g in range(4) if out["kept"][g] > 0]
    assert new.sizes == [int(out["kept"][g]) for g in kept_groups]
    allw = np.sort(np.concatenate(out["eigenvalues"]))
    assert abs(allw.sum() - 1.0) < 1e-12                     # trace of rho = |psi|^2
    assert abs(out["discarded"] - np.abs(allw[:len(allw) - 9]).sum()) < 1e-15


def test_group_eigenvalue_phase(tmp_path):
    """The library's host eigenvalue phase (tridiag.cpp, compiled here with
    g++): AVX2 and baseline reductions bitwise alike, the square-root-free QL
    against the QL with rotations, and group_eigenvalues over mixed group
    sizes and thread counts against each group's serial reduction."""
    exe = str(tmp_path / "group_eigen_check")
    csrc = os.path.join(ROOT, "dmrgpp_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + csrc,
                    os.path.join(ROOT, "tests", "group_eigen_check.cpp"),
                    os.path.join(csrc, "tridiag.cpp"), "-o", exe, "-lpthread"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr


def _shim(tmp_path):
    import ctypes
    so = str(tmp_path / "libtruncation_host_shim.so")
    csrc = os.path.join(ROOT, "dmrgpp_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O2", "-shared", "-fPIC", "-I" + csrc,
                    os.path.join(ROOT, "tests", "truncation_host_shim.cpp"),
                    os.path.join(csrc, "tridiag.cpp"), "-o", so, "-lpthread"], check=True)
    return ctypes.CDLL(so)


def _host_truncate(lib, rho, m, tol, mmin, threads):
    """The library's host steps on the oracle's density matrices, in the
    order dmrgpp_density_truncate takes them: eigenvalues of every group,
    the ranking (ascending, ties by group then index) and computeKeptStates,
    then the kept eigenvectors (the device's V = Q Z done by apply_q)."""
    import ctypes
    ng = len(rho)
    n = np.array([r.shape[0] for r in rho], dtype=np.uint64)
    a = [np.asfortranarray(r).copy() for r in rho]
    w = [np.zeros(int(k)) for k in n]
    P = ctypes.POINTER(ctypes.c_double)
    ap = (P * ng)(*[x.ctypes.data_as(P) for x in a])
    wp = (P * ng)(*[x.ctypes.data_as(P) for x in w])
    szp = ctypes.POINTER(ctypes.c_size_t)
    assert lib.shim_eigenvalues(ctypes.c_size_t(ng), n.ctypes.data_as(szp), ap, wp, threads) == 0
    flat = np.concatenate(w) if ng else np.zeros(0)
    order = np.argsort(flat, kind="stable")
    N = len(flat)
    K = min(to.compute_kept_states(m, tol, mmin, flat[order]), N)
    gof = np.repeat(np.arange(ng), n.astype(np.int64))
    kept = n.astype(np.int64).copy()
    for q in order[:N - K]:
        kept[gof[q]] -= 1
    z = [np.zeros(max(int(nn) * int(k), 1)) for nn, k in zip(n, kept)]
    wk = (P * ng)(*[(x[len(x) - k:] if k else x).ctypes.data_as(P) for x, k in zip(w, kept)])
    zp = (P * ng)(*[x.ctypes.data_as(P) for x in z])
    kk = kept.astype(np.uint64)
    lib.shim_vectors(ctypes.c_size_t(ng), n.ctypes.data_as(szp), kk.ctypes.data_as(szp), wk, zp, threads)
    vecs = [x[:int(nn) * int(k)].reshape(int(nn), int(k), order="F") for x, nn, k in zip(z, n, kept)]
    return w, kept, K, vecs


def test_host_truncation_pipeline_against_the_oracle(tmp_path):
    """The library's host phases of the truncation (group_eigenvalues with a
    thread team for the largest group, the kept-state rule, group_eigenvectors
    and the reflectors' back-transformation) on the oracle's density matrices,
    for both blocks, one and two weighted targets, random and low-rank sector
    vectors, groups shared by patches and a group without patches: the same
    kept states as the oracle's SVD route (where the cut lies above rounding
    noise), eigenvalues within 1e-14,
    orthonormal eigenvectors of the oracle's rho_g to 1e-13, the kept
    subspace the oracle's where the cut has a gap."""
    lib = _shim(tmp_path)
    for side in (0, 1):
        for targets in (1, 2):
            for low_rank in (False, True):
                rng = np.random.default_rng(100 * side + 10 * targets + low_rank)
                gsize = [150, 37, 64, 5, 1, 90, 12]
                lsz, rsz, pg = [], [], []
                for g, n in enumerate(gsize):
                    for _ in range(int(rng.integers(1, 3))):
                        other = int(rng.integers(1, 60 if low_rank else 200))
                        lsz.append(n if side == 0 else other)
                        rsz.append(other if side == 0 else n)
                        pg.append(g)
                gs = gsize + [9]
                D = int(np.dot(lsz, rsz))
                psis = []
                for _ in range(targets):
                    p = rng.standard_normal(D)
                    if low_rank:   # a decaying spectrum: most weights far below the norm
                        p *= np.exp(-0.02 * np.arange(D))
                    psis.append(p / np.linalg.norm(p))
                wts = [1.0] if targets == 1 else [0.6, 0.4]
                Ntot = sum(gs)
                for m, tol, mmin in ((Ntot // 3, -1.0, 0), (Ntot // 2, 1e-6, 4), (Ntot + 5, -1.0, 0)):
                    ref = to.truncate(lsz, rsz, pg, gs, side, psis, m, tol, mmin, weights=wts)
                    w, kept, K, vecs = _host_truncate(lib, ref["rho"], m, tol, mmin, threads=8)
                    assert K == ref["kept_total"], (side, targets, low_rank, m)
                    # below ~1e-12 of the largest weight rho_g's eigenvalues are
                    # rounding noise and their order against the SVD's is arbitrary:
                    # the kept states per group are compared where the cut is above it
                    allw = np.sort(np.concatenate(ref["eigenvalues"]))
                    if K == 0 or K == len(allw) or allw[len(allw) - K] > 1e-12 * allw[-1]:
                        assert np.array_equal(kept, ref["kept"]), (side, targets, low_rank, m)
                    for g in range(len(gs)):
                        we, wr = w[g], ref["eigenvalues"][g]
                        assert np.abs(we - wr).max(initial=0.0) <= 1e-14, g
                        V, n, k = vecs[g], gs[g], int(kept[g])
                        assert np.abs(V.T @ V - np.eye(k)).max(initial=0.0) < 1e-12, g
                        assert np.abs(ref["rho"][g] @ V - V * we[n - k:]).max(initial=0.0) < 1e-13, g
                        if 0 < k < n and wr[n - k] - wr[n - k - 1] > 1e-9:
                            Pr = ref["vectors"][g][:, n - k:]
                            assert np.abs(V @ V.T - Pr @ Pr.T).max() < 1e-8, g
