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
