"""Host parts of the eigensolver (no GPU): the library's tridiagonal
eigensolver against SciPy, and the reference-Lanczos fixtures against exact
diagonalisation."""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("n", [1, 2, 3, 7, 40, 200, 600])
def test_tridiag_eigen_matches_scipy(cuda_lib, n):
    from scipy.linalg import eigh_tridiagonal
    from dmrgpp_b200 import plugin
    rng = np.random.default_rng(n)
    d = rng.standard_normal(n)
    e = rng.standard_normal(max(n - 1, 0))
    if n > 10:
        e[n // 2] = 0.0   # reducible matrix
        e[n // 4] = 1e-300
    w, Z = plugin.tridiag_eigen(d, e)
    w_ref = eigh_tridiagonal(d, e, eigvals_only=True)
    scale = max(1.0, np.abs(w_ref).max())
    assert np.abs(w - w_ref).max() < 1e-13 * scale
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    assert np.abs(T @ Z - Z * w).max() < 1e-12 * scale
    assert np.abs(Z.T @ Z - np.eye(n)).max() < 1e-12


def test_tridiag_eigen_lanczos_like_spectrum(cuda_lib):
    """Wilkinson's W21+ (pairs of nearly equal eigenvalues)."""
    from scipy.linalg import eigh_tridiagonal
    from dmrgpp_b200 import plugin
    d = np.abs(np.arange(21) - 10.0)
    e = np.ones(20)
    w = plugin.tridiag_eigen(d, e, vectors=False)
    assert np.abs(w - eigh_tridiagonal(d, e, eigvals_only=True)).max() < 1e-13


def test_reference_lanczos_fixtures_are_exact():
    """PsimagLite::LanczosSolver (compiled from the reference) reproduces exact
    diagonalisation to 1e-12 relative on the small fixture sectors."""
    g = json.load(open(os.path.join(GOLDEN, "lanczos_reference.json")))
    for name, c in g.items():
        if c["exact"] is not None:
            assert abs(c["energy"] - c["exact"]) < 1e-12 * abs(c["exact"]), name
        assert abs(c["z_norm"] - 1.0) < 1e-10
    assert abs(g["kron_data31"]["exact"] - (-3.374932598687897)) < 1e-12


def test_lanczos_params_defaults_mirror_reference(cuda_lib):
    import ctypes
    from dmrgpp_b200 import _capi
    p = _capi.LanczosParams()
    cuda_lib.dmrgpp_lanczos_params_init(ctypes.byref(p))
    # ParametersForSolver.h:93-120: LanczosSteps 200, MinSteps 4, Eps 1e-12, EigsForStop 1
    assert (p.steps, p.min_steps, p.eigs_for_stop, p.tolerance) == (200, 4, 1, 1e-12)
