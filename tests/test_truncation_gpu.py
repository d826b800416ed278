"""dmrgpp_density_truncate through the C ABI against the numpy oracle
(oracle/truncation_oracle.py): density-matrix eigenvalues, eigenvectors, the
kept states per group and the discarded weight, for the system and the
environment block, one and two weighted targets, groups shared by several
patches and groups without patches; and whole DMRG runs whose every
truncation goes through the library."""
import json
import os

import numpy as np
import pytest

from oracle import truncation_oracle as to

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _layout(seed, side):
    """Patches whose block-side groups are shared in pairs, plus one empty
    group at the end."""
    rng = np.random.default_rng(seed)
    ng = 5
    gsize = rng.integers(1, 90, ng)
    lsz, rsz, pg = [], [], []
    for g in range(ng):
        for _ in range(int(rng.integers(1, 3))):
            other = int(rng.integers(1, 120))
            lsz.append(int(gsize[g]) if side == 0 else other)
            rsz.append(other if side == 0 else int(gsize[g]))
            pg.append(g)
    return lsz, rsz, pg, [int(x) for x in gsize] + [7]


@pytest.mark.parametrize("side", [0, 1])
@pytest.mark.parametrize("targets", [1, 2])
def test_truncation_matches_oracle(cuda_lib, cuda_device, side, targets):
    import torch
    from dmrgpp_b200.truncation import density_truncate
    lsz, rsz, pg, gs = _layout(10 * side + targets, side)
    D = int(np.dot(lsz, rsz))
    rng = np.random.default_rng(targets)
    psis = [rng.standard_normal(D) for _ in range(targets)]
    psis = [p / np.linalg.norm(p) for p in psis]
    w = [1.0] if targets == 1 else [0.7, 0.3]
    N = sum(gs)
    for m, tol, mmin in ((N // 3, -1.0, 0), (N // 2, 1e-3, 5), (N + 10, -1.0, 0)):
        ref = to.truncate(lsz, rsz, pg, gs, side, psis, m, tol, mmin, weights=w)
        psi_d = torch.tensor(np.concatenate(psis), device="cuda")
        out = density_truncate(lsz, rsz, pg, gs, side, psi_d, m, tol, mmin,
                               weights=w if targets > 1 else None)
        assert out["kept_total"] == ref["kept_total"]
        assert np.array_equal(out["kept"], ref["kept"])
        assert abs(out["discarded"] - ref["discarded"]) <= 1e-13
        for g in range(len(gs)):
            we, wr = out["eigenvalues"][g], ref["eigenvalues"][g]
            assert np.abs(we - wr).max(initial=0.0) <= 1e-14, g
            V = out["vectors"][g]
            n, k = gs[g], int(out["kept"][g])
            assert V.shape == (n, k)
            assert np.abs(V.T @ V - np.eye(k)).max(initial=0.0) < 1e-12
            # eigenvectors of the oracle's density matrix for the kept eigenvalues
            assert np.abs(ref["rho"][g] @ V - V * we[n - k:]).max(initial=0.0) < 1e-13
            if 0 < k < n and wr[n - k] - wr[n - k - 1] > 1e-9:
                P = V @ V.T
                Pr = ref["vectors"][g][:, n - k:] @ ref["vectors"][g][:, n - k:].T
                assert np.abs(P - Pr).max() < 1e-8, g
        assert np.abs(out["eigenvalues"][-1]).max() == 0.0    # the group without patches
        if targets == 1:
            assert abs(sum(x.sum() for x in out["eigenvalues"]) - 1.0) < 1e-12


def test_low_rank_group_keeps_the_states_of_an_svd(cuda_lib, cuda_device):
    """A group whose stacked matrix M_g has singular values 1, 1e-3, 1e-5,
    1e-7, 1e-8 and zeros (weights down to 1e-16), beside a group of full rank,
    with a discarded-weight tolerance of 1e-12: the library (eigenpairs of
    rho_g = M_g M_g^T) keeps the same states per group as the reference's SVD
    of M_g (the oracle), the kept weights agree to 1e-5 relative, and the kept
    subspace agrees with the SVD's to 1e-5.  (rho_g's eigenvalues carry an
    absolute error of about eps ||rho_g||: weights below ~1e-12 ||rho_g|| lose
    relative accuracy, which only a tolerance below that would see.)"""
    import torch
    from dmrgpp_b200.truncation import density_truncate
    rng = np.random.default_rng(5)
    n0, cols0 = 40, (30, 50)
    U, _ = np.linalg.qr(rng.standard_normal((n0, n0)))
    V, _ = np.linalg.qr(rng.standard_normal((sum(cols0), n0)))
    sv = np.zeros(n0)
    sv[:5] = [1.0, 1e-3, 1e-5, 1e-7, 1e-8]
    M0 = U @ np.diag(sv) @ V.T                      # 40 x 80, rank 5
    n1, cols1 = 25, (20,)
    M1 = 0.3 * rng.standard_normal((n1, sum(cols1)))
    lsz, rsz, pg, psi = [], [], [], []
    for g, (M, cols) in enumerate(((M0, cols0), (M1, cols1))):
        c0 = 0
        for c in cols:              # side 0: patch p contributes X_p^T = M[:, c0:c0+c]
            X = M[:, c0:c0 + c].T   # r_p x l_p
            lsz.append(M.shape[0])
            rsz.append(c)
            pg.append(g)
            psi.append(X.flatten(order="F"))
            c0 += c
    psi = np.concatenate(psi)
    gs = [n0, n1]
    ref = to.truncate(lsz, rsz, pg, gs, 0, [psi], m=n0 + n1, tolerance=1e-12, m_min=0)
    out = density_truncate(lsz, rsz, pg, gs, 0, torch.tensor(psi, device="cuda"), n0 + n1, 1e-12, 0)
    assert np.array_equal(out["kept"], ref["kept"]) and out["kept_total"] == ref["kept_total"]
    assert int(out["kept"][0]) == 3                  # weights 1, 1e-6, 1e-10
    for g in range(2):
        k = int(out["kept"][g])
        we, wr = out["eigenvalues"][g][-k:], ref["eigenvalues"][g][-k:]
        assert np.all(np.abs(we - wr) <= 1e-5 * wr), g
        V_l, V_r = out["vectors"][g], ref["vectors"][g][:, -k:]
        assert np.abs(V_l @ V_l.T - V_r @ V_r.T).max() < 1e-5, g


def test_truncation_argument_checks(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200 import _capi
    from dmrgpp_b200.truncation import density_truncate
    psi = torch.zeros(6, dtype=torch.float64, device="cuda")
    with pytest.raises(_capi.DmrgppError):       # group size differs from the patch's
        density_truncate([2], [3], [0], [3], 0, psi, 2)
    with pytest.raises(_capi.DmrgppError):       # group out of range
        density_truncate([2], [3], [1], [2], 0, psi, 2)
    with pytest.raises(_capi.DmrgppError):       # m_min above m
        density_truncate([2], [3], [0], [2], 0, psi, 1, 1e-3, 2)


def gpu_solver(prob, init):
    """FP64 device Lanczos of one superblock sector."""
    from dmrgpp_b200 import plugin
    bg = plugin.BatchedGemm.from_problem(prob)
    try:
        return bg.lanczos_lowest(init, steps=200, tolerance=1e-10)
    finally:
        bg.close()


def gpu_truncator(prob, patches, psi, side, blk, m):
    """The driver's truncation through dmrgpp_density_truncate (groups of the
    enlarged block that appear in the sector, as the driver's own does)."""
    import torch
    from oracle.dmrg_driver import KeptBasis
    from dmrgpp_b200.truncation import density_truncate
    groups = sorted({p[side] for p in patches})
    index = {g: q for q, g in enumerate(groups)}
    pg = [index[p[side]] for p in patches]
    gs = [blk.sizes[g] for g in groups]
    out = density_truncate(prob.lsz, prob.rsz, pg, gs, side,
                           torch.tensor(np.asarray(psi), device="cuda"), m)
    kb = KeptBasis()
    for q, g in enumerate(groups):
        kb[g] = out["vectors"][q]
    return kb


def test_dmrg_with_device_truncation_matches_reference(cuda_lib, cuda_device):
    """Heisenberg L=32, m=128, every solve and every truncation on the device:
    the reference's own test energy (dmrg/CMakeLists.txt:343-344) and the
    run with the driver's host truncation."""
    from oracle import dmrg_driver as dd
    g = json.load(open(os.path.join(GOLDEN, "dmrg_heisenberg_L32_m128.json")))
    d = dd.DMRG(dd.Heisenberg(), L=32, m=128, solver=gpu_solver)
    d.truncator = gpu_truncator
    e = d.run(sweeps=2)
    assert abs(e - g["reference_test_energy"]) < g["reference_test_tolerance"]
    assert abs(e - g["energy"]) < 1e-6, (e, g["energy"])


def test_hubbard_with_device_truncation_is_exact_at_u0(cuda_lib, cuda_device):
    from oracle import dmrg_driver as dd
    d = dd.DMRG(dd.Hubbard(U=0.0), L=8, m=256, solver=gpu_solver)
    d.truncator = gpu_truncator
    e = d.run(sweeps=1)
    assert abs(e - (-9.51754)) < 1e-5          # dmrg/CMakeLists.txt:180-181
    assert abs(e - dd.free_fermion_energy(8, 4, 4)) < 1e-9


def test_operator_change_of_basis_through_wft(cuda_lib, cuda_device):
    """After a truncation, every block operator O(gi, gj) of the block becomes
    U_gi^T O(gi, gj) U_gj (the reference's changeBasis / truncateBasis): one
    dmrgpp_wft call with the operator blocks as patches (rows = right index,
    columns = left index), WR = U_gi^T and WL = U_gj^T; FP64 against numpy."""
    import torch
    from dmrgpp_b200.truncation import density_truncate
    from dmrgpp_b200.wft import WaveFunctionTransform
    lsz, rsz, pg, gs = _layout(7, 0)
    D = int(np.dot(lsz, rsz))
    rng = np.random.default_rng(70)
    psi = rng.standard_normal(D)
    psi /= np.linalg.norm(psi)
    out = density_truncate(lsz, rsz, pg, gs, 0, torch.tensor(psi, device="cuda"), sum(gs) // 2)
    U = out["vectors"]
    kept = [int(k) for k in out["kept"]]
    # block operator: diagonal blocks and neighbouring-group couplings
    pairs = [(g, h) for g in range(len(gs)) for h in range(len(gs))
             if abs(g - h) <= 1 and kept[g] > 0 and kept[h] > 0]
    O = {(g, h): rng.standard_normal((gs[g], gs[h])) for g, h in pairs}
    r_in = [gs[g] for g, h in pairs]
    l_in = [gs[h] for g, h in pairs]
    r_out = [kept[g] for g, h in pairs]
    l_out = [kept[h] for g, h in pairs]
    WR = [U[g].T for g, h in pairs]
    WL = [U[h].T for g, h in pairs]
    w = WaveFunctionTransform(l_in, r_in, l_out, r_out, list(range(len(pairs))), WL, WR)
    x = np.concatenate([O[p].ravel(order="F") for p in pairs])
    y = w(x)
    off = 0
    for (g, h), ro, lo in zip(pairs, r_out, l_out):
        ref = U[g].T @ O[(g, h)] @ U[h]
        got = y[off:off + ro * lo].reshape(ro, lo, order="F")
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), (g, h)
        off += ro * lo
    w.close()
