"""Complex sectors (BatchedGemm<std::complex<double>> of the reference,
BatchedGemm.cpp:117-119): the real embedding of dmrgpp_kron_create_complex
against the reference's complex known-answer test
(test_KronConnections.cpp:132-178), the numpy oracle (1e-12), the real
handle on real-valued blocks, host against device pointers, TF32x3, and the
solvers' refusal."""
import json
import os

import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _random_complex(seed, npatches, K, maxs, hermitian=False):
    rng = np.random.default_rng(seed)
    l = rng.integers(1, maxs + 1, npatches)
    r = rng.integers(1, maxs + 1, npatches)
    A, B = {}, {}
    for k in range(K):
        for i in range(npatches):
            for j in range(npatches):
                if rng.random() < 0.3:
                    continue
                A[(i, j, k)] = rng.standard_normal((l[i], l[j])) + 1j * rng.standard_normal((l[i], l[j]))
                B[(i, j, k)] = rng.standard_normal((r[i], r[j])) + 1j * rng.standard_normal((r[i], r[j]))
    if hermitian:   # H + H^dagger: add the (j, i) partner of every term
        A2, B2 = dict(A), dict(B)
        for (i, j, k), a in A.items():
            A2[(j, i, k + K)] = a.conj().T
            B2[(j, i, k + K)] = B[(i, j, k)].conj().T
        A, B, K = A2, B2, 2 * K
    return l, r, K, A, B


def _tables(l, r, K, A, B):
    n = len(l)
    tot = n * n * K
    TA, TB = [None] * tot, [None] * tot
    ldA, ldB = np.zeros(tot, dtype=np.uint64), np.zeros(tot, dtype=np.uint64)
    for (i, j, k), a in A.items():
        t = i + j * n + k * n * n
        TA[t], TB[t] = np.asfortranarray(a), np.asfortranarray(B[(i, j, k)])
        ldA[t], ldB[t] = a.shape[0], B[(i, j, k)].shape[0]
    return TA, ldA, TB, ldB


def _handle(l, r, K, A, B, **kw):
    from dmrgpp_b200 import plugin
    TA, ldA, TB, ldB = _tables(l, r, K, A, B)
    return plugin.BatchedGemm(K, len(l), l, r, TA, ldA, TB, ldB, **kw)


def rel_err(y, ref):
    return float(np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300))


def test_reference_complex_known_answer(cuda_lib, cuda_device):
    g = json.load(open(os.path.join(GOLDEN, "kron_connections_complex.json")))
    A, B = {}, {}
    for blk in g["blocks"]:
        A[(blk["out"], blk["in"], 0)] = np.array([[complex(*blk["A"])]])
        B[(blk["out"], blk["in"], 0)] = np.array([[complex(*blk["B"])]])
    bg = _handle(np.array([1, 1]), np.array([1, 1]), 1, A, B)
    try:
        assert bg.is_complex and bg.dim == 2
        x = np.array([complex(*v) for v in g["input"]])
        y = bg(x)
        np.testing.assert_allclose(y, [complex(*v) for v in g["expected_H_input"]], rtol=0, atol=1e-12)
        x_out = np.array([complex(*v) for v in g["x_out_before"]])
        np.testing.assert_allclose(x_out + y, [complex(*v) for v in g["expected_x_out_plus_H_input"]],
                                   rtol=0, atol=1e-12)
    finally:
        bg.close()


@pytest.mark.parametrize("seed,np_,K,maxs", [(1, 1, 1, 3), (2, 4, 2, 17), (3, 6, 3, 40), (4, 3, 2, 120)])
def test_random_complex_sectors_match_oracle(cuda_lib, cuda_device, seed, np_, K, maxs):
    import torch
    from oracle import complex_kron
    l, r, K, A, B = _random_complex(seed, np_, K, maxs)
    bg = _handle(l, r, K, A, B)
    try:
        rng = np.random.default_rng(seed + 100)
        x = rng.standard_normal(bg.dim) + 1j * rng.standard_normal(bg.dim)
        ref = complex_kron.kron_apply(l, r, A, B, x)
        y = bg(x)
        assert rel_err(y, ref) < 1e-12
        yd = bg(torch.from_numpy(x).cuda())
        torch.cuda.synchronize()
        assert np.array_equal(yd.cpu().numpy(), y)
    finally:
        bg.close()


def test_real_valued_blocks_as_complex_equal_the_real_handle(cuda_lib, cuda_device):
    from dmrgpp_b200 import plugin
    prob = sb.random_problem(npatches=5, noperator=3, max_size=30, seed=8, zero_block_rate=0.2)
    real = plugin.BatchedGemm.from_problem(prob)
    Ac = {t: a.astype(np.complex128) for t, a in prob.A.items()}
    Bc = {t: b.astype(np.complex128) for t, b in prob.B.items()}
    cplx = _handle(prob.lsz, prob.rsz, prob.noperator, Ac, Bc)
    try:
        rng = np.random.default_rng(9)
        xr, xi = rng.standard_normal(prob.dim), rng.standard_normal(prob.dim)
        y = cplx(xr + 1j * xi)
        assert rel_err(y.real, real(xr)) < 1e-13 and rel_err(y.imag, real(xi)) < 1e-13
    finally:
        real.close()
        cplx.close()


def test_hermitian_sector_dense_and_solvers_refuse(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200 import _capi, plugin
    l, r, K, A, B = _random_complex(21, 3, 2, 6, hermitian=True)
    bg = _handle(l, r, K, A, B, precision=plugin.TF32X3)
    try:
        D = bg.dim
        H = np.zeros((D, D), dtype=np.complex128)
        from oracle import complex_kron
        for c in range(D):
            e = np.zeros(D, dtype=np.complex128)
            e[c] = 1.0
            H[:, c] = complex_kron.kron_apply(l, r, A, B, e)
        assert np.abs(H - H.conj().T).max() < 1e-12
        x = np.random.default_rng(2).standard_normal(D) + 0j
        bg.set_precision(plugin.FP64)
        assert rel_err(bg(x), H @ x) < 1e-12
        bg.set_precision(plugin.TF32X3)
        assert rel_err(bg(x), H @ x) < 2e-5
        with pytest.raises(_capi.DmrgppError) as err:
            bg.lanczos_lowest(torch.ones(D, dtype=torch.complex128, device="cuda"))
        assert err.value.status == _capi.NOT_SUPPORTED
    finally:
        bg.close()
