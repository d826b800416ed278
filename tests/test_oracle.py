"""Pins of the CPU oracle (no GPU): against the reference's own golden
vectors, against the reference code compiled from its sources, and against
an explicit dense sector matrix."""
import json
import os

import numpy as np

import oracle
import pytest

from dmrgpp_b200 import superblock as sb

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_matches_reference_unit_test_known_answer(oracle_built):
    """dmrg/Engine/tests/test_BatchedGemm.cpp:171-259 (1 patch, 2x2 (x) 3x3)."""
    g = json.load(open(os.path.join(GOLDEN, "batchedgemm_1patch.json")))
    A = np.asfortranarray(np.array(g["A"]))
    B = np.asfortranarray(np.array(g["B"]))
    prob = sb.KronProblem(np.array([2]), np.array([3]), 1, {(0, 0, 0): A}, {(0, 0, 0): B})
    y = oracle_built.kron_apply(prob, np.array(g["vin"]))
    # the reference test's own tolerance: Catch::Approx(..).epsilon(1e-12)
    np.testing.assert_allclose(y, g["expected"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(y, g["reference_batched_gemm_cpu"], rtol=1e-14, atol=1e-16)


def test_oracle_matches_kron_data31_dump(oracle_built):
    """TestSuite/inputs/kron_data31_0_ref.txt (Heisenberg L=8 H*v dump)."""
    from make_golden import load_kron_data31
    prob, vin, y_ref, rq = load_kron_data31()
    y = oracle_built.kron_apply(prob, vin)
    np.testing.assert_allclose(y, y_ref, rtol=1e-13, atol=1e-15)
    # the dumped vector is the L=8 ground state: <v|H|v>/<v|v> is the exact
    # open-chain energy -3.374932598687897 (to the dump's convergence)
    assert abs(vin @ y / (vin @ vin) - (-3.374932598687897)) < 1e-9
    H = prob.dense()
    np.testing.assert_allclose(H, H.T, atol=1e-12)
    assert abs(np.linalg.eigvalsh(H)[0] - (-3.374932598687897)) < 1e-9


@pytest.mark.parametrize("seed", range(6))
def test_oracle_vs_dense(oracle_built, seed):
    prob = sb.random_problem(npatches=2 + seed % 4, noperator=1 + seed % 3, max_size=9,
                             seed=seed, zero_block_rate=0.3)
    x = np.random.default_rng(seed).standard_normal(prob.dim)
    y = oracle_built.kron_apply(prob, x)
    np.testing.assert_allclose(y, prob.dense() @ x, rtol=1e-12, atol=1e-12)
    assert oracle_built.kron_flops(prob) == prob.flops()


def test_zero_and_missing_blocks_do_not_contribute(oracle_built):
    """setup_nC.cpp:67-121: a triple with an all-zero A or B block is skipped."""
    l, r = np.array([3, 2]), np.array([2, 4])
    rng = np.random.default_rng(1)
    A = {(0, 0, 0): np.asfortranarray(rng.standard_normal((3, 3))),
         (1, 0, 0): np.asfortranarray(np.zeros((2, 3))),
         (0, 1, 0): np.asfortranarray(rng.standard_normal((3, 2)))}
    B = {(0, 0, 0): np.asfortranarray(rng.standard_normal((2, 2))),
         (1, 0, 0): np.asfortranarray(rng.standard_normal((4, 2))),
         (0, 1, 0): np.asfortranarray(np.zeros((2, 4)))}
    prob = sb.KronProblem(l, r, 1, A, B)
    assert prob.triples() == [(0, 0, 0)]
    x = rng.standard_normal(prob.dim)
    y = oracle_built.kron_apply(prob, x)
    assert np.all(y[6:] == 0.0)
    np.testing.assert_allclose(y, prob.dense() @ x, rtol=1e-13)


@pytest.mark.skipif(not os.path.isdir(oracle.REFERENCE_TREE) and
                    not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle",
                                                    "_ref", "libref_kron.so")),
                    reason="reference harness not built")
@pytest.mark.parametrize("seed", range(3))
def test_oracle_vs_reference_batched_gemm_cpu(oracle_built, seed):
    """The restatement against Dmrg::BatchedGemmCpu compiled from the reference."""
    prob = sb.random_problem(npatches=4 + seed, noperator=3, max_size=11, seed=10 + seed)
    x = np.random.default_rng(seed).standard_normal(prob.dim)
    y_ref = oracle_built.RefKron(prob).apply(x)
    y = oracle_built.kron_apply(prob, x)
    np.testing.assert_allclose(y, y_ref, rtol=1e-12, atol=1e-13)


@pytest.mark.skipif(not os.path.isdir(oracle.REFERENCE_TREE) and
                    not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle",
                                                    "_ref", "libref_kron.so")),
                    reason="reference harness not built")
def test_oracle_vs_reference_on_microbench_sector(oracle_built):
    prob = sb.c2_problem()
    assert prob.dim == 76406 and len(prob.triples()) == 103
    assert abs(prob.flops() - 1.30138856e8) < 1.0
    x = sb.random_unit_vector(prob.dim, seed=3)
    y_ref = oracle_built.RefKron(prob).apply(x)
    y = oracle_built.kron_apply(prob, x)
    assert np.abs(y - y_ref).max() / np.abs(y_ref).max() < 1e-13


def test_gather_index_restates_copy_in(oracle_built):
    """InitKronHamiltonian.h:158-221: index map from super-basis order to
    patch order, checked against a direct loop on a random permutation."""
    rng = np.random.default_rng(4)
    left_part = np.array([0, 2, 5, 6])     # 3 left groups
    right_part = np.array([0, 1, 4, 6])    # 3 right groups
    nl, nr = 6, 6
    perm_inv = rng.permutation(nl * nr)
    patch_left = np.array([0, 1, 2])
    patch_right = np.array([2, 1, 0])
    dim = sum((left_part[g + 1] - left_part[g]) * (right_part[h + 1] - right_part[h])
              for g, h in zip(patch_left, patch_right))
    # super-basis rows of this sector are a contiguous range starting at offset
    rows = []
    for g, h in zip(patch_left, patch_right):
        for il in range(left_part[g], left_part[g + 1]):
            for ir in range(right_part[h], right_part[h + 1]):
                rows.append(perm_inv[il + ir * nl])
    offset = min(rows)
    remap = {r: i for i, r in enumerate(sorted(rows))}
    perm_inv2 = perm_inv.copy()
    for k in range(len(perm_inv2)):
        if perm_inv2[k] in remap:
            perm_inv2[k] = remap[perm_inv2[k]] + offset
    idx = oracle_built.gather_index(3, left_part, right_part, patch_left, patch_right, nl,
                                    perm_inv2, offset, dim)
    vin = rng.standard_normal(dim)
    yin = vin[idx]
    q = 0
    for g, h in zip(patch_left, patch_right):
        sl, sr = left_part[g + 1] - left_part[g], right_part[h + 1] - right_part[h]
        for il in range(sl):
            for ir in range(sr):
                r = perm_inv2[(il + left_part[g]) + (ir + right_part[h]) * nl]
                assert yin[q + ir + il * sr] == vin[r - offset]
        q += sl * sr
    assert sorted(idx.tolist()) == list(range(dim))


@pytest.mark.skipif(not os.path.isdir(oracle.REFERENCE_TREE) and
                    not os.path.exists(oracle.REF_KC_SO), reason="reference harness not built")
@pytest.mark.parametrize("threads", [1, 4])
def test_reference_nonbatched_path_matches_restatement(oracle_built, threads):
    """The reference's default CPU H*x (KronConnections::doTask with
    den_kron_mult per block, compiled from its sources) against the
    restatement, on a ragged sector with absent and all-zero blocks and on
    the microbench sector."""
    for prob in (sb.random_problem(npatches=6, noperator=3, max_size=40, seed=3,
                                   zero_block_rate=0.2), sb.c2_problem()):
        x = np.random.default_rng(1).standard_normal(prob.dim)
        y = oracle_built.RefKronConn(prob).apply(x, threads=threads)
        ref = oracle_built.kron_apply(prob, x)
        assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.skipif(not os.path.isdir(oracle.REFERENCE_TREE) and
                    not os.path.exists(oracle.REF_KC_SO), reason="reference harness not built")
def test_reference_kron_methods_on_the_kronutil_test_grid(oracle_built):
    """The grid of the reference's own KronUtil test (dmrg/KronUtil/test1.cpp:
    A blocks of 1, 4, 7 rows and columns, B blocks of 1, 4, 7, 10 rows and
    1, 4, 7 columns, each entry kept with probability 1 - threshold for
    thresholds 0, 0.1, ..., 1.1), untransposed as the plugin path uses them:
    a two-patch sector whose one term couples patch 1 into patch 0 with such
    blocks, through the reference's den_kron_mult (which picks method 1, 2 or
    3 from the blocks' nonzero counts; at threshold 1.1 a block is all zero
    and the term drops out) against the restatement.  Every threshold pair,
    three block shapes each."""
    from dmrgpp_b200.superblock import KronProblem
    rng = np.random.default_rng(7)
    shapes = [(ra, ca, rb, cb) for ra in (1, 4, 7) for ca in (1, 4, 7)
              for rb in (1, 4, 7, 10) for cb in (1, 4, 7)]
    count = 0
    for ia in range(12):
        for ib in range(12):
            for q in range(3):
                ra, ca, rb, cb = shapes[(37 * (12 * ia + ib) + 11 * q) % len(shapes)]

                def sparse(rows, cols, thr):
                    m = rng.standard_normal((rows, cols))
                    m[rng.random((rows, cols)) < thr] = 0.0
                    return np.asfortranarray(m)

                A = {(0, 1, 0): sparse(ra, ca, 0.1 * ia)}
                B = {(0, 1, 0): sparse(rb, cb, 0.1 * ib)}
                prob = KronProblem(np.array([ra, ca], dtype=np.int64), np.array([rb, cb], dtype=np.int64),
                                   1, A, B, name="kronutil-grid")
                x = rng.standard_normal(prob.dim)
                y = oracle_built.RefKronConn(prob).apply(x, threads=1)
                ref = oracle_built.kron_apply(prob, x)
                assert np.abs(y - ref).max(initial=0.0) <= 1e-13 * max(1.0, np.abs(ref).max(initial=0.0)), \
                    (ia, ib, ra, ca, rb, cb)
                count += 1
    assert count == 432
