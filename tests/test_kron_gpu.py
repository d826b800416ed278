"""Parity of the CUDA H*x path (through the C ABI) with the oracle.

FP64 tolerance: max |y - y_oracle| <= 1e-12 * max |y_oracle| (the reference
unit test's epsilon, test_BatchedGemm.cpp:232-257); runs are also required
to be bitwise reproducible from call to call.
"""
import json
import os

import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-12


def rel_err(y, ref):
    return float(np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300))


def gpu_apply(prob, x, **kw):
    from dmrgpp_b200 import plugin
    bg = plugin.BatchedGemm.from_problem(prob, **kw)
    try:
        return bg(np.ascontiguousarray(x))
    finally:
        bg.close()


def test_known_answer_of_reference_unit_test(cuda_lib, cuda_device):
    g = json.load(open(os.path.join(GOLDEN, "batchedgemm_1patch.json")))
    prob = sb.KronProblem(np.array([2]), np.array([3]), 1,
                          {(0, 0, 0): np.asfortranarray(np.array(g["A"]))},
                          {(0, 0, 0): np.asfortranarray(np.array(g["B"]))})
    y = gpu_apply(prob, np.array(g["vin"]))
    np.testing.assert_allclose(y, g["expected"], rtol=1e-12, atol=0)


def test_kron_data31_dump(cuda_lib, cuda_device):
    from make_golden import load_kron_data31
    prob, vin, y_ref, rq = load_kron_data31()
    y = gpu_apply(prob, vin)
    assert rel_err(y, y_ref) < RTOL
    assert abs(vin @ y / (vin @ vin) - rq) < 1e-13


@pytest.mark.parametrize("seed,np_,K,maxs", [(0, 3, 1, 5), (1, 5, 3, 17), (2, 8, 5, 40),
                                             (3, 4, 2, 100), (4, 6, 4, 70), (5, 2, 2, 200),
                                             (6, 10, 6, 33), (7, 1, 1, 1)])
def test_random_ragged_sectors(cuda_lib, cuda_device, oracle_built, seed, np_, K, maxs):
    prob = sb.random_problem(npatches=np_, noperator=K, max_size=maxs, seed=seed,
                             zero_block_rate=0.2)
    x = np.random.default_rng(seed).standard_normal(prob.dim)
    y = gpu_apply(prob, x)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL


def test_large_patches_multi_tile(cuda_lib, cuda_device, oracle_built):
    # patch sizes above the 64x64 tile and odd leading dimensions
    prob = sb.random_problem(npatches=3, noperator=2, max_size=300, min_size=190, seed=11,
                             zero_block_rate=0.0)
    x = np.random.default_rng(2).standard_normal(prob.dim)
    y = gpu_apply(prob, x)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL


def test_output_patch_without_terms_is_zeroed(cuda_lib, cuda_device, oracle_built):
    rng = np.random.default_rng(3)
    l, r = np.array([4, 3, 5]), np.array([2, 6, 3])
    A = {(0, 0, 0): np.asfortranarray(rng.standard_normal((4, 4))),
         (2, 0, 0): np.asfortranarray(rng.standard_normal((5, 4)))}
    B = {(0, 0, 0): np.asfortranarray(rng.standard_normal((2, 2))),
         (2, 0, 0): np.asfortranarray(rng.standard_normal((3, 2)))}
    prob = sb.KronProblem(l, r, 1, A, B)
    from dmrgpp_b200 import plugin
    bg = plugin.BatchedGemm.from_problem(prob)
    x = rng.standard_normal(prob.dim)
    y = np.full(prob.dim, np.nan)
    bg.apply_Htarget(x, y)
    assert np.all(y[8:26] == 0.0)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL


def test_microbench_sector_host_and_device_pointers(cuda_lib, cuda_device, oracle_built):
    import torch
    from dmrgpp_b200 import plugin
    prob = sb.c2_problem()
    x = sb.random_unit_vector(prob.dim, seed=5)
    y_or = oracle_built.kron_apply(prob, x)
    bg = plugin.BatchedGemm.from_problem(prob,
                                         stream=torch.cuda.current_stream().cuda_stream)
    y_host = bg(x)
    assert rel_err(y_host, y_or) < RTOL
    xd = torch.from_numpy(x).to(cuda_device)
    yd = torch.empty_like(xd)
    bg.apply_Htarget(xd, yd)
    torch.cuda.synchronize()
    y_dev = yd.cpu().numpy()
    assert np.array_equal(y_dev, y_host)          # same kernels, same order
    for _ in range(3):                             # bitwise reproducible
        assert np.array_equal(bg(x), y_host)
    bg.close()


def test_symmetric_operator_gives_symmetric_products(cuda_lib, cuda_device):
    prob = sb.c2_problem()
    rng = np.random.default_rng(8)
    u, v = rng.standard_normal(prob.dim), rng.standard_normal(prob.dim)
    from dmrgpp_b200 import plugin
    bg = plugin.BatchedGemm.from_problem(prob)
    a, b = u @ bg(v), v @ bg(u)
    assert abs(a - b) < 1e-11 * (abs(a) + abs(b))
    # linearity
    np.testing.assert_allclose(bg(2.0 * u - 3.0 * v), 2.0 * bg(u) - 3.0 * bg(v), rtol=1e-12,
                               atol=1e-10)


def test_dependency_wait_times_out_and_handle_recovers(cuda_lib, cuda_device, oracle_built):
    """Failure detection without a GPU fault: the test hook makes the kernel's
    waits on input patch 0 unsatisfiable; they give up after their time limit,
    the apply reports TIMEOUT, and the next apply is correct again."""
    from dmrgpp_b200 import _capi, plugin
    prob = sb.c2_problem()
    x = sb.random_unit_vector(prob.dim, seed=9)
    bg = plugin.BatchedGemm.from_problem(prob)
    y_ok = bg(x)
    assert cuda_lib.dmrgpp_kron_test_stall_dependency(bg.handle, 1) == _capi.OK
    with pytest.raises(_capi.DmrgppError) as ei:
        bg(x)
    assert ei.value.status == _capi.TIMEOUT
    assert cuda_lib.dmrgpp_kron_test_stall_dependency(bg.handle, 0) == _capi.OK
    y_again = bg(x)
    assert np.array_equal(y_again, y_ok)
    assert rel_err(y_again, oracle_built.kron_apply(prob, x)) < RTOL
    bg.close()


def test_device_pointer_applies_then_synchronize(cuda_lib, cuda_device, oracle_built):
    """Back-to-back asynchronous applies on one stream (the persistent kernel
    resets its own counters between launches), checked after one sync."""
    import torch
    from dmrgpp_b200 import _capi, plugin
    prob = sb.random_problem(npatches=9, noperator=5, max_size=150, seed=31)
    s = torch.cuda.Stream()
    bg = plugin.BatchedGemm.from_problem(prob, stream=s.cuda_stream)
    rng = np.random.default_rng(4)
    xs = [rng.standard_normal(prob.dim) for _ in range(4)]
    with torch.cuda.stream(s):
        xd = [torch.from_numpy(x).to(cuda_device) for x in xs]
        yd = [torch.empty_like(v) for v in xd]
    for a, b in zip(xd, yd):
        bg.apply_Htarget(a, b)
    assert cuda_lib.dmrgpp_kron_synchronize(bg.handle) == _capi.OK
    for x, y in zip(xs, yd):
        assert rel_err(y.cpu().numpy(), oracle_built.kron_apply(prob, x)) < RTOL
    bg.close()


@pytest.mark.parametrize("cfg", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("ipc", [1, 4])
def test_every_tile_configuration(cuda_lib, cuda_device, oracle_built, cfg, ipc):
    """Each tile configuration / work split of the persistent kernel, on a
    sector with ragged patches (1..150) and many K-segments per output tile."""
    from dmrgpp_b200 import plugin
    prob = sb.random_problem(npatches=12, noperator=4, max_size=150, seed=40 + cfg,
                             density=0.6, zero_block_rate=0.1)
    x = np.random.default_rng(cfg).standard_normal(prob.dim)
    bg = plugin.BatchedGemm.from_problem(prob)
    bg.set_config(cfg, ipc)
    assert bg.get_config() == (cfg, ipc)
    y = bg(x)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL
    assert np.array_equal(bg(x), y)
    bg.close()


def test_autotune_then_cache_hit(cuda_lib, cuda_device, oracle_built, tmp_path):
    from dmrgpp_b200 import plugin
    prob = sb.c2_problem()
    x = sb.random_unit_vector(prob.dim, seed=12)
    cache = str(tmp_path / "tune.txt")
    bg = plugin.BatchedGemm.from_problem(prob)
    cfg, us = bg.autotune(cache, reps=3)
    assert 0 <= cfg < 8 and us > 0
    assert rel_err(bg(x), oracle_built.kron_apply(prob, x)) < RTOL
    bg.close()
    lines = open(cache).read().split("\n")
    assert len([ln for ln in lines if ln.strip()]) == 1
    bg2 = plugin.BatchedGemm.from_problem(prob)
    cfg2, us2 = bg2.autotune(cache, reps=3)      # cache hit: same choice, no new line
    assert (cfg2, us2) == (cfg, pytest.approx(us, rel=1e-6))
    assert len([ln for ln in open(cache).read().split("\n") if ln.strip()]) == 1
    bg2.close()


def test_ladder_shaped_sector(cuda_lib, cuda_device, oracle_built):
    prob = sb.ladder_problem(total_states=1500, sigma=2.0, seed=3)
    x = np.random.default_rng(5).standard_normal(prob.dim)
    y = gpu_apply(prob, x)
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL


def test_blocks_in_larger_arrays(cuda_lib, cuda_device, oracle_built):
    """Blocks whose leading dimension exceeds their rows (ld = rows + 3) go
    through the staged upload column by column."""
    from dmrgpp_b200 import plugin
    prob = sb.random_problem(npatches=5, noperator=3, max_size=60, seed=21, zero_block_rate=0.2)
    A, ldA, B, ldB = prob.tables()
    keep = []

    def embed(tab, ld):
        out, lds = [], list(ld)
        for q, m in enumerate(tab):
            if m is None:
                out.append(None)
                continue
            m = np.asfortranarray(m)
            big = np.zeros((m.shape[0] + 3, m.shape[1]), order="F")
            big[:m.shape[0], :] = m
            keep.append(big)
            out.append(big.ctypes.data)
            lds[q] = m.shape[0] + 3
        return out, lds
    Ap, ldAp = embed(A, ldA)
    Bp, ldBp = embed(B, ldB)
    bg = plugin.BatchedGemm(prob.noperator, prob.npatches, prob.lsz, prob.rsz, Ap, ldAp, Bp, ldBp)
    try:
        x = np.random.default_rng(4).standard_normal(prob.dim)
        assert rel_err(bg(x), oracle_built.kron_apply(prob, x)) < RTOL
    finally:
        bg.close()


def test_operators_spanning_several_upload_chunks(cuda_lib, cuda_device, oracle_built):
    """36 MB of packed operators: more than one 32 MB staging chunk, so the
    pinned buffers are refilled while earlier chunks are in flight."""
    from dmrgpp_b200 import plugin
    prob = sb.ladder_problem(total_states=4000, sigma=2.5, seed=9)
    bg = plugin.BatchedGemm.from_problem(prob)
    try:
        ph = bg.setup_profile()
        assert ph["total"] >= ph["upload"] >= ph["upload_fill"] > 0.0 and ph["plan"] > 0.0
        assert ph["mixed"] == 0.0
        x = np.random.default_rng(8).standard_normal(prob.dim)
        assert rel_err(bg(x), oracle_built.kron_apply(prob, x)) < RTOL
    finally:
        bg.close()


@pytest.mark.parametrize("seed,np_,K,maxs", [(31, 4, 3, 30), (32, 7, 5, 12), (33, 1, 1, 1)])
def test_device_diagonal_matches_dense_h(cuda_lib, cuda_device, seed, np_, K, maxs):
    """The create-time diagonal (Jacobi and learned preconditioners) equals
    diag(H) of the explicit sector matrix."""
    import torch
    from dmrgpp_b200 import plugin
    prob = sb.random_problem(npatches=np_, noperator=K, max_size=maxs, seed=seed,
                             zero_block_rate=0.2)
    bg = plugin.BatchedGemm.from_problem(prob)
    try:
        d = bg.diagonal()
        torch.cuda.synchronize()
        ref = np.diag(prob.dense())
        np.testing.assert_allclose(d.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    finally:
        bg.close()


def test_memory_pool_reuses_freed_handles(cuda_lib, cuda_device):
    """A destroyed handle's device memory stays in the library's pool and
    serves the next create of the same size; releasing the cache returns it."""
    from dmrgpp_b200 import plugin
    prob = sb.ladder_problem(total_states=1500, sigma=2.0, seed=3)
    plugin.BatchedGemm.from_problem(prob).close()
    r1, u1 = plugin.cached_memory()
    assert r1 > 0
    bg = plugin.BatchedGemm.from_problem(prob)
    r2, u2 = plugin.cached_memory()
    bg.close()
    assert r2 <= r1 and u2 > u1
    plugin.release_cached_memory()
    r3, u3 = plugin.cached_memory()
    assert u3 <= r3 < r1


def test_large_blocks_are_reused_from_the_free_list(cuda_lib, cuda_device, oracle_built):
    """Blocks of 64 MB and more (here the 8000-state ladder sector's packed
    operators, 134 MB) go to a free list when a handle is destroyed and serve
    the next create of the same sector without the pool growing; they are
    not counted as in use, and releasing the cache returns them."""
    from dmrgpp_b200 import plugin
    prob = sb.ladder_problem(total_states=8000)
    x = np.random.default_rng(4).standard_normal(prob.dim)
    plugin.BatchedGemm.from_problem(prob).close()
    r1, u1 = plugin.cached_memory()
    bg = plugin.BatchedGemm.from_problem(prob)
    r2, u2 = plugin.cached_memory()
    y = bg(x)
    bg.close()
    r3, u3 = plugin.cached_memory()
    assert r2 == r1 and r3 == r1
    assert u2 - u1 >= prob.operator_bytes() and u3 == u1
    assert rel_err(y, oracle_built.kron_apply(prob, x)) < RTOL
    plugin.release_cached_memory()
    r4, _ = plugin.cached_memory()
    assert r4 < r1 - prob.operator_bytes()


@pytest.mark.parametrize("which", ["c2", "ladder", "group"])
def test_page_locked_host_vectors(cuda_lib, cuda_device, oracle_built, which):
    """Page-locked host x and y (copied in and out around the launch): the
    result is bitwise the device-pointer result on a single sector, a larger
    sector and a group handle, and repeated calls agree."""
    import torch
    from dmrgpp_b200 import plugin
    if which == "group":
        probs = [sb.random_problem(npatches=n, noperator=3, max_size=40, seed=50 + n) for n in (2, 5, 7)]
        bg = plugin.BatchedGemm.from_problems(probs)
    else:
        prob = sb.c2_problem() if which == "c2" else sb.ladder_problem(total_states=1500, sigma=2.0, seed=3)
        bg = plugin.BatchedGemm.from_problem(prob)
    try:
        x = np.random.default_rng(12).standard_normal(bg.dim)
        xp = torch.from_numpy(x).pin_memory()
        yp = torch.empty(bg.dim, dtype=torch.float64).pin_memory()
        xd = xp.cuda()
        yd = torch.empty_like(xd)
        bg.apply_Htarget(xd, yd)
        torch.cuda.synchronize()
        ref = yd.cpu().numpy()
        for _ in range(3):
            yp.zero_()
            bg.apply_Htarget(xp.numpy(), yp.numpy())
            assert np.array_equal(yp.numpy(), ref)
        if which == "c2":
            assert rel_err(ref, oracle_built.kron_apply(prob, x)) < RTOL
    finally:
        bg.close()


def test_tuning_cache_hits_across_similar_sectors(cuda_lib, cuda_device, oracle_built, tmp_path):
    """The tuning cache key is a bucketed histogram of the sector's shape:
    a sector whose patches differ by a state or two (as between consecutive
    sweep steps) reuses the first sector's entry; a sector of another shape
    does not."""
    from dmrgpp_b200 import plugin
    sizes = sb.gaussian_sector_sizes(1024, 13, 2.5)
    nearby = sizes.copy()
    nearby[len(sizes) // 2] += 1
    nearby[len(sizes) // 2 + 1] -= 1
    other = sb.gaussian_sector_sizes(4096, 21, 4.0)
    cache = str(tmp_path / "tune.txt")

    def lines():
        return [ln for ln in open(cache).read().split("\n") if ln.strip()]
    for n, (sz, seed) in enumerate(((sizes, 1), (nearby, 2), (other, 3))):
        prob = sb.spin_chain_like(sz, seed=seed)
        bg = plugin.BatchedGemm.from_problem(prob)
        cfg, us = bg.autotune(cache, reps=2)
        x = np.random.default_rng(seed).standard_normal(prob.dim)
        assert rel_err(bg(x), oracle_built.kron_apply(prob, x)) < RTOL
        bg.close()
        assert len(lines()) == (1 if n < 2 else 2), n
