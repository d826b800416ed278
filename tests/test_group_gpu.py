"""Many independent sectors in one handle (dmrgpp_kron_create_group) and the
lockstep group Lanczos (dmrgpp_lanczos_lowest_group), through the C ABI.

H*x of a group is checked sector by sector against the oracle (1e-12, the
FP64 bar); group Lanczos energies against the single-sector device Lanczos
and, for small sectors, dense diagonalisation."""
import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def rel_err(y, ref):
    return float(np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300))


def mixed_sectors():
    return [sb.random_problem(npatches=5, noperator=3, max_size=40, seed=1, symmetric=True),
            sb.c2_problem(seed=5),
            sb.random_problem(npatches=1, noperator=1, max_size=1, seed=2, symmetric=True),
            sb.ladder_problem(total_states=600, sigma=1.5, seed=3, legs=1),
            sb.random_problem(npatches=3, noperator=2, max_size=2, min_size=1, seed=4,
                              symmetric=True),
            sb.spin_chain_like(sb.gaussian_sector_sizes(128, 7, 1.4), seed=6)]


def test_group_apply_matches_oracle_per_sector(cuda_lib, cuda_device, oracle_built):
    from dmrgpp_b200 import plugin
    probs = mixed_sectors()
    bg = plugin.BatchedGemm.from_problems(probs)
    offs = bg.sector_offsets()
    assert len(offs) == len(probs) + 1 and offs[-1] == bg.dim
    assert abs(bg.f_alg - sum(p.flops() for p in probs)) < 1e-6 * bg.f_alg
    x = np.random.default_rng(0).standard_normal(bg.dim)
    y = bg(x)
    for s, p in enumerate(probs):
        xs = x[offs[s]:offs[s + 1]]
        assert rel_err(y[offs[s]:offs[s + 1]], oracle_built.kron_apply(p, xs)) < RTOL, s
    assert np.array_equal(bg(x), y)            # bitwise reproducible
    bg.close()


def test_group_lanczos_matches_single_sector_solves(cuda_lib, cuda_device):
    from dmrgpp_b200 import plugin
    probs = mixed_sectors()
    bg = plugin.BatchedGemm.from_problems(probs)
    offs = bg.sector_offsets()
    init = np.random.default_rng(11).standard_normal(bg.dim)
    e, z, steps = bg.lanczos_lowest_group(init, steps=200, tolerance=1e-12)
    for s, p in enumerate(probs):
        xs = init[offs[s]:offs[s + 1]]
        single = plugin.BatchedGemm.from_problem(p)
        e1, z1, n1 = single.lanczos_lowest(xs, steps=200, tolerance=1e-12)
        single.close()
        assert abs(e[s] - e1) <= 1e-11 * max(1.0, abs(e1)), (s, e[s], e1)
        zs = z[offs[s]:offs[s + 1]]
        assert abs(np.linalg.norm(zs) - 1.0) < 1e-10
        assert 1.0 - abs(float(zs @ z1)) < 1e-8, s
        if p.dim <= 2000:
            exact = np.linalg.eigvalsh(p.dense())[0]
            assert abs(e[s] - exact) <= 1e-11 * max(1.0, abs(exact)), (s, e[s], exact)
        assert 0 <= steps[s] < max(p.dim, 1) and steps[s] <= 200
    bg.close()


def test_group_lanczos_device_vectors_and_one_sector_group(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200 import plugin
    p = sb.c2_problem(seed=8)
    g = plugin.BatchedGemm.from_problems([p])
    assert list(g.sector_offsets()) == [0, p.dim]
    init = torch.from_numpy(np.random.default_rng(3).standard_normal(p.dim)).cuda()
    e, z, steps = g.lanczos_lowest_group(init, steps=200)
    single = plugin.BatchedGemm.from_problem(p)
    e1, z1, n1 = single.lanczos_lowest(init, steps=200)
    assert isinstance(z, torch.Tensor) and z.is_cuda
    assert abs(e[0] - e1) <= 1e-11 * abs(e1)
    assert 1.0 - abs(float(torch.dot(z, z1))) < 1e-9
    g.close()
    single.close()


def test_serving_batch_subset(cuda_lib, cuda_device):
    """Eight problems of the serving-style batch: group energies equal the
    single-problem FP64 solves."""
    from dmrgpp_b200 import plugin
    probs, meta = sb.serving_batch(8, seed=77)
    bg = plugin.BatchedGemm.from_problems(probs)
    offs = bg.sector_offsets()
    init = np.random.default_rng(5).standard_normal(bg.dim)
    e, z, steps = bg.lanczos_lowest_group(init)
    for s, p in enumerate(probs):
        single = plugin.BatchedGemm.from_problem(p)
        e1, _, _ = single.lanczos_lowest(init[offs[s]:offs[s + 1]])
        single.close()
        assert abs(e[s] - e1) <= 1e-11 * max(1.0, abs(e1)), (meta[s], e[s], e1)
    bg.close()


def test_group_apply_in_tf32x3(cuda_lib, cuda_device, oracle_built):
    """A group created in TF32x3: the union's tensor-core plan applies every
    sector within the mixed-precision bar (2e-5) of the oracle."""
    from dmrgpp_b200 import plugin
    probs = mixed_sectors()
    bg = plugin.BatchedGemm.from_problems(probs, precision=plugin.TF32X3)
    offs = bg.sector_offsets()
    x = np.random.default_rng(3).standard_normal(bg.dim)
    y = bg(x)
    for s, p in enumerate(probs):
        ref = oracle_built.kron_apply(p, x[offs[s]:offs[s + 1]])
        assert rel_err(y[offs[s]:offs[s + 1]], ref) < 2e-5, s
    bg.close()


def test_group_handle_as_one_sector_with_graph_replay(cuda_lib, cuda_device):
    """The single-sector Lanczos on a group handle treats the union as one
    block-diagonal sector: its lowest energy is the lowest over the sectors,
    and the CUDA-graph form is bitwise identical to launch by launch."""
    import torch
    from dmrgpp_b200 import plugin
    probs = [sb.random_problem(npatches=4, noperator=2, max_size=20, seed=s, symmetric=True)
             for s in (5, 6, 7)]
    bg = plugin.BatchedGemm.from_problems(probs)
    init = torch.from_numpy(np.random.default_rng(9).standard_normal(bg.dim)).cuda()
    e0, z0, n0 = bg.lanczos_lowest(init, steps=300, use_graph=False)
    e1, z1, n1 = bg.lanczos_lowest(init, steps=300, use_graph=True)
    assert e0 == e1 and n0 == n1 and torch.equal(z0, z1)
    exact = min(np.linalg.eigvalsh(p.dense())[0] for p in probs)
    assert abs(e0 - exact) <= 1e-10 * abs(exact)
    bg.close()


@pytest.mark.parametrize("precision,reortho,jacobi", [("tf32x3", True, False), ("tf32x3", False, False),
                                                     ("fp64", True, False), ("tf32x3", False, True)])
def test_group_refinement_matches_single_fp64_solves(cuda_lib, cuda_device, precision, reortho, jacobi):
    """Serving-style problems in one group handle: a loose lockstep group
    Lanczos (the handle's matvecs: tensor-core TF32x3 or FP64; with or without
    reorthogonalisation, as the start vectors only), then the
    lockstep FP64 refinement (dmrgpp_refine_lowest_group).  Every sector
    converges; its energy is within 1e-9 per site (and 1e-10 relative) of its
    single-problem FP64 Lanczos, its vector has unit norm and overlaps the
    FP64 Ritz vector to 1e-8.  Also with the diagonally preconditioned
    correction solves (dmrgpp_set_correction_preconditioner)."""
    import torch
    from dmrgpp_b200 import _capi, plugin
    probs, meta = sb.serving_batch(8, seed=77)
    prec = plugin.TF32X3 if precision == "tf32x3" else plugin.FP64
    bg = plugin.BatchedGemm.from_problems(probs, precision=prec)
    if jacobi:
        bg.set_correction_preconditioner(_capi.PRECOND_JACOBI)
    offs = bg.sector_offsets()
    init = torch.from_numpy(np.random.default_rng(5).standard_normal(bg.dim)).cuda()
    _, z, _ = bg.lanczos_lowest_group(init, steps=100, tolerance=1e-4, reortho=reortho)
    e, conv, st = bg.refine_lowest_group(z, max_outer=8, tolerance=1e-10, inner_iterations=80,
                                         inner_tolerance=1e-2)
    assert conv.all() and st["converged"] == 1 and st["fp64_matvecs"] >= 1
    for s, p in enumerate(probs):
        single = plugin.BatchedGemm.from_problem(p)
        e1, z1, _ = single.lanczos_lowest(init[offs[s]:offs[s + 1]].contiguous(), tolerance=1e-12)
        single.close()
        assert abs(e[s] - e1) / meta[s]["L"] <= 1e-9, (meta[s], e[s], e1)
        assert abs(e[s] - e1) <= 1e-10 * abs(e1), (meta[s], e[s], e1)
        zs = z[offs[s]:offs[s + 1]]
        assert abs(float(torch.linalg.norm(zs)) - 1.0) < 1e-12
        assert 1.0 - abs(float(torch.dot(zs, z1))) < 1e-8, s
    bg.close()


def test_group_refinement_edge_sectors(cuda_lib, cuda_device):
    """Uneven sectors (one of dimension 1, tiny ones, C2) refined from random
    vectors in a TF32x3 group: the 1-state sector converges at once, the
    others reach the dense-diagonalisation energies; with max_outer = 0 only
    the Rayleigh quotients are formed and unconverged sectors are reported."""
    import torch
    from dmrgpp_b200 import plugin
    probs = mixed_sectors()
    bg = plugin.BatchedGemm.from_problems(probs, precision=plugin.TF32X3)
    offs = bg.sector_offsets()
    x = torch.from_numpy(np.random.default_rng(21).standard_normal(bg.dim)).cuda()
    e0, conv0, st0 = bg.refine_lowest_group(x.clone(), max_outer=0, raise_on_no_convergence=False)
    assert st0["inner_matvecs"] == 0 and st0["fp64_matvecs"] == 1
    assert conv0[2] and not conv0.all()
    for s, p in enumerate(probs):
        xs = x[offs[s]:offs[s + 1]].cpu().numpy()
        rq = float(xs @ (p.dense() @ xs) / (xs @ xs)) if p.dim <= 2000 else None
        if rq is not None:
            assert abs(e0[s] - rq) <= 1e-12 * max(1.0, abs(rq)), s
    _, z, _ = bg.lanczos_lowest_group(x, steps=150, tolerance=1e-5)
    e, conv, st = bg.refine_lowest_group(z, max_outer=12, tolerance=1e-10, inner_iterations=150,
                                         inner_tolerance=1e-3)
    assert conv.all()
    for s, p in enumerate(probs):
        if p.dim <= 2000:
            exact = np.linalg.eigvalsh(p.dense())[0]
            assert abs(e[s] - exact) <= 1e-10 * max(1.0, abs(exact)), (s, e[s], exact)
    bg.close()


def test_group_lanczos_reuses_larger_work_buffers(cuda_lib, cuda_device):
    """A group solve with fewer steps after one with more reuses the larger
    work buffers: same energies and Ritz vectors (bitwise) as on a fresh
    handle."""
    import torch
    from dmrgpp_b200 import plugin
    probs, _ = sb.serving_batch(6, seed=13)
    bg = plugin.BatchedGemm.from_problems(probs)
    init = torch.from_numpy(np.random.default_rng(2).standard_normal(bg.dim)).cuda()
    bg.lanczos_lowest_group(init, steps=200)
    e1, z1, n1 = bg.lanczos_lowest_group(init, steps=40)
    bg.close()
    fresh = plugin.BatchedGemm.from_problems(probs)
    e2, z2, n2 = fresh.lanczos_lowest_group(init, steps=40)
    fresh.close()
    assert np.array_equal(e1, e2) and np.array_equal(n1, n2)
    assert torch.equal(z1, z2)


@pytest.mark.parametrize("tolerance", [1e-10, 1e-17])
def test_solve_lowest_group_with_fallback(cuda_lib, cuda_device, tolerance):
    """The library's group solve (TF32x3 group Lanczos, lockstep FP64
    refinement with Jacobi correction solves, FP64 group Lanczos for the
    sectors left unconverged) on serving-style problems: energies within
    1e-9 per site of single-problem FP64 Lanczos.  With an unreachable
    refinement tolerance (1e-17) every sector takes the FP64 fallback."""
    import torch
    from dmrgpp_b200 import plugin
    probs, meta = sb.serving_batch(8, seed=77)
    bg = plugin.BatchedGemm.from_problems(probs, precision=plugin.TF32X3)
    offs = bg.sector_offsets()
    init = torch.from_numpy(np.random.default_rng(5).standard_normal(bg.dim)).cuda()
    e, z, st = bg.solve_lowest_group(init, tolerance=tolerance)
    assert bg.get_precision() == plugin.TF32X3
    bg.close()
    if tolerance < 1e-16:
        assert st["fallbacks"] == len(probs)
    for s, p in enumerate(probs):
        single = plugin.BatchedGemm.from_problem(p)
        e1, z1, _ = single.lanczos_lowest(init[offs[s]:offs[s + 1]].contiguous(), tolerance=1e-12)
        single.close()
        assert abs(e[s] - e1) / meta[s]["L"] <= 1e-9, (meta[s], e[s], e1, st["fallbacks"])
        zs = z[offs[s]:offs[s + 1]]
        assert 1.0 - abs(float(torch.dot(zs, z1))) < 1e-6, s


def test_masked_group_lanczos(cuda_lib, cuda_device):
    """dmrgpp_lanczos_lowest_group_masked: the sectors in the mask get the
    energies and vectors of the unmasked solve (each sector's arithmetic does
    not depend on the others); the rest get NaN and zeros."""
    import torch
    from dmrgpp_b200 import plugin
    probs, meta = sb.serving_batch(8, seed=78)
    bg = plugin.BatchedGemm.from_problems(probs)
    offs = bg.sector_offsets()
    init = torch.from_numpy(np.random.default_rng(6).standard_normal(bg.dim)).cuda()
    e_all, z_all, n_all = bg.lanczos_lowest_group(init, steps=200, tolerance=1e-12)
    mask = np.zeros(len(probs), dtype=bool)
    mask[[1, 4]] = True
    e_m, z_m, n_m = bg.lanczos_lowest_group(init, steps=200, tolerance=1e-12, mask=mask)
    bg.close()
    for s in range(len(probs)):
        zs = z_m[offs[s]:offs[s + 1]]
        if mask[s]:
            assert abs(e_m[s] - e_all[s]) <= 1e-13 * abs(e_all[s]), s
            assert n_m[s] == n_all[s]
            assert float(torch.linalg.vector_norm(zs - z_all[offs[s]:offs[s + 1]])) <= 1e-10
        else:
            assert np.isnan(e_m[s]) and n_m[s] == 0
            assert float(torch.abs(zs).max()) == 0.0
