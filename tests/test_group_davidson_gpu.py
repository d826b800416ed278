"""The lockstep group Davidson (dmrgpp_davidson_lowest_group) and the
learned correction of a group of sectors (dmrgpp_mlp_precondition_group),
through the C ABI: per-sector results against the single-sector solvers and
the FP64 Lanczos energies, in FP64 and with TF32x3 matvecs followed by the
group FP64 refinement."""
import os

import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dmrgpp_b200",
                       "weights", "serving_mlp.npz")


def _group_problems():
    probs, meta = sb.serving_batch(6, seed=31)
    one = sb.random_problem(npatches=1, noperator=1, max_size=1, seed=2, symmetric=True)
    small = sb.random_problem(npatches=3, noperator=2, max_size=4, min_size=1, seed=4, symmetric=True)
    return probs + [one, small], [m["L"] for m in meta] + [1, 1]


@pytest.mark.parametrize("mode", ["tensor_cores", "cuda_cores"])
def test_mlp_group_correction_equals_per_sector(cuda_lib, cuda_device, mode):
    """Each sector's slice of the group correction is bitwise the
    single-sector correction with that sector's Ritz value and residual norm."""
    import torch
    from dmrgpp_b200.mlp import MLPPreconditioner
    m = MLPPreconditioner.load(WEIGHTS)
    m.set_inference(MLPPreconditioner.TENSOR_CORES if mode == "tensor_cores"
                    else MLPPreconditioner.CUDA_CORES)
    rng = np.random.default_rng(3)
    sizes = [1, 700, 128 * 5, 3001, 129]
    starts = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    n = int(starts[-1])
    d = torch.tensor(rng.standard_normal(n) * 4, dtype=torch.float64, device="cuda")
    r = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device="cuda")
    theta = torch.tensor(rng.uniform(-30, 5, len(sizes)), dtype=torch.float64, device="cuda")
    rnorm = torch.tensor([float(torch.linalg.vector_norm(r[starts[s]:starts[s + 1]]))
                          for s in range(len(sizes))], dtype=torch.float64, device="cuda")
    t = m.precondition_group(d, r, torch.tensor(starts, device="cuda"), theta, rnorm)
    for s in range(len(sizes)):
        a, b = int(starts[s]), int(starts[s + 1])
        ts = m.precondition(d[a:b].contiguous(), r[a:b].contiguous(), float(theta[s]),
                            float(rnorm[s]))
        torch.cuda.synchronize()
        assert torch.equal(t[a:b], ts), s
    m.close()


@pytest.mark.parametrize("pre", [0, 1, 2])
def test_group_davidson_matches_single_sector_solves(cuda_lib, cuda_device, pre):
    """FP64 group Davidson with no, Jacobi and the learned preconditioner:
    every sector converges (the 1-state sector at once), energies within
    1e-10 of the single-sector FP64 Lanczos and of the single-sector Davidson
    with the same preconditioner, unit Ritz vectors."""
    import torch
    from dmrgpp_b200 import plugin
    from dmrgpp_b200.mlp import MLPPreconditioner
    probs, _ = _group_problems()
    mlp = MLPPreconditioner.load(WEIGHTS) if pre == 2 else None
    bg = plugin.BatchedGemm.from_problems(probs)
    offs = bg.sector_offsets()
    init = torch.from_numpy(np.random.default_rng(8).standard_normal(bg.dim)).cuda()
    e, z, conv, st = bg.davidson_lowest_group(init, preconditioner=pre, mlp=mlp, tolerance=1e-9,
                                              max_iterations=1500, max_subspace=32)
    assert conv.all() and st["converged"] == 1 and st["fp64_matvecs"] == st["iterations"]
    for s, p in enumerate(probs):
        xs = init[offs[s]:offs[s + 1]].contiguous()
        single = plugin.BatchedGemm.from_problem(p)
        e1, _, _ = single.lanczos_lowest(xs, tolerance=1e-13)
        e2, _, st2 = single.davidson_lowest(xs, preconditioner=pre, mlp=mlp, tolerance=1e-9,
                                            max_iterations=1500, max_subspace=32)
        single.close()
        assert abs(e[s] - e1) <= 1e-10 * max(1.0, abs(e1)), (s, e[s], e1)
        assert abs(e[s] - e2) <= 1e-10 * max(1.0, abs(e1)), (s, e[s], e2)
        zs = z[offs[s]:offs[s + 1]]
        assert abs(float(torch.linalg.vector_norm(zs)) - 1.0) < 1e-12
    bg.close()
    if mlp is not None:
        mlp.close()


def test_group_davidson_learned_in_tf32x3_then_refinement(cuda_lib, cuda_device):
    """The serving form: TF32x3 group matvecs and the learned correction to a
    loose residual, then the lockstep FP64 refinement: every sector within
    1e-9 per site of its single-problem FP64 Lanczos."""
    import torch
    from dmrgpp_b200 import plugin
    from dmrgpp_b200.mlp import MLPPreconditioner
    probs, sites = _group_problems()
    mlp = MLPPreconditioner.load(WEIGHTS)
    bg = plugin.BatchedGemm.from_problems(probs, precision=plugin.TF32X3)
    offs = bg.sector_offsets()
    init = torch.from_numpy(np.random.default_rng(9).standard_normal(bg.dim)).cuda()
    _, z, conv, st = bg.davidson_lowest_group(init, preconditioner=2, mlp=mlp, tolerance=1e-5,
                                              max_iterations=800, max_subspace=32)
    assert conv.all() and st["mixed_matvecs"] == st["iterations"] and st["fp64_matvecs"] == 0
    e, rconv, rst = bg.refine_lowest_group(z, max_outer=10, tolerance=1e-10, inner_iterations=80,
                                           inner_tolerance=1e-2)
    assert rconv.all()
    for s, p in enumerate(probs):
        single = plugin.BatchedGemm.from_problem(p)
        e1, _, _ = single.lanczos_lowest(init[offs[s]:offs[s + 1]].contiguous(), tolerance=1e-13)
        single.close()
        assert abs(e[s] - e1) / sites[s] <= 1e-9, (s, e[s], e1)
    bg.close()
    mlp.close()


def test_group_davidson_argument_checks(cuda_lib, cuda_device):
    from dmrgpp_b200 import _capi, plugin
    probs, _ = _group_problems()
    bg = plugin.BatchedGemm.from_problems(probs[:2])
    x = np.ones(bg.dim)
    for kw in ({"max_subspace": 129}, {"max_subspace": 1}, {"preconditioner": 2}):
        with pytest.raises(_capi.DmrgppError) as ei:
            bg.davidson_lowest_group(x, **kw)
        assert ei.value.status == _capi.INVALID_ARG
    bg.close()
