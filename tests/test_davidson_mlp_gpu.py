"""Davidson, the FP64 refinement of the mixed-precision mode, and the learned
preconditioner: gradients against the FP64 oracle, training, and an ablation
of what the trained network gains.  (No counterpart in the reference;
convergence is decided by the FP64 residual, and energies are checked
against the reference Lanczos.)"""
import json
import os

import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _start(prob, seed=2024):
    return np.random.default_rng(seed).standard_normal(prob.dim)


@pytest.mark.parametrize("pre", [0, 1])
def test_davidson_matches_reference_lanczos_energy(cuda_lib, cuda_device, oracle_built, pre):
    from dmrgpp_b200 import plugin
    g = json.load(open(os.path.join(GOLDEN, "lanczos_reference.json")))["microbench_1024"]
    prob = sb.c2_problem()
    bg = plugin.BatchedGemm.from_problem(prob)
    e, z, st = bg.davidson_lowest(_start(prob), preconditioner=pre, tolerance=1e-9,
                                  max_iterations=2000)
    assert st["converged"] == 1
    assert abs(e - g["energy"]) <= 1e-11 * abs(g["energy"]), (e, g["energy"])
    hz = oracle_built.kron_apply(prob, z)
    assert np.linalg.norm(hz - e * z) <= 1e-9 * 1.0e1 * abs(e)
    bg.close()


def test_mixed_precision_davidson_with_fp64_refinement(cuda_lib, cuda_device, oracle_built):
    """TF32x3 matvecs for most of the solve, FP64 for the end: the energy
    agrees with the FP64 oracle pair to far below 1e-9 per site."""
    from dmrgpp_b200 import plugin
    g = json.load(open(os.path.join(GOLDEN, "lanczos_reference.json")))["microbench_1024"]
    prob = sb.c2_problem()
    bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
    e, z, st = bg.davidson_lowest(_start(prob), preconditioner=1, tolerance=1e-9,
                                  max_iterations=2000)
    assert st["converged"] == 1 and st["mixed_matvecs"] > 0 and st["fp64_matvecs"] > 0
    assert abs(e - g["energy"]) <= 1e-11 * abs(g["energy"])
    ov = abs(float(z @ oracle_built.RefKron(prob).lanczos(_start(prob))[1])) if oracle_built.ref_available() else 1.0
    assert 1.0 - ov < 1e-9
    bg.close()


def test_mlp_gradients_match_fp64_oracle(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200.mlp import MLPPreconditioner
    from oracle import mlp_oracle
    rng = np.random.default_rng(0)
    m = MLPPreconditioner(seed=3)
    p = m.get_params().astype(np.float64)
    rows = 1000
    x = rng.standard_normal((rows, 4))
    y = rng.standard_normal(rows)
    xd = torch.tensor(x, dtype=torch.float32, device="cuda")
    yd = torch.tensor(y, dtype=torch.float32, device="cuda")
    out = m.forward(xd)
    loss = m.backward(xd, yd)
    g = m.get_grads().astype(np.float64)
    x32 = x.astype(np.float32).astype(np.float64)
    y32 = y.astype(np.float32).astype(np.float64)
    o_ref, _ = mlp_oracle.forward(p, x32)
    loss_ref, g_ref = mlp_oracle.loss_and_grads(p, x32, y32)
    assert np.abs(out.cpu().numpy() - o_ref).max() < 1e-4 * max(1, np.abs(o_ref).max())
    assert abs(loss - loss_ref) < 1e-5 * loss_ref
    scale = np.abs(g_ref).max()
    assert np.abs(g - g_ref).max() < 1e-4 * scale
    # finite-difference check of the oracle itself on a few coordinates
    for k in [5, 1500, 40000, m.n_params - 1]:
        q = p.copy()
        q[k] += 1e-6
        lp, _ = mlp_oracle.loss_and_grads(q, x32, y32)
        q[k] -= 2e-6
        lm, _ = mlp_oracle.loss_and_grads(q, x32, y32)
        assert abs((lp - lm) / 2e-6 - g_ref[k]) < 1e-6 + 1e-4 * abs(g_ref[k])
    m.close()


def test_mlp_inference_uses_bf16_weights(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200.mlp import MLPPreconditioner
    from oracle import mlp_oracle
    rng = np.random.default_rng(1)
    m = MLPPreconditioner(seed=5)
    m.set_inference(MLPPreconditioner.CUDA_CORES)
    p = m.get_params()
    pb = torch.tensor(p).to(torch.bfloat16).to(torch.float64).numpy()
    n = 5000
    d = torch.tensor(rng.standard_normal(n) * 3, dtype=torch.float64, device="cuda")
    r = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device="cuda")
    theta, rn = -1.7, float(torch.linalg.vector_norm(r))
    t = m.precondition(d, r, theta, rn)
    torch.cuda.synchronize()
    x = mlp_oracle.features(d.cpu().numpy(), r.cpu().numpy(), theta, rn)
    o, _ = mlp_oracle.forward(pb, x.astype(np.float32).astype(np.float64))
    t_ref = o * (rn / np.sqrt(n)) / max(1.0, abs(theta))
    assert np.abs(t.cpu().numpy() - t_ref).max() < 2e-4 * np.abs(t_ref).max()
    m.close()


@pytest.mark.parametrize("n", [5000, 128 * 37 + 1, 1, 300_000])
def test_mlp_tensor_core_inference(cuda_lib, cuda_device, n):
    """The fused tcgen05 inference (BF16 weights and first hidden layer,
    BF16 MMAs with FP32 accumulation in tensor memory, SFU tanh) against the
    FP64 oracle with the same BF16 roundings, and against the CUDA-core path;
    ragged last tiles and more tiles than SMs included; reproducible."""
    import torch
    from dmrgpp_b200.mlp import MLPPreconditioner
    from oracle import mlp_oracle
    rng = np.random.default_rng(n)
    m = MLPPreconditioner(seed=7)
    p = m.get_params()
    p[:] = p * 1.5 + rng.normal(0.0, 0.1, p.shape)   # biases away from zero too
    m.set_params(p.astype(np.float32))
    pb = mlp_oracle.to_bf16(m.get_params())
    d = torch.tensor(rng.standard_normal(n) * 3, dtype=torch.float64, device="cuda")
    r = torch.tensor(rng.standard_normal(n), dtype=torch.float64, device="cuda")
    theta, rn = -1.7, float(torch.linalg.vector_norm(r))
    t1 = m.precondition(d, r, theta, rn)
    t2 = m.precondition(d, r, theta, rn)
    m.set_inference(MLPPreconditioner.CUDA_CORES)
    tc = m.precondition(d, r, theta, rn)
    torch.cuda.synchronize()
    assert torch.equal(t1, t2)
    x = m.features(d, r, theta, rn).double().cpu().numpy()
    o, _ = mlp_oracle.forward(pb, x, bf16_hidden=True)
    t_ref = o * (rn / np.sqrt(n)) / max(1.0, abs(theta))
    scale = np.abs(t_ref).max()
    assert np.abs(t1.cpu().numpy() - t_ref).max() < 1e-2 * scale
    assert np.abs(t1.cpu().numpy() - tc.cpu().numpy()).max() < 2e-2 * scale
    m.close()


def _family(name, seed):
    sizes = sb.gaussian_sector_sizes(256, 13, 2.5)
    if name == "random":
        return sb.spin_chain_like(sizes, seed=seed)
    return sb.spin_chain_dominant(sizes, seed=seed)


@pytest.mark.parametrize("family", ["random", "dominant"])
def test_learned_preconditioner_training_and_ablation(cuda_lib, cuda_device, family):
    """Train on solver-generated exact corrections of small spin-chain-like
    sectors; on held-out sectors count Davidson iterations to the same FP64
    residual with no preconditioner, the diagonal (Jacobi) one and the
    learned one.  The learned correction must do at least as well as the
    Jacobi-preconditioned Davidson it is meant to improve, and never lose
    more than 5% to the better of the two local rules."""
    import torch
    from dmrgpp_b200 import plugin
    from dmrgpp_b200.mlp import MLPPreconditioner, correction_pairs, train
    torch.manual_seed(0)
    Xs, Ys, infos = [], [], []
    for seed in range(4):
        prob = _family(family, 100 + seed)
        bg = plugin.BatchedGemm.from_problem(prob)
        init = torch.tensor(_start(prob, seed), device="cuda")
        for x, y, info in correction_pairs(bg, init):
            Xs.append(x)
            Ys.append(y)
            infos.append(info)
        bg.close()
    print(family, "cos(exact correction, Jacobi | residual):",
          [(round(i["cos_jacobi"], 3), round(i["cos_residual"], 3)) for i in infos])
    X = torch.cat(Xs)
    Y = torch.cat(Ys).clamp(-20, 20)
    m = MLPPreconditioner(seed=11)
    losses = train(m, X, Y, steps=400, batch=8192, lr=2e-3)
    print(family, "loss first/last:", np.mean(losses[:20]), np.mean(losses[-20:]))
    assert np.mean(losses[-20:]) < 0.9 * np.mean(losses[:20])

    its = {0: [], 1: [], 2: []}
    for seed in range(3):
        prob = _family(family, 500 + seed)
        bg = plugin.BatchedGemm.from_problem(prob)
        exact = np.linalg.eigvalsh(prob.dense())[0]
        for pre in (0, 1, 2):
            e, z, st = bg.davidson_lowest(_start(prob, seed), preconditioner=pre,
                                          mlp=m if pre == 2 else None, tolerance=1e-8,
                                          max_iterations=3000, raise_on_no_convergence=False)
            assert st["converged"] == 1, (pre, st)
            assert abs(e - exact) < 1e-10 * abs(exact)
            its[pre].append(st["iterations"])
        bg.close()
    summary = {k: float(np.mean(v)) for k, v in its.items()}
    print(family, "Davidson iterations (none, Jacobi, learned):", summary)
    out_dir = os.environ.get("DMRGPP_ABLATION_OUT")   # optional record of the ablation
    if out_dir and os.path.isdir(out_dir):
        with open(os.path.join(out_dir, f"mlp_ablation_{family}.json"), "w") as f:
            json.dump({"iterations": its, "mean": summary}, f)
    assert summary[2] <= summary[1]
    assert summary[2] <= 1.05 * min(summary[0], summary[1])
    m.close()
