"""Runs a fixed number of H*x applies (or one sector solve) of a named sector
on cuda:0 and nothing else, so that a profiler's launch list and captures see
only the kernels of that workload.

    python -m dmrgpp_b200.profile_case c2 [--precision fp64|tf32x3] [--applies N]
                                          [--config C --ipc I]
    python -m dmrgpp_b200.profile_case ladder --states 4000 --precision tf32x3
    python -m dmrgpp_b200.profile_case ladder --states 4000 --solve lanczos
    python -m dmrgpp_b200.profile_case mlp --elements 300000 [--inference cuda_cores]
    python -m dmrgpp_b200.profile_case wft --states 4000
    python -m dmrgpp_b200.profile_case truncation --states 16000
    python -m dmrgpp_b200.profile_case serving --problems 256

Workloads: c2 = the 1024 x 1024-state, 21-group, K=5 microbench sector;
ladder = the ladder-shaped (N_up, N_down) sector with `--states` left and
right states (K = 10); mlp = learned-preconditioner applications (seeded
network, seeded diagonal and residual of `--elements` entries); wft = the
wave-function transformation of the ladder-shaped layout with seeded square
N(0,1)/sqrt(n) blocks; truncation = the density-matrix truncation of the
ladder-shaped layout's system block (one group per patch) for a seeded unit
sector vector, a quarter of the states kept.  Prints one line "ok ..." at the
end.  serving = the serving-style batch (superblock.serving_batch) in one TF32x3
group handle, solved once as the bench does: group Lanczos to a Ritz-value
change of 1e-5, then the lockstep FP64 group refinement.
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    p = argparse.ArgumentParser()
    p.add_argument("workload", choices=["c2", "ladder", "mlp", "wft", "truncation", "serving"])
    p.add_argument("--problems", type=int, default=256, help="serving: problems in the batch")
    p.add_argument("--elements", type=int, default=300000, help="mlp: vector length")
    p.add_argument("--inference", default="tensor_cores", choices=["tensor_cores", "cuda_cores"])
    p.add_argument("--states", type=int, default=4000, help="ladder: left = right states")
    p.add_argument("--precision", default="fp64", choices=["fp64", "tf32x3"])
    p.add_argument("--applies", type=int, default=6)
    p.add_argument("--config", type=int, default=None, help="FP64 tile configuration")
    p.add_argument("--ipc", type=int, default=2, help="FP64 items per CTA")
    p.add_argument("--solve", default=None, choices=["lanczos"],
                   help="run one FP64 Lanczos solve instead of bare applies")
    p.add_argument("--steps", type=int, default=60)
    a = p.parse_args(argv)

    import torch
    from . import plugin
    from . import superblock as sb

    if a.workload == "mlp":
        import numpy as np
        from .mlp import MLPPreconditioner
        m = MLPPreconditioner(seed=7)
        m.set_inference(m.TENSOR_CORES if a.inference == "tensor_cores" else m.CUDA_CORES)
        rng = np.random.default_rng(0)
        d = torch.tensor(rng.standard_normal(a.elements) * 3, dtype=torch.float64, device="cuda")
        r = torch.tensor(rng.standard_normal(a.elements), dtype=torch.float64, device="cuda")
        rn = float(torch.linalg.vector_norm(r))
        for _ in range(a.applies):
            t = m.precondition(d, r, -1.7, rn)
        torch.cuda.synchronize()
        print("ok", a.elements, float(t.abs().max()))
        m.close()
        return 0

    if a.workload == "wft":
        import numpy as np
        from .wft import WaveFunctionTransform
        prob = sb.ladder_problem(total_states=a.states, sigma=2.5, seed=9)
        rng = np.random.default_rng(17)
        l, r = prob.lsz, prob.rsz
        WL = [rng.standard_normal((int(n), int(n))) / np.sqrt(n) for n in l]
        WR = [rng.standard_normal((int(n), int(n))) / np.sqrt(n) for n in r]
        w = WaveFunctionTransform(l, r, l, r, list(range(prob.npatches)), WL, WR)
        x = torch.from_numpy(rng.standard_normal(w.dim_in)).cuda()
        y = torch.empty(w.dim_out, dtype=torch.float64, device="cuda")
        for _ in range(a.applies):
            w(x, y)
        torch.cuda.synchronize()
        print("ok", w.dim_in, w.flops, float(y.norm()))
        w.close()
        return 0

    if a.workload == "serving":
        import numpy as np
        probs, _ = sb.serving_batch(a.problems)
        bg = plugin.BatchedGemm.from_problems(probs, precision=plugin.TF32X3)
        init = torch.from_numpy(np.random.default_rng(1).standard_normal(bg.dim)).cuda()
        _, z, steps = bg.lanczos_lowest_group(init, steps=200, tolerance=1e-5)
        e, conv, st = bg.refine_lowest_group(z, max_outer=10, tolerance=1e-10, inner_iterations=80,
                                             inner_tolerance=1e-2, raise_on_no_convergence=False)
        torch.cuda.synchronize()
        print("ok", bg.dim, int(steps.max()), int(conv.sum()), st["inner_matvecs"])
        bg.close()
        return 0

    if a.workload == "truncation":
        import numpy as np
        from .truncation import density_truncate
        prob = sb.ladder_problem(total_states=a.states, sigma=2.5, seed=9)
        l, r = prob.lsz, prob.rsz
        psi = torch.from_numpy(sb.random_unit_vector(prob.dim)).cuda()
        for _ in range(a.applies):
            out = density_truncate(l, r, list(range(prob.npatches)), l, 0, psi, a.states // 4)
        torch.cuda.synchronize()
        print("ok", prob.dim, out["kept_total"], out["discarded"])
        return 0

    prob = (sb.c2_problem() if a.workload == "c2"
            else sb.ladder_problem(total_states=a.states, sigma=2.5, seed=9))
    prec = plugin.TF32X3 if a.precision == "tf32x3" else plugin.FP64
    s = torch.cuda.Stream()
    torch.cuda.set_stream(s)
    bg = plugin.BatchedGemm.from_problem(prob, stream=s.cuda_stream, precision=prec)
    if prec == plugin.FP64 and a.config is not None:
        bg.set_config(a.config, a.ipc)
    x = torch.from_numpy(sb.random_unit_vector(prob.dim)).cuda()
    y = torch.empty_like(x)
    if a.solve == "lanczos":
        e, z, n = bg.lanczos_lowest(x, steps=a.steps, tolerance=1e-12)
        y = z
        print("E", e, "steps", n)
    else:
        for _ in range(a.applies):
            bg.apply_Htarget(x, y)
    torch.cuda.synchronize()
    print("ok", prob.dim, prob.flops(), float(y.norm()))
    bg.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
