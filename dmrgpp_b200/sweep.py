"""Sector eigensolves as they occur in one finite-sweep step, timed on the
device: the plain FP64 method (Lanczos with full reorthogonalisation, the
reference's PsimagLite::LanczosSolver configuration) against FP64 Davidson
and the mixed-precision solve (TF32x3 Lanczos, then the FP64 refinement),
from a random and from a warm start, and the attribution of the mixed
solve's gain to its scheme and its precision.  Energies are compared per
site and states by overlap."""
from __future__ import annotations

import time
from typing import Dict

import numpy as np

from . import plugin


def _timed(fn):
    import torch
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    a.record()
    out = fn()
    b.record()
    b.synchronize()
    return out, a.elapsed_time(b) / 1e3, time.perf_counter() - t0


def sector_solves(prob, sites: int, mlp=None, seed: int = 7, lanczos_steps: int = 300,
                  tolerance: float = 1e-9, mixed_steps: int = 60,
                  refine_inner: int = 80, refine_inner_tolerance: float = 1e-2,
                  with_davidson: bool = True, mixed_reortho: bool = False) -> Dict:
    """Lowest state of one sector by
      fp64_lanczos           -- the plain method: FP64 Lanczos, full reorthogonalisation,
                                eigenvalue-change tolerance 1e-12 (reference defaults);
      fp64_davidson          -- FP64 Davidson, Jacobi correction, |r| <= tolerance |E|
                                (the converged FP64 pair the others are compared with);
      mixed_lanczos_refined  -- TF32x3 Lanczos (FP64 recurrence; reorthogonalisation only
                                with mixed_reortho: this phase only supplies the start
                                vector) for mixed_steps steps, then FP64 Rayleigh-quotient
                                and residual refinement with TF32x3 correction solves;
      mixed_davidson         -- TF32x3 Davidson with the learned (or Jacobi)
                                correction, FP64 restart phase.
    Seconds are device time around each whole solve (host work included);
    setup_seconds is the handle creation of each form (plan, packing and
    upload: the plugin constructor a sweep step also pays), and
    speedup_with_setup compares setup + solve of the two forms."""
    import torch
    init = torch.from_numpy(np.random.default_rng(seed).standard_normal(prob.dim)).cuda()
    # steady state of a sweep: the previous step's handle and solver buffers
    # have gone back to the library's memory pool and the pinned staging
    # buffers exist.  Stand-in: one untimed create of the same sector with a
    # few Lanczos steps sized for lanczos_steps (the basis is allocated for
    # the step limit) and one Davidson iteration (its subspace buffers), then
    # destroyed.
    warm = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
    warm.set_precision(plugin.FP64)
    warm.lanczos_lowest(init, steps=lanczos_steps, min_steps=2, tolerance=1e300)
    warm.davidson_lowest(init, preconditioner=1, tolerance=1e300, max_iterations=1,
                         raise_on_no_convergence=False)
    warm.close()
    pool_before = plugin.cached_memory()[0]
    b64 = plugin.BatchedGemm.from_problem(prob, precision=plugin.FP64)
    setup_fp64, phases_fp64 = b64.create_seconds, b64.setup_profile()
    b64.close()
    bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
    setup_mixed, phases_mixed = bg.create_seconds, bg.setup_profile()
    out = {"sector_dim": prob.dim, "f_alg_per_matvec": prob.flops(), "sites": sites,
           "setup_seconds": {"fp64": setup_fp64, "tf32x3": setup_mixed},
           "setup_phases": {"fp64": phases_fp64, "tf32x3": phases_mixed}}

    bg.set_precision(plugin.FP64)
    bg.autotune(None, reps=3)
    (e_l, z_l, n_l), t_l, _ = _timed(lambda: bg.lanczos_lowest(init, steps=lanczos_steps,
                                                              tolerance=1e-12))
    out["fp64_lanczos"] = {"energy": e_l, "seconds": t_l, "matvecs": n_l + 1}

    (e_j, z_j, s_j), t_j, _ = _timed(lambda: bg.davidson_lowest(
        init, preconditioner=1, tolerance=tolerance, max_iterations=4000,
        raise_on_no_convergence=False))
    out["fp64_davidson"] = {"energy": e_j, "seconds": t_j, "matvecs": s_j["fp64_matvecs"],
                            "converged": s_j["converged"]}

    def compare(e, z):
        return {"abs_dE_per_site_vs_fp64": abs(e - e_j) / sites,
                "one_minus_overlap_vs_fp64": 1.0 - abs(float(torch.dot(z, z_j))),
                "abs_dE_per_site_vs_fp64_lanczos": abs(e - e_l) / sites}

    bg.set_precision(plugin.TF32X3)

    def mixed_refined():
        e1, z1, n1 = bg.lanczos_lowest(init, steps=mixed_steps, tolerance=1e-4,
                                       reortho=mixed_reortho)
        e2, st = bg.refine_lowest(z1, max_outer=8, tolerance=tolerance,
                                  inner_iterations=refine_inner,
                                  inner_tolerance=refine_inner_tolerance,
                                  raise_on_no_convergence=False)
        return e2, z1, n1, st
    (e_r, z_r, n_r, st_r), t_r, _ = _timed(mixed_refined)
    out["mixed_lanczos_refined"] = dict(
        energy=e_r, seconds=t_r, mixed_lanczos_steps=n_r + 1,
        refine_mixed_matvecs=st_r["inner_matvecs"], fp64_matvecs=st_r["fp64_matvecs"],
        converged=st_r["converged"], **compare(e_r, z_r))
    out["speedup_vs_fp64_lanczos"] = t_l / t_r
    out["speedup_with_setup"] = (t_l + setup_fp64) / (t_r + setup_mixed)
    # growth of the memory pool during the timed creates and solves (0: every
    # buffer came from memory the warm-up step had returned)
    out["pool_growth_bytes"] = plugin.cached_memory()[0] - pool_before

    # warm start: the previous sweep step's state transformed to this
    # superblock is close to the answer; stand-in: the FP64 ground state plus
    # seeded noise with overlap ~0.95.  FP64 Lanczos from it against the FP64
    # refinement alone (TF32x3 correction solves), no Lanczos phase.
    g = torch.from_numpy(np.random.default_rng(seed + 1).standard_normal(prob.dim)).cuda()
    g -= torch.dot(g, z_j) * z_j
    g /= torch.linalg.norm(g)
    warm = 0.95 * z_j + np.sqrt(1.0 - 0.95 ** 2) * g
    bg.set_precision(plugin.FP64)
    (e_wl, _, n_wl), t_wl, _ = _timed(lambda: bg.lanczos_lowest(warm, steps=lanczos_steps,
                                                               tolerance=1e-12))
    bg.set_precision(plugin.TF32X3)

    def warm_refined():
        psi = warm.clone()
        e2, st = bg.refine_lowest(psi, max_outer=12, tolerance=tolerance,
                                  inner_iterations=refine_inner,
                                  inner_tolerance=refine_inner_tolerance,
                                  raise_on_no_convergence=False)
        return e2, psi, st
    (e_wr, z_wr, st_wr), t_wr, _ = _timed(warm_refined)
    out["warm_start"] = {
        "start_overlap": 0.95,
        "fp64_lanczos": {"energy": e_wl, "seconds": t_wl, "matvecs": n_wl + 1},
        "mixed_refinement": dict(energy=e_wr, seconds=t_wr,
                                 refine_mixed_matvecs=st_wr["inner_matvecs"],
                                 fp64_matvecs=st_wr["fp64_matvecs"], converged=st_wr["converged"],
                                 **compare(e_wr, z_wr)),
        "speedup": t_wl / t_wr}

    if with_davidson:
        pre = 2 if mlp is not None else 1
        (e_m, z_m, s_m), t_m, _ = _timed(lambda: bg.davidson_lowest(
            init, preconditioner=pre, mlp=mlp, tolerance=tolerance, max_iterations=4000,
            raise_on_no_convergence=False))
        out["mixed_davidson"] = dict(
            energy=e_m, seconds=t_m, mixed_matvecs=s_m["mixed_matvecs"],
            fp64_matvecs=s_m["fp64_matvecs"], converged=s_m["converged"],
            preconditioner="learned" if mlp is not None else "jacobi", **compare(e_m, z_m))
    bg.close()
    return out


def step_attribution(prob, sites: int, repeats: int = 5, seed: int = 7,
                     lanczos_steps: int = 300, mixed_steps: int = 60,
                     tolerance: float = 1e-9) -> Dict:
    """Separates the mixed solve's gain over the plain method into its causes,
    each arm on its own handle, every arm repeated `repeats` times in
    interleaved order (median, min, max seconds of device time):
      fp64_lanczos        -- the plain method: FP64 handle, FP64 Lanczos with
                             full reorthogonalisation, eigenvalue change 1e-12;
      fp64_refined        -- the mixed solve's scheme in FP64: mixed_steps
                             Lanczos steps without reorthogonalisation (1e-4
                             Ritz-value change), then the FP64 refinement
                             whose correction solves also run in FP64;
      mixed_refined       -- the same scheme with TF32x3 matvecs in the Lanczos
                             phase and the correction solves (TF32X3 handle).
    scheme_gain = fp64_lanczos / fp64_refined, precision_gain = fp64_refined /
    mixed_refined; their product is the total.  Before timing, every arm runs
    once untimed, so the library's memory pool already holds what the timed
    solves need (pool_growth_bytes reports any growth during the timing)."""
    import torch
    init = torch.from_numpy(np.random.default_rng(seed).standard_normal(prob.dim)).cuda()
    b64 = plugin.BatchedGemm.from_problem(prob, precision=plugin.FP64)
    bmx = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
    for b in (b64, bmx):
        b.set_precision(plugin.FP64)
        b.autotune(None, reps=3)
    bmx.set_precision(plugin.TF32X3)

    def refined(bg):
        e1, z1, n1 = bg.lanczos_lowest(init, steps=mixed_steps, tolerance=1e-4, reortho=False)
        e2, st = bg.refine_lowest(z1, max_outer=8, tolerance=tolerance, inner_iterations=80,
                                  inner_tolerance=1e-2, raise_on_no_convergence=False)
        return e2, z1, st

    arms = {"fp64_lanczos": lambda: b64.lanczos_lowest(init, steps=lanczos_steps, tolerance=1e-12),
            "fp64_refined": lambda: refined(b64),
            "mixed_refined": lambda: refined(bmx)}
    for fn in arms.values():             # untimed: sizes the memory pool
        fn()
    pool_before = plugin.cached_memory()[0]
    times = {k: [] for k in arms}
    results = {}
    for _ in range(repeats):
        for k, fn in arms.items():
            results[k], t, _ = _timed(fn)
            times[k].append(t)
    pool_growth = plugin.cached_memory()[0] - pool_before
    b64.close()
    bmx.close()
    e_ref, z_ref, n_ref = results["fp64_lanczos"]
    out = {"sector_dim": prob.dim, "repeats": repeats, "pool_growth_bytes": pool_growth}
    for k in arms:
        ts = sorted(times[k])
        rec = {"median_seconds": ts[len(ts) // 2], "min_seconds": ts[0], "max_seconds": ts[-1]}
        if k == "fp64_lanczos":
            rec.update(energy=e_ref, matvecs=n_ref + 1)
        else:
            e, z, st = results[k]
            rec.update(energy=e, converged=st["converged"], refine_inner_matvecs=st["inner_matvecs"],
                       refine_fp64_matvecs=st["fp64_matvecs"],
                       abs_dE_per_site_vs_fp64_lanczos=abs(e - e_ref) / sites,
                       one_minus_overlap_vs_fp64_lanczos=1.0 - abs(float(torch.dot(z, z_ref))))
        out[k] = rec
    med = {k: out[k]["median_seconds"] for k in arms}
    out["scheme_gain"] = med["fp64_lanczos"] / med["fp64_refined"]
    out["precision_gain"] = med["fp64_refined"] / med["mixed_refined"]
    out["total_gain"] = med["fp64_lanczos"] / med["mixed_refined"]
    return out
