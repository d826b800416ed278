"""Whole DMRG runs of the configurations the benchmark names, with every
sector eigensolve on the GPU (test infrastructure: the sweep engine is the
oracle's two-site driver, oracle/dmrg_driver.py).

    python tests/dmrg_runs.py c3 [--L 64 --m 1000 --sweeps 6] [--out run.json]
    python tests/dmrg_runs.py ladder [--Lx 32 --m-inf 4000 --m 4000 --steps 1] [--mlp w.npz]
                                    [--out run.json]
    python tests/dmrg_runs.py ladder-mlp --mlp w.npz [--out run.json]
    python tests/dmrg_runs.py serving [--out run.json]

c3: Fermi-Hubbard chain, t=1, U=4, open BC, half filling, m states kept, the
    given finite sweeps.  The trajectory follows the mixed-precision solve
    (TF32x3 Lanczos without reorthogonalisation, then the FP64 residual
    refinement with TF32x3 correction solves); at every step the same sector
    is also solved from the same start vector by the plain FP64 Lanczos (full
    reorthogonalisation, eigenvalue-change tolerance 1e-10), and |dE|/site and
    1 - |<psi|psi_FP64>| are recorded.  A second run along the FP64 trajectory
    gives the final-energy comparison of the two runs.
ladder: two-leg Hubbard ladder Lx x 2, t_leg = t_rung = 1, U=8, 56 electrons
    (Sz=0) on 64 sites; infinite growth at m_inf states, then finite steps at
    m states (or, with m_inf = m, the last infinite-growth steps measured:
    their blocks hold ~4 m states each, as in a sweep at m).  Each finite step's sector is solved by the plain FP64 Lanczos
    (its own FP64 handle), by TF32x3 Lanczos + FP64 refinement, by the FP64
    Jacobi-preconditioned Davidson and by the mixed Davidson with the learned
    correction (weights trained on this ladder at m <= 1000); seconds (device
    time of the whole solve, handle set-up separate), iterations and energies
    per site are recorded.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import dmrg_driver as dd  # noqa: E402


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _timed(fn):
    import torch
    torch.cuda.synchronize()
    a, b = _events()
    a.record()
    out = fn()
    b.record()
    b.synchronize()
    return out, a.elapsed_time(b) / 1e3


def mixed_solve(bg, init, sites, tolerance=1e-10):
    """The library's mixed sector solve (BatchedGemm.solve_lowest, method
    "mixed"): TF32x3 Lanczos without reorthogonalisation (up to 150 steps or
    a 1e-7 Ritz-value change), then the FP64 refinement to |r| <= tolerance
    |E|, and FP64 Lanczos from the refined state when the refinement reports
    no convergence (counted as a fallback in the returned stats)."""
    e, z, st = bg.solve_lowest(init, tolerance=tolerance, method="mixed")
    return e, z, st["mixed_lanczos_steps"], st


def c3(L=64, U=4.0, m=1000, sweeps=6, fp64_run=True, log=print, method="mixed", tune=True,
       repeats=1, correction="jacobi"):
    """method: the library's solve_lowest method of the measured arm
    ("mixed", or "auto": mixed only where the tuned TF32x3 H*x is at least
    1.5x the tuned FP64 one).  tune: autotune every sector's FP64
    configuration through one tuning cache for the run (its bucketed keys let
    later steps reuse earlier timings; the tuning seconds are recorded).
    repeats: each step's two solves are timed that many times from the same
    start (the first result drives the sweep; every time is recorded, and
    the per-step minimum separates the solvers' own time from stalls that
    come from outside them)."""
    import tempfile
    import torch
    from dmrgpp_b200 import plugin
    steps = []
    cache = os.path.join(tempfile.mkdtemp(prefix="dmrgpp_tune_"), "tune.txt") if tune else None

    def solve(prob, init):
        x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
        bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
        try:
            t_tune, t64_us, t32_us = 0.0, -1.0, -1.0
            if tune:
                t0 = time.perf_counter()
                bg.autotune(cache, reps=5)
                t_tune = time.perf_counter() - t0
                t64_us, t32_us = bg.tuned_times()
            pool0 = plugin.cached_memory()[0]
            (e, z, st), t_mx = _timed(lambda: bg.solve_lowest(x, tolerance=1e-10, method=method,
                                                              correction=correction))
            pool1 = plugin.cached_memory()[0]
            bg.set_precision(plugin.FP64)
            (e64, z64, n64), t_64 = _timed(lambda: bg.lanczos_lowest(x, steps=400, tolerance=1e-10))
            pool2 = plugin.cached_memory()[0]
            t_mx_all, t_64_all = [t_mx], [t_64]
            for _ in range(repeats - 1):
                bg.set_precision(plugin.TF32X3)
                t_mx_all.append(_timed(lambda: bg.solve_lowest(x, tolerance=1e-10, method=method,
                                                              correction=correction))[1])
                bg.set_precision(plugin.FP64)
                t_64_all.append(_timed(lambda: bg.lanczos_lowest(x, steps=400, tolerance=1e-10))[1])
        finally:
            bg.close()
        n1 = st.get("mixed_lanczos_steps", st.get("fp64_lanczos_steps", 0))
        rec = dict(dim=prob.dim, f_alg=prob.flops(), e_mixed=e, e_fp64=e64,
                   abs_dE_per_site=abs(e - e64) / L,
                   one_minus_overlap=1.0 - abs(float(torch.dot(z, z64))),
                   mixed_seconds=t_mx, fp64_seconds=t_64, fp64_lanczos_steps=n64,
                   method=st["method"], mixed_lanczos_steps=n1, fallback=int(st.get("fallback", 0)),
                   refine_converged=int(st["converged"]),
                   mixed_lanczos_seconds=st.get("mixed_lanczos_seconds", 0.0),
                   refine_seconds=st.get("refine_seconds", 0.0),
                   refine_outer=int(st.get("outer_iterations", -1)),
                   refine_inner_matvecs=int(st.get("inner_matvecs", -1)),
                   tune_seconds=t_tune, tuned_fp64_us=t64_us, tuned_tf32x3_us=t32_us,
                   pool_growth_mixed=pool1 - pool0, pool_growth_fp64=pool2 - pool1,
                   mixed_seconds_all=t_mx_all, fp64_seconds_all=t_64_all)
        steps.append(rec)
        if len(steps) % 20 == 0:
            log(f"step {len(steps)} dim {prob.dim} E {e:.12f} dE/site {rec['abs_dE_per_site']:.2e}")
        return e, z.cpu().numpy(), n1

    t0 = time.time()
    # half filling at every stage (the model scales the target with the sites)
    d = dd.DMRG(dd.Hubbard(U=U), L=L, m=m, solver=solve)
    e_mixed = d.run(sweeps=sweeps)
    out = dict(config=f"Hubbard chain L={L} U={U} half filling m={m} {sweeps} finite sweeps",
               steps=len(steps), final_energy_mixed_run=e_mixed,
               max_abs_dE_per_site_same_input=max(s["abs_dE_per_site"] for s in steps),
               max_one_minus_overlap=max(s["one_minus_overlap"] for s in steps),
               all_converged=all(s["refine_converged"] for s in steps),
               fallbacks=sum(s["fallback"] for s in steps),
               max_dim=max(s["dim"] for s in steps),
               solve_seconds_mixed=sum(s["mixed_seconds"] for s in steps),
               solve_seconds_fp64=sum(s["fp64_seconds"] for s in steps),
               solve_seconds_mixed_min_of_repeats=sum(min(s["mixed_seconds_all"]) for s in steps),
               solve_seconds_fp64_min_of_repeats=sum(min(s["fp64_seconds_all"]) for s in steps),
               repeats=repeats, correction=correction,
               tune_seconds=sum(s["tune_seconds"] for s in steps), method=method,
               steps_solved_mixed=sum(s["method"] == "mixed" for s in steps),
               wall_seconds_mixed_run=time.time() - t0, per_step=steps)
    if fp64_run:
        t1 = time.time()
        n64 = []

        def solve64(prob, init):
            bg = plugin.BatchedGemm.from_problem(prob)
            try:
                if tune:
                    bg.autotune(cache, reps=5)
                e, z, n = bg.lanczos_lowest(init, steps=400, tolerance=1e-10)
            finally:
                bg.close()
            n64.append(n)
            return e, z, n
        d64 = dd.DMRG(dd.Hubbard(U=U), L=L, m=m, solver=solve64)
        e64 = d64.run(sweeps=sweeps)
        out.update(final_energy_fp64_run=e64, final_abs_dE_per_site=abs(e_mixed - e64) / L,
                   wall_seconds_fp64_run=time.time() - t1)
    return out


def ladder_electrons(Lx):
    """Filling 0.875 with Sz = 0 (56 electrons on 32 x 2 sites)."""
    return int(round(0.875 * 2 * Lx / 2)) * 2


def ladder_model(Lx=32, U=8.0, electrons=None):
    ne = electrons if electrons is not None else ladder_electrons(Lx)
    return dd.HubbardLadder(Lx, t_leg=1.0, t_rung=1.0, U=U, n_up=ne // 2, n_dn=ne // 2)


def ladder_sectors(Lx=32, U=8.0, electrons=None, m_inf=1000, m=4000, finite_steps=2,
                   on_sector=None, log=print):
    """Runs the ladder's infinite growth at m_inf (mixed solves), then
    finite_steps left-to-right steps from the middle at m states; calls
    on_sector(prob, init, step_index) for each finite step's sector, which
    returns the (energy, state) the run continues with."""
    import torch
    from dmrgpp_b200 import plugin
    L = 2 * Lx

    def solve(prob, init):
        x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
        bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
        try:
            e, z, n, st = mixed_solve(bg, x, L)
        finally:
            bg.close()
        return e, z.cpu().numpy(), n

    d = dd.DMRG(ladder_model(Lx, U, electrons), L=L, m=m_inf, solver=solve)
    b_l = b_r = d.site
    left, right = {1: b_l}, {1: b_r}
    n = 1
    while 2 * (n + 1) <= L:
        t0 = time.time()
        e, lp, rp, rl, rr = d.step(b_l, b_r, 2 * (n + 1))
        b_l, b_r = d.truncate(lp, rl), d.truncate(rp, rr)
        n += 1
        left[n], right[n] = b_l, b_r
        log(f"infinite {n}: E {e:.10f} left states {sum(lp.sizes)} ({time.time() - t0:.1f} s)")
    d.m = m
    records = []
    for q, nl in enumerate(range(L // 2, L // 2 + finite_steps)):
        lp, rp = d.grow_left(left[nl]), d.grow_right(right[L - nl - 2], L)
        target = d.model.target(L)
        prob, patches = d.superblock(lp, rp, target, L)
        init = d.rng.standard_normal(prob.dim)
        e, psi, rec = on_sector(prob, init, q)
        records.append(rec)
        rho_l = {}
        xs = prob.xy_start
        for p, (gl, gr) in enumerate(patches):
            X = psi[xs[p]:xs[p + 1]].reshape(int(prob.lsz[p]), int(prob.rsz[p])).T
            rho_l[gl] = rho_l.get(gl, 0.0) + X.T @ X
        left[nl + 1] = d.truncate(lp, rho_l)
        log(f"finite step {q}: E {e:.10f} dim {prob.dim} left states {sum(lp.sizes)}")
    return records


def ladder_infinite(Lx=32, U=8.0, m=4000, measure_last=1, on_sector=None, log=print):
    """Infinite growth of the ladder at m states to 2 Lx sites (mixed solves);
    the last measure_last steps (blocks of ~4 m states each once m is
    reached: the superblocks of a sweep at m) go to on_sector(prob, init, q),
    which returns (energy, state, record)."""
    import torch
    from dmrgpp_b200 import plugin
    L = 2 * Lx

    def solve(prob, init):
        x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
        bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
        try:
            e, z, n, st = mixed_solve(bg, x, L)
        finally:
            bg.close()
        return e, z.cpu().numpy(), n

    records = []
    d = dd.DMRG(ladder_model(Lx, U), L=L, m=m, solver=solve)
    b_l = b_r = d.site
    nsteps = L // 2 - 1
    for n in range(1, nsteps + 1):
        t0 = time.time()
        q = n - (nsteps - measure_last) - 1
        if q >= 0:
            def measured(prob, init, q=q):
                e, z, rec = on_sector(prob, init, q)
                rec["sites"] = 2 * (n + 1)
                records.append(rec)
                return e, z, 0
            d.solver = measured
        e, lp, rp, rl, rr = d.step(b_l, b_r, 2 * (n + 1))
        d.solver = solve
        if n < nsteps:
            b_l, b_r = d.truncate(lp, rl), d.truncate(rp, rr)
        log(f"infinite {n}: N {2 * (n + 1)} E {e:.10f} left states {sum(lp.sizes)} "
            f"({time.time() - t0:.1f} s)")
    return records


def ladder_step_measurement(prob, init, sites, mlp=None, lanczos_steps=400):
    """One ladder sector solved every way (see the module docstring)."""
    import torch
    from dmrgpp_b200 import plugin
    x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
    rec = dict(dim=prob.dim, npatches=prob.npatches, noperator=prob.noperator,
               f_alg=prob.flops())
    # plain FP64 on its own FP64 handle; a warm create first (the previous
    # step's buffers back in the pool, as in a sweep)
    warm = plugin.BatchedGemm.from_problem(prob)
    warm.lanczos_lowest(x, steps=lanczos_steps, min_steps=2, tolerance=1e300)
    warm.close()
    b64, t_set64 = _timed(lambda: plugin.BatchedGemm.from_problem(prob))
    b64.autotune(None, reps=3)
    (e64, z64, n64), t64 = _timed(lambda: b64.lanczos_lowest(x, steps=lanczos_steps,
                                                             tolerance=1e-10))
    (ej, zj, sj), tj = _timed(lambda: b64.davidson_lowest(x, preconditioner=1, tolerance=1e-9,
                                                          max_iterations=4000,
                                                          raise_on_no_convergence=False))
    b64.close()
    rec["fp64_lanczos"] = dict(energy=e64, seconds=t64, setup_seconds=t_set64, matvecs=n64 + 1)
    rec["fp64_jacobi_davidson"] = dict(energy=ej, seconds=tj, iterations=sj["iterations"],
                                       converged=sj["converged"])
    bmx, t_setmx = _timed(lambda: plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3))
    bmx.set_precision(plugin.FP64)
    bmx.autotune(None, reps=3)
    (e, z, n1, st), tmx = _timed(lambda: mixed_solve(bmx, x, sites, tolerance=1e-9))
    rec["mixed_lanczos_refined"] = dict(
        energy=e, seconds=tmx, setup_seconds=t_setmx, lanczos_steps=n1 + 1,
        refine_mixed_matvecs=st["inner_matvecs"], fp64_matvecs=st["fp64_matvecs"],
        converged=st["converged"], fallback=st["fallback"], abs_dE_per_site=abs(e - e64) / sites,
        one_minus_overlap=1.0 - abs(float(torch.dot(z, z64))))
    for name, pre, m in (("mixed_davidson_none", 0, None), ("mixed_davidson_jacobi", 1, None),
                         ("mixed_davidson_learned", 2, mlp)):
        if pre == 2 and mlp is None:
            continue
        bmx.set_precision(plugin.TF32X3)
        (ed, zd, sd), td = _timed(lambda: bmx.davidson_lowest(
            x, preconditioner=pre, mlp=m, tolerance=1e-9, max_iterations=4000,
            raise_on_no_convergence=False))
        rec[name] = dict(energy=ed, seconds=td, iterations=sd["iterations"],
                         converged=sd["converged"], abs_dE_per_site=abs(ed - e64) / sites)
    bmx.close()
    rec["speedup_mixed_vs_fp64"] = t64 / tmx
    rec["speedup_with_setup"] = (t64 + t_set64) / (tmx + t_setmx)
    return e, z.cpu().numpy(), rec


def ladder_mlp(train_specs=((12, 400), (16, 600)), test_specs=((16, 1000),), sectors_per_run=3,
               out_path=None, log=print):
    """The learned correction trained on real ladder superblocks: two-leg
    Hubbard ladders (U=8, filling 0.875) of Lx rungs run at m states (mixed
    solves); the last sectors_per_run finite-step sectors of each training
    run give solver-generated (features, exact correction) pairs
    (dmrgpp_b200.mlp.correction_pairs), the 3 x 256 network is trained by the
    library's kernels, and on the test runs' sectors Davidson runs to
    |r| <= 1e-9 |E| with no correction, the Jacobi correction and the learned
    one (TF32x3 matvecs, FP64 restart phase) are counted and timed.  Returns
    the summary; writes the weights to out_path."""
    import torch
    from dmrgpp_b200 import plugin
    from dmrgpp_b200.mlp import MLPPreconditioner, correction_pairs, train

    def sectors(Lx, m):
        kept = []

        def on_sector(prob, init, q):
            x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
            bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
            try:
                e, z, n, st = mixed_solve(bg, x, 2 * Lx)
            finally:
                bg.close()
            kept.append((prob, init))
            return e, z.cpu().numpy(), None
        ladder_sectors(Lx=Lx, m_inf=m, m=m, finite_steps=sectors_per_run,
                       on_sector=on_sector, log=lambda *a: None)
        return kept

    t0 = time.time()
    Xs, Ys, infos = [], [], []
    for Lx, m in train_specs:
        for prob, init in sectors(Lx, m):
            bg = plugin.BatchedGemm.from_problem(prob)
            x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
            for xx, yy, info in correction_pairs(bg, x):
                Xs.append(xx)
                Ys.append(yy)
                infos.append(info)
            bg.close()
        log(f"training data: Lx={Lx} m={m}: {sum(x.shape[0] for x in Xs)} rows "
            f"({time.time() - t0:.0f} s)")
    X = torch.cat(Xs)
    Y = torch.cat(Ys).clamp(-20, 20)
    mlp = MLPPreconditioner(seed=2026)
    losses = train(mlp, X, Y, steps=800, batch=8192, lr=2e-3)
    if out_path:
        mlp.save(out_path)
    summary = dict(rows=int(X.shape[0]), loss_first=float(np.mean(losses[:20])),
                   loss_last=float(np.mean(losses[-20:])),
                   cos_exact_vs_jacobi=float(np.mean([i["cos_jacobi"] for i in infos])),
                   cos_exact_vs_residual=float(np.mean([i["cos_residual"] for i in infos])),
                   train_seconds=time.time() - t0, held_out=[])
    for Lx, m in test_specs:
        for prob, init in sectors(Lx, m):
            bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
            x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
            rec = dict(Lx=Lx, m=m, dim=prob.dim)
            for name, pre, mm in (("none", 0, None), ("jacobi", 1, None), ("learned", 2, mlp)):
                (e, z, st), t = _timed(lambda: bg.davidson_lowest(
                    x, preconditioner=pre, mlp=mm, tolerance=1e-9, max_iterations=4000,
                    raise_on_no_convergence=False))
                rec[name] = dict(energy=e, seconds=t, iterations=st["iterations"],
                                 converged=st["converged"])
            bg.set_precision(plugin.FP64)
            (e, z, st), t = _timed(lambda: bg.davidson_lowest(
                x, preconditioner=1, tolerance=1e-9, max_iterations=4000,
                raise_on_no_convergence=False))
            rec["fp64_jacobi"] = dict(energy=e, seconds=t, iterations=st["iterations"],
                                      converged=st["converged"])
            bg.close()
            summary["held_out"].append(rec)
            log(json.dumps(rec, default=float))
    mlp.close()
    return summary


def serving_problems(n=256, seed=20261203, log=print):
    """The serving-style batch built from real DMRG superblocks: n problems,
    each a Heisenberg (J=1) or Hubbard (t=1, U uniform in [0, 8]) chain
    (seeded coin) with L uniform in [16, 48] (rounded down to even) and m from
    {64, 128, 256, 512}; its sector is the last infinite-growth superblock
    (N = L sites, Sz = 0 or half filling) of a driver run at m states (mixed
    solves along the way).  Heisenberg problems of one m share one run to
    their largest L.  Returns (probs, meta)."""
    import torch
    from dmrgpp_b200 import plugin
    rng = np.random.default_rng(seed)
    specs = []
    for q in range(n):
        L = int(rng.integers(16, 49)) // 2 * 2
        m = int(rng.choice([64, 128, 256, 512]))
        if rng.random() < 0.5:
            specs.append(("heisenberg", L, 0.0, m))
        else:
            specs.append(("hubbard", L, float(rng.uniform(0.0, 8.0)), m))

    def solve(prob, init):
        x = torch.from_numpy(np.ascontiguousarray(init)).cuda()
        bg = plugin.BatchedGemm.from_problem(prob, precision=plugin.TF32X3)
        try:
            e, z, nn, st = mixed_solve(bg, x, 1)
        finally:
            bg.close()
        return e, z.cpu().numpy(), nn

    def run(model, Lmax, m, wanted):
        d = dd.DMRG(model, L=Lmax, m=m, solver=solve)
        got = {}
        b_l = b_r = d.site
        n_ = 1
        while 2 * (n_ + 1) <= Lmax:
            N = 2 * (n_ + 1)
            if N in wanted:
                d.keep_sectors = True
            e, lp, rp, rl, rr = d.step(b_l, b_r, N)
            if d.keep_sectors:
                got[N] = d.sectors.pop()
                d.keep_sectors = False
            b_l, b_r = d.truncate(lp, rl), d.truncate(rp, rr)
            n_ += 1
        return got

    t0 = time.time()
    sectors = {}
    for m in sorted({s[3] for s in specs if s[0] == "heisenberg"}):
        Ls = {s[1] for s in specs if s[0] == "heisenberg" and s[3] == m}
        for L, p in run(dd.Heisenberg(), max(Ls), m, Ls).items():
            sectors[("heisenberg", L, 0.0, m)] = p
    for q, s in enumerate(specs):
        if s[0] == "hubbard":
            sectors[s] = run(dd.Hubbard(U=s[2]), s[1], s[3], {s[1]})[s[1]]
        if q % 32 == 31:
            log(f"serving batch: {q + 1} problems ({time.time() - t0:.0f} s)")
    probs = [sectors[s] for s in specs]
    meta = [{"model": s[0], "L": s[1], "U": s[2], "m": s[3]} for s in specs]
    return probs, meta


def serving(n=256, log=print):
    """bench.py's serving measurements on the batch of real superblocks."""
    import torch
    sys.path.insert(0, ROOT)
    import bench
    probs, meta = serving_problems(n, log=log)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    out = bench.serving_measurements(
        torch, dev, stream, cpu_sample=True, probs=probs, meta=meta, correction="jacobi",
        workload=f"serving-batch-{n} of real DMRG superblocks (Heisenberg / Hubbard chains, "
                 "L 16-48, U 0-8, m 64-512, last infinite-growth sector)")
    out["dims"] = {"min": int(min(p.dim for p in probs)), "max": int(max(p.dim for p in probs))}
    return out


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("what", choices=["c3", "ladder", "ladder-mlp", "serving"])
    p.add_argument("--L", type=int, default=64)
    p.add_argument("--m", type=int, default=None)
    p.add_argument("--sweeps", type=int, default=6)
    p.add_argument("--Lx", type=int, default=32)
    p.add_argument("--m-inf", type=int, default=1000)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--no-fp64-run", action="store_true")
    p.add_argument("--method", default="mixed", choices=["mixed", "auto"])
    p.add_argument("--no-tune", action="store_true")
    p.add_argument("--repeats", type=int, default=1)
    p.add_argument("--correction", default="jacobi", choices=["none", "jacobi"])
    p.add_argument("--mlp", default=None, help="learned-correction weights (.npz)")
    p.add_argument("--out", default=None)
    a = p.parse_args(argv)
    if a.what == "serving":
        out = serving()
        text = json.dumps(out, indent=1, default=float)
        if a.out:
            with open(a.out, "w") as f:
                f.write(text)
        print(json.dumps({k: v for k, v in out.items() if k not in ("group_davidson",)},
                         default=float))
        return
    if a.what == "ladder-mlp":
        out = ladder_mlp(out_path=a.mlp)
        print(json.dumps({k: v for k, v in out.items() if k != "held_out"}, default=float))
        for r in out["held_out"]:
            print(json.dumps(r, default=float))
        if a.out:
            with open(a.out, "w") as f:
                json.dump(out, f, indent=1, default=float)
        return
    if a.what == "c3":
        out = c3(L=a.L, m=a.m or 1000, sweeps=a.sweeps, fp64_run=not a.no_fp64_run,
                 method=a.method, tune=not a.no_tune, repeats=a.repeats,
                 correction=a.correction)
    else:
        from dmrgpp_b200.mlp import MLPPreconditioner
        mlp = MLPPreconditioner.load(a.mlp) if a.mlp else None
        L = 2 * a.Lx
        measure = lambda prob, init, q: ladder_step_measurement(prob, init, L, mlp=mlp)
        if a.m_inf == (a.m or 4000):
            recs = ladder_infinite(Lx=a.Lx, m=a.m_inf, measure_last=a.steps, on_sector=measure)
            how = f"infinite growth at m={a.m_inf}, the last {a.steps} steps measured"
        else:
            recs = ladder_sectors(Lx=a.Lx, m_inf=a.m_inf, m=a.m or 4000, finite_steps=a.steps,
                                  on_sector=measure)
            how = f"m_inf={a.m_inf}, then {a.steps} finite steps at m={a.m or 4000}"
        out = dict(config=f"Hubbard ladder {a.Lx}x2, t_leg = t_rung = 1, U=8, "
                          f"{ladder_electrons(a.Lx)} electrons (Sz=0); {how}", steps=recs)
    text = json.dumps(out, indent=1, default=float)
    if a.out:
        with open(a.out, "w") as f:
            f.write(text)
    summary = {k: v for k, v in out.items() if k not in ("per_step", "steps")}
    print(json.dumps(summary, default=float))
    if a.what == "ladder":
        for r in out["steps"]:
            print(json.dumps({k: v for k, v in r.items()}, default=float))


if __name__ == "__main__":
    main()
