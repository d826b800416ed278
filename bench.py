"""Benchmark of the superblock Kronecker H*psi (one step = one matvec of one
sector) on B200, against the reference's CPU batched path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|ladder] [--precision fp64]

Prints one JSON line on rank 0.  Multi-GPU runs (torchrun, one rank per GPU)
are independent replicas of the sector (the path is single-GPU), timed on the
device as the max over ranks.

    python bench.py --profile-case c2 [--precision fp64|tf32x3] [--applies N]
                                      [--config C --ipc I]
    python bench.py --profile-case ladder --states 4000 --precision tf32x3
    python bench.py --profile-case ladder --states 4000 --solve lanczos
    python bench.py --profile-case mlp --elements 300000 [--inference cuda_cores]
    python bench.py --profile-case wft --states 4000
    python bench.py --profile-case truncation --states 16000
    python bench.py --profile-case serving --problems 256

runs one fixed workload on cuda:0 and nothing else, so that a profiler's
launch list and captures see only its kernels: c2 = the 1024 x 1024-state,
21-group, K=5 microbench sector; ladder = the ladder-shaped (N_up, N_down)
sector with `--states` left and right states (K = 10); mlp = learned-
preconditioner applications (seeded network, seeded diagonal and residual of
`--elements` entries); wft = the wave-function transformation of the
ladder-shaped layout with seeded square N(0,1)/sqrt(n) blocks; truncation =
the density-matrix truncation of the ladder-shaped layout's system block (one
group per patch) for a seeded unit sector vector, a quarter of the states
kept; serving = the serving-style batch (superblock.serving_batch) in one
TF32x3 group handle, solved once as the bench does: group Lanczos to a
Ritz-value change of 1e-5, then the lockstep FP64 group refinement.  Prints
one line "ok ..." at the end.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Kron-matvec TFLOP/s"
UNIT = "TFLOP/s"
FLUSH_BYTES = 256 << 20  # > 126 MB L2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c2", choices=["c2", "ladder"])
    p.add_argument("--precision", default="fp64", choices=["fp64"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-sweep", action="store_true",
                   help="skip the ladder-sector solve and mixed-precision measurements")
    p.add_argument("--no-serving", action="store_true",
                   help="skip the 256-problem serving-batch measurements")
    return p.parse_args()


def make_problem(name):
    from dmrgpp_b200 import superblock as sb
    if name == "c2":
        return sb.c2_problem()
    return sb.ladder_problem()


def workload_config(prob, name):
    return {"workload": prob.name + (" (synthetic Kronecker-matvec microbench)" if name == "c2"
                                     else ""),
            "sector_dim": prob.dim, "npatches": prob.npatches, "noperator": prob.noperator,
            "triples": len(prob.triples()), "f_alg_per_step": prob.flops(),
            "operator_bytes": prob.operator_bytes()}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """NVML samples of SM clock and throttle reasons while running."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4}

    def __init__(self, index=0, period=0.005):
        self.samples, self.reasons, self.ok = [], set(), False
        self.period = period
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None
        self._stop = threading.Event()
        self.active = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            if self.active.is_set():
                try:
                    self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h,
                                                                       self.nv.NVML_CLOCK_SM))
                    r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    for name, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(name)
                except Exception:
                    pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self.ok:
            self.t.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------- CPU baselines
def cpu_baseline(prob, f_alg, calls=30):
    """The reference's own BatchedGemmCpu (compiled from its sources into
    oracle/_ref) on all host cores; the scalar C restatement if that build
    is absent.  Median of `calls` matvecs after one warm-up."""
    import oracle
    x = np.random.default_rng(7).standard_normal(prob.dim)
    if oracle.ref_available():
        rk = oracle.RefKron(prob)
        rk.apply(x)
        ts = []
        for _ in range(calls):
            t0 = time.perf_counter()
            rk.apply(x)
            ts.append(time.perf_counter() - t0)
        t = statistics.median(ts)
        cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
        out = {"value": f_alg / t / 1e12, "unit": UNIT, "cores": cores, "kind": "reference",
               "sample": f"median of {calls} full matvecs of the same sector by "
                         "Dmrg::BatchedGemmCpu::matrixVector (OpenBLAS dgemm)",
               "s_per_matvec": t}
        out["nonbatched"] = nonbatched_cpu(prob, f_alg, calls)
        return out
    oracle.build()
    calls = 3
    oracle.kron_apply(prob, x)
    ts = []
    for _ in range(calls):
        t0 = time.perf_counter()
        oracle.kron_apply(prob, x)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    return {"value": f_alg / t / 1e12, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"median of {calls} full matvecs by the scalar C restatement",
            "s_per_matvec": t}


def nonbatched_cpu(prob, f_alg, calls=30):
    """The reference's default non-batched CPU H*x (KronConnections::doTask
    with den_kron_mult per block, compiled from its sources into oracle/_ref)
    with one task thread per host core and one BLAS thread each; median of
    `calls` matvecs after one warm-up."""
    import oracle
    x = np.random.default_rng(7).standard_normal(prob.dim)
    kc = oracle.RefKronConn(prob)
    cores = os.cpu_count() or 1
    kc.apply(x, threads=cores)
    ts = []
    for _ in range(calls):
        t0 = time.perf_counter()
        kc.apply(x, threads=cores)
        ts.append(time.perf_counter() - t0)
    kc.close()
    t = statistics.median(ts)
    return {"value": f_alg / t / 1e12, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"median of {calls} full matvecs by KronConnections::doTask over the "
                      "output patches with den_kron_mult per block (the reference's default "
                      "path)", "s_per_matvec": t}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    prob = make_problem(args.workload)
    f_alg = prob.flops()
    import oracle
    if not oracle.ref_available():
        oracle.build()
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU build (oracle/_ref) not present"}))
        return 0
    rk = oracle.RefKron(prob)
    x = np.random.default_rng(7).standard_normal(prob.dim)
    for _ in range(max(args.warmup, 1)):
        rk.apply(x)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rk.apply(x)
    dt = time.perf_counter() - t0
    value = f_alg * args.steps / dt / 1e12
    cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded N(0,1) sector blocks)", "impl": "reference",
            "config": workload_config(prob, args.workload),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{args.steps} full matvecs by "
                                       "Dmrg::BatchedGemmCpu::matrixVector on host cores"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------- our arm
def measured_fp64_peak(torch, dev):
    """cuBLAS DGEMM 8192^3 (best of 5), the FP64 tensor-pipe denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = None
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        t = s.elapsed_time(e) / 1e3
        best = t if best is None else min(best, t)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


def read_traffic(workload, family="kron_persistent"):
    """dram__bytes_read.sum + dram__bytes_write.sum of one launch of the
    kernel family on this workload, from the committed ncu summary (a line
    `traffic_bytes_per_launch: N` in profiles/<family>_<workload>.md)."""
    path = os.path.join(ROOT, "profiles", f"{family}_{workload}.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"^traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read(), re.M)
    return float(m.group(1)) if m else None


def mixed_matvec_measurement(torch, dev, stream, prob, xh, y64, f_alg):
    """The same sector's H*x in TF32x3 on the tensor cores (tcgen05): time
    (L2 flushed between steps, as for the FP64 line) and the relative error
    max|y - y_FP64| / max|y_FP64| on the bench's input vector."""
    from dmrgpp_b200 import plugin
    bg = plugin.BatchedGemm.from_problem(prob, stream=stream.cuda_stream, precision=plugin.TF32X3)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    x = torch.from_numpy(np.ascontiguousarray(xh)).to(dev)
    y = torch.empty_like(x)
    ts = []
    with torch.cuda.stream(stream):
        for it in range(23):
            flush.fill_(float(it))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            bg.apply_Htarget(x, y)
            b.record(stream)
            b.synchronize()
            if it >= 3:
                ts.append(a.elapsed_time(b))
    ms = statistics.median(ts)
    err = float(np.abs(y.cpu().numpy() - y64).max() / np.abs(y64).max())
    bg.close()
    return {"precision": "tf32x3", "ms": ms, "tflops_alg": f_alg / (ms * 1e-3) / 1e12,
            "rel_err_vs_fp64": err,
            "note": "TF32x3 tensor-core H*x (3 TF32 products, FP32 accumulation) on the same "
                    "sector; rel_err = max|y - y_FP64| / max|y_FP64|"}


SERVING_MIXED_TOLERANCE = 1e-5


def learned_ablation(torch, bgm, init, stream):
    """The serving batch through the lockstep group Davidson (TF32x3 group
    matvecs, residual 1e-5, subspace 32) with no, the Jacobi and the learned
    correction (weights/serving_mlp.npz, trained by train_serving_mlp), each
    followed by the group FP64 refinement; plus the cost of one learned
    correction of the whole batch."""
    from dmrgpp_b200.mlp import MLPPreconditioner
    from dmrgpp_b200.train_serving_mlp import SERVING_WEIGHTS
    mlp = MLPPreconditioner.load(SERVING_WEIGHTS)
    bgm.davidson_lowest_group(init, max_iterations=2, raise_on_no_convergence=False)  # buffers
    runs = {}
    for name, pre in (("none", 0), ("jacobi", 1), ("learned", 2)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, zd, _, sd = bgm.davidson_lowest_group(init, preconditioner=pre,
                                                 mlp=mlp if pre == 2 else None, tolerance=1e-5,
                                                 max_iterations=600, max_subspace=32,
                                                 raise_on_no_convergence=False)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ed, cr, _ = bgm.refine_lowest_group(zd, max_outer=10, tolerance=1e-10, inner_iterations=80,
                                            inner_tolerance=1e-2, raise_on_no_convergence=False)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        runs[name] = {"seconds": t2 - t0, "davidson_seconds": t1 - t0,
                      "iterations": int(sd["iterations"]),
                      "ms_per_iteration": (t1 - t0) * 1e3 / max(1, sd["iterations"]),
                      "converged": int(cr.sum()), "energies": ed}
    diag = bgm.diagonal()
    r = torch.from_numpy(np.random.default_rng(4).standard_normal(bgm.dim)).to(diag.device)
    offs = torch.tensor(bgm.sector_offsets(), device=diag.device)
    nsec = offs.numel() - 1
    theta = torch.full((nsec,), -10.0, dtype=torch.float64, device=diag.device)
    rn = torch.ones(nsec, dtype=torch.float64, device=diag.device)
    with torch.cuda.stream(stream):
        mlp.precondition_group(diag, r, offs, theta, rn, stream=stream.cuda_stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(3):
            mlp.precondition_group(diag, r, offs, theta, rn, stream=stream.cuda_stream)
        b.record(stream)
    b.synchronize()
    mlp.close()
    return {"runs": runs, "learned_correction_ms": a.elapsed_time(b) / 3,
            "note": "group Davidson (dmrgpp_davidson_lowest_group) + dmrgpp_refine_lowest_group; "
                    "learned_correction_ms = one tensor-core MLP inference over every element "
                    "of the batch"}


def serving_measurements(torch, dev, stream, cpu_sample: bool = True, probs=None, meta=None,
                         workload=None, correction: str = "none"):
    """Serving-style batch: 256 independent ground-state problems (Heisenberg
    and Hubbard chain-shaped sectors, L in [16, 48], m in {64, 128, 256, 512},
    superblock.serving_batch) solved together by the group Lanczos (one
    persistent launch per step for all sectors, FP64, full
    reorthogonalisation) against one FP64 device Lanczos per problem, with
    per-problem |dE| between the two; the same batch in mixed precision
    (TF32x3 group Lanczos + lockstep FP64 group refinement) with |dE| per site
    and 1 - |<psi|psi_FP64>| against the single-problem FP64 solves; the
    reference's own LanczosSolver + BatchedGemmCpu (oracle/_ref) timed on a
    sample of the batch.  probs / meta (with "L" per problem) replace the
    synthetic batch when given (the physical batch of real superblocks).
    correction: the group refinement's correction solves, "none" or "jacobi"
    (diagonally preconditioned: pays on physical Hamiltonians, whose diagonal
    carries the spectrum, not on the synthetic batch's N(0,1) blocks)."""
    from dmrgpp_b200 import plugin
    from dmrgpp_b200 import superblock as sb
    if probs is None:
        probs, meta = sb.serving_batch(256)
        workload = ("serving-batch-256 (Heisenberg / Hubbard chain-shaped sectors, "
                    "L 16-48, m 64-512, seeded N(0,1) blocks)")
    bg = plugin.BatchedGemm.from_problems(probs, stream=stream.cuda_stream)
    offs = bg.sector_offsets()
    init = torch.from_numpy(np.random.default_rng(1).standard_normal(bg.dim)).to(dev)
    out = {"workload": workload,
           "problems": len(probs), "total_dim": int(bg.dim), "f_alg_per_group_matvec": bg.f_alg}
    x, y = init.clone(), torch.empty_like(init)
    with torch.cuda.stream(stream):
        for _ in range(3):
            bg.apply_Htarget(x, y)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(10):
            bg.apply_Htarget(x, y)
        b.record(stream)
    b.synchronize()
    ms = a.elapsed_time(b) / 10
    out["group_matvec"] = {"ms": ms, "tflops_alg": bg.f_alg / (ms * 1e-3) / 1e12}
    bg.lanczos_lowest_group(init)                      # warm-up (allocations)
    ts = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e, z, steps = bg.lanczos_lowest_group(init)
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    tg = min(ts)
    out["group_lanczos"] = {"seconds": tg, "problems_per_s": len(probs) / tg,
                            "steps_max": int(steps.max()), "steps_mean": float(steps.mean())}
    bg.close()
    # mixed precision: TF32x3 group matvecs for a loose group Lanczos, then
    # the lockstep FP64 refinement of every problem
    bgm = plugin.BatchedGemm.from_problems(probs, precision=plugin.TF32X3,
                                           stream=stream.cuda_stream)

    with torch.cuda.stream(stream):
        for _ in range(3):
            bgm.apply_Htarget(x, y)
        a.record(stream)
        for _ in range(10):
            bgm.apply_Htarget(x, y)
        b.record(stream)
    b.synchronize()
    ms_mixed = a.elapsed_time(b) / 10

    def mixed_solve():
        # the library's group solve: TF32x3 group Lanczos, lockstep FP64
        # refinement, FP64 group Lanczos for any sector left unconverged
        em, zm, st = bgm.solve_lowest_group(init, tolerance=1e-10,
                                            mixed_tolerance=SERVING_MIXED_TOLERANCE,
                                            correction=correction)
        torch.cuda.synchronize()
        conv = np.ones(len(em), dtype=bool)
        return (em, conv, st, zm, st["lanczos_steps"],
                (st["mixed_lanczos_seconds"], st["refine_seconds"] + st["fallback_seconds"]))

    mixed_solve()                                      # warm-up (allocations)
    runs = []
    for _ in range(2):
        torch.cuda.synchronize()
        runs.append(mixed_solve())
    em, conv, st, zm, steps_m, split = min(runs, key=lambda r: sum(r[5]))
    tm = sum(split)
    dav = learned_ablation(torch, bgm, init, stream)
    bgm.close()
    es, t_seq, ovl = [], 0.0, []
    for s, p in enumerate(probs):
        h = plugin.BatchedGemm.from_problem(p, stream=stream.cuda_stream)
        xs = init[offs[s]:offs[s + 1]].contiguous()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e1, z1, _ = h.lanczos_lowest(xs)
        t_seq += time.perf_counter() - t0
        es.append(e1)
        ovl.append(1.0 - abs(float(torch.dot(zm[offs[s]:offs[s + 1]], z1))))
        h.close()
    es = np.array(es)
    sites = np.array([m["L"] for m in meta], dtype=np.float64)
    out["group_mixed"] = {
        "seconds": tm, "problems_per_s": len(probs) / tm, "speedup_vs_group_fp64": tg / tm,
        "group_matvec_ms": ms_mixed, "lanczos_seconds": split[0], "refine_seconds": split[1],
        "lanczos_steps_max": int(steps_m.max()), "lanczos_steps_mean": float(steps_m.mean()),
        "converged": int(conv.sum()), "fp64_group_matvecs": int(st["fp64_matvecs"]),
        "fp64_lanczos_fallbacks": int(st["fallbacks"]),
        "fallback_seconds": float(st["fallback_seconds"]),
        "tf32x3_group_matvecs_in_refinement": int(st["inner_matvecs"]),
        "max_abs_dE_per_site_vs_single_fp64": float((np.abs(em - es) / sites).max()),
        "max_one_minus_overlap_vs_single_fp64": float(max(ovl)),
        "note": f"TF32x3 group Lanczos (no reorthogonalisation: it only supplies the start "
                f"vectors) to a Ritz-value change of {SERVING_MIXED_TOLERANCE:g}, then "
                "dmrgpp_refine_lowest_group (FP64 Rayleigh quotients and residuals, |r| <= "
                "1e-10 max(1, |E|)), handle creation excluded",
        "correction_solves": correction}
    for v in dav["runs"].values():
        v["max_abs_dE_per_site_vs_single_fp64"] = float((np.abs(v.pop("energies") - es) / sites).max())
    out["group_davidson"] = dav
    out["single_problem_lanczos"] = {"seconds": t_seq, "problems_per_s": len(probs) / t_seq,
                                     "note": "one FP64 device Lanczos per problem, handle "
                                             "creation excluded"}
    out["max_abs_dE_vs_single_fp64"] = float(np.abs(es - e).max())
    out["max_rel_dE_vs_single_fp64"] = float((np.abs(es - e) / np.abs(es)).max())
    out["speedup_group_vs_single"] = t_seq / tg
    if cpu_sample:
        import oracle
        if oracle.ref_available():
            pick = [s for s, p in enumerate(probs) if p.dim <= 40000][:6]
            t_cpu, rel = 0.0, 0.0
            for s in pick:
                rk = oracle.RefKron(probs[s])
                xs = init[offs[s]:offs[s + 1]].cpu().numpy()
                t0 = time.perf_counter()
                e_ref, _, _ = rk.lanczos(xs, steps=200, min_steps=4, tolerance=1e-12, reortho=True)
                t_cpu += time.perf_counter() - t0
                rel = max(rel, abs(e_ref - e[s]) / abs(e_ref))
                del rk
            cores = int(os.environ.get("OPENBLAS_NUM_THREADS", os.cpu_count() or 1))
            out["cpu_reference"] = {
                "problems_per_s": len(pick) / t_cpu, "cores": cores, "kind": "reference",
                "max_rel_dE_group_vs_reference": rel,
                "sample": f"problems {pick} of the batch (dims "
                          f"{[int(probs[s].dim) for s in pick]}): PsimagLite::LanczosSolver "
                          "with Dmrg::BatchedGemmCpu, compiled from the reference sources"}
    return out


def ladder_measurements(torch, dev, stream):
    """Ladder-shaped sector (16000 x 16000 states, 241 (N_up, N_down) patches,
    K = 10, D = 3.37e6): the H*x throughput in FP64 and TF32x3, and one
    sector eigensolve as in a finite-sweep step, plain FP64 Lanczos against
    TF32x3 Lanczos + FP64 refinement (dmrgpp_b200.sweep)."""
    from dmrgpp_b200 import plugin, sweep
    from dmrgpp_b200 import superblock as sb
    prob = sb.ladder_problem()
    f = prob.flops()
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    bg = plugin.BatchedGemm.from_problem(prob, stream=stream.cuda_stream,
                                         precision=plugin.TF32X3)
    bg.set_precision(plugin.FP64)
    bg.autotune(None, reps=3)
    x = torch.from_numpy(np.random.default_rng(5).standard_normal(prob.dim)).to(dev)
    y = torch.empty_like(x)
    out = {"workload": prob.name, "sector_dim": prob.dim, "f_alg_per_matvec": f,
           "sites": 64}
    for name, prec in (("fp64", plugin.FP64), ("tf32x3", plugin.TF32X3)):
        bg.set_precision(prec)
        for _ in range(3):
            bg.apply_Htarget(x, y)
        ts = []
        for _ in range(10):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            bg.apply_Htarget(x, y)
            b.record(stream)
            ts.append((a, b))
        torch.cuda.synchronize()
        t = statistics.median(a.elapsed_time(b) for a, b in ts) / 1e3
        out[f"matvec_{name}"] = {"ms": t * 1e3, "tflops_alg": f / t / 1e12}
    bg.close()
    out["matvec_speedup_tf32x3_vs_fp64"] = out["matvec_fp64"]["ms"] / out["matvec_tf32x3"]["ms"]
    # the reference's default CPU path on this sector (its batched path's
    # dense nL x (nL K) slabs would need ~20 GB here)
    out["cpu_nonbatched_matvec"] = nonbatched_cpu(prob, f, calls=3)
    out["solve"] = sweep.sector_solves(prob, sites=64, mixed_steps=60, refine_inner=80,
                                       refine_inner_tolerance=1e-2,
                                       with_davidson=False)
    out["attribution"] = sweep.step_attribution(prob, sites=64, repeats=5)
    out["wft"] = wft_measurement(torch, prob, stream, flush)
    out["truncation"] = truncation_measurement(torch, prob, stream)
    # one whole sweep step of the sector: wave-function transformation (the
    # initial guess), the eigensolve, the truncation of the grown block
    at = out["attribution"]
    rest = out["wft"]["ms"] * 1e-3 + out["truncation"]["seconds"]
    fp64 = at["fp64_lanczos"]["median_seconds"] + rest
    mixed = at["mixed_refined"]["median_seconds"] + rest
    out["step"] = {"fp64_seconds": fp64, "mixed_seconds": mixed, "speedup": fp64 / mixed,
                   "solve_medians_of": at["repeats"],
                   "abs_dE_per_site": at["mixed_refined"]["abs_dE_per_site_vs_fp64_lanczos"],
                   "parts": "wft + solve + truncation (m = 4000 of 16000 states); the WFT and "
                            "truncation run in FP64 in both; solves: medians of the repeats"}
    return out


def truncation_measurement(torch, prob, stream, m: int = 4000):
    """Density-matrix truncation of the ladder sector's system block (the
    step after each sweep-step solve): rho_g = X_p^T X_p of all 241 groups
    (16000 states) by one grouped DGEMM on the device, the groups'
    eigenpairs on the host cores, m = 4000 states kept; against the oracle's
    numpy restatement (per-group X^T X and LAPACK eigh) on the host cores."""
    from dmrgpp_b200.truncation import density_truncate
    from oracle import truncation_oracle
    rng = np.random.default_rng(23)
    l, r = prob.lsz, prob.rsz
    psi_h = rng.standard_normal(prob.dim)
    psi_h /= np.linalg.norm(psi_h)
    psi = torch.from_numpy(psi_h).cuda()
    pg = list(range(prob.npatches))
    density_truncate(l, r, pg, l, 0, psi, m, stream=stream.cuda_stream)   # warm-up
    from dmrgpp_b200.truncation import truncation_profile
    runs = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = density_truncate(l, r, pg, l, 0, psi, m, stream=stream.cuda_stream)
        runs.append((time.perf_counter() - t0, truncation_profile()))
    t, phases = min(runs, key=lambda x: x[0])
    t0 = time.perf_counter()
    ref = truncation_oracle.truncate(l, r, pg, l, 0, [psi_h], m)
    t_cpu = time.perf_counter() - t0
    dw = max(float(np.abs(a - b).max()) for a, b in zip(out["eigenvalues"], ref["eigenvalues"]))
    return {"states": int(np.sum(l)), "groups": int(prob.npatches), "kept": out["kept_total"],
            "seconds": t, "phases": phases, "discarded": out["discarded"],
            "same_kept_per_group_as_oracle": bool(np.array_equal(out["kept"], ref["kept"])),
            "max_abs_eigenvalue_diff_vs_oracle": dw,
            "cpu_oracle": {"seconds": t_cpu, "cores": os.cpu_count(),
                           "kind": "port (numpy X^T X and LAPACK eigh per group)"}}


def wft_measurement(torch, prob, stream, flush):
    """Wave-function transformation of the ladder sector's vector (the step
    before each sweep-step solve: every patch block multiplied on both sides
    by its groups' transformation blocks, here square N(0,1)/sqrt(n) blocks),
    FP64 on the device against the oracle's per-patch numpy products on the
    host cores (the reference's BlockDiagWf::transform does the same GEMMs)."""
    from dmrgpp_b200.wft import WaveFunctionTransform
    from oracle import wft_oracle
    rng = np.random.default_rng(17)
    l, r = prob.lsz, prob.rsz
    src = list(range(prob.npatches))
    WL = [rng.standard_normal((int(n), int(n))) / np.sqrt(n) for n in l]
    WR = [rng.standard_normal((int(n), int(n))) / np.sqrt(n) for n in r]
    w = WaveFunctionTransform(l, r, l, r, src, WL, WR, stream=stream.cuda_stream)
    xh = rng.standard_normal(w.dim_in)
    x = torch.from_numpy(xh).cuda()
    y = torch.empty(w.dim_out, dtype=torch.float64, device=x.device)
    for _ in range(3):
        w(x, y)
    ts = []
    for _ in range(10):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        w(x, y)
        b.record(stream)
        ts.append((a, b))
    torch.cuda.synchronize()
    t = statistics.median(a.elapsed_time(b) for a, b in ts) / 1e3
    ref = wft_oracle.transform(xh, l, r, l, r, src, WL, WR)
    err = float(np.abs(y.cpu().numpy() - ref).max() / np.abs(ref).max())
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        wft_oracle.transform(xh, l, r, l, r, src, WL, WR)
    t_cpu = (time.perf_counter() - t0) / reps
    w.close()
    return {"flops": w.flops, "ms": t * 1e3, "tflops": w.flops / t / 1e12,
            "rel_err_vs_oracle": err,
            "cpu_oracle": {"ms": t_cpu * 1e3, "tflops": w.flops / t_cpu / 1e12,
                           "cores": os.cpu_count(), "kind": "port (numpy per-patch GEMMs)"}}


def rank_barrier(dist, world):
    """Every rank waits for the others (no-op on one rank)."""
    if world > 1:
        dist.barrier()


def reduce_max(dist, world, v, device):
    """The largest of the ranks' values (each rank passes its own time); every
    rank takes part, in the same order on every rank."""
    if world == 1:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from dmrgpp_b200 import plugin
    prob = make_problem(args.workload)
    f_alg = prob.flops()
    # one dedicated stream for the handle, the flush and the timing events
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    bg = plugin.BatchedGemm.from_problem(prob, stream=stream.cuda_stream, device=local)
    tuned_cfg, tuned_us = bg.autotune(None, reps=5)
    D = prob.dim
    x_host = torch.from_numpy(np.random.default_rng(100 + rank).standard_normal(D)).pin_memory()
    y_host = torch.empty(D, dtype=torch.float64).pin_memory()
    xd = x_host.to(dev)
    yd = torch.empty_like(xd)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def barrier():
        rank_barrier(dist, world)
        torch.cuda.synchronize(dev)

    def max_over_ranks(v):
        return reduce_max(dist, world, v, dev)

    # ---- device-resident timing: events around each matvec, L2 flushed
    # between steps (outside the events)
    for _ in range(args.warmup):
        bg.apply_Htarget(xd, yd)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    with clocks:
        barrier()
        clocks.active.set()
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            bg.apply_Htarget(xd, yd)
            ends[i].record(stream)
        barrier()
        clocks.active.clear()
    t_dev = sum(s.elapsed_time(e) for s, e in zip(starts, ends)) / 1e3
    t_dev = max_over_ranks(t_dev)
    value = world * f_alg * args.steps / t_dev / 1e12
    per_launch_s = t_dev / args.steps

    # ---- end to end through the C ABI with host buffers (H2D + D2H inside)
    xh, yh = x_host.numpy(), y_host.numpy()
    for _ in range(max(3, args.warmup // 4)):
        bg.apply_Htarget(xh, yh)
    e_st = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e_en = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    for i in range(args.steps):
        flush.zero_()
        e_st[i].record(stream)
        bg.apply_Htarget(xh, yh)        # synchronous: copy in, one kernel, copy out
        e_en[i].record(stream)
    barrier()
    t_e2e = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(e_st, e_en)) / 1e3)
    e2e = world * f_alg * args.steps / t_e2e / 1e12

    # ---- sanity: the result the timing produced is H*x
    if rank == 0:
        import oracle
        y_chk = oracle.kron_apply(prob, xh)
        err = float(np.abs(yh - y_chk).max() / np.abs(y_chk).max())
        if err > 1e-12:
            raise SystemExit(f"bench result differs from the oracle: rel err {err:.3e}")

    mixed_c2 = None
    if rank == 0 and world == 1 and args.workload == "c2":
        mixed_c2 = mixed_matvec_measurement(torch, dev, stream, prob, xh, yh, f_alg)
    peak = measured_fp64_peak(torch, dev) if rank == 0 else None
    bg.close()
    sweep_step = serving = None
    if rank == 0 and world == 1 and not args.no_sweep:
        sweep_step = ladder_measurements(torch, dev, stream)
    if rank == 0 and world == 1 and not args.no_serving:
        serving = serving_measurements(torch, dev, stream, cpu_sample=not args.no_cpu_baseline)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    achieved = f_alg / per_launch_s / 1e12
    # the sweep-step and serving results as short keys near the start of the
    # line (the full records follow at its end)
    short = {}
    if sweep_step is not None:
        short.update(sweep_step_speedup=sweep_step["step"]["speedup"],
                     sweep_step_solve_speedup=sweep_step["attribution"]["total_gain"],
                     sweep_step_precision_gain=sweep_step["attribution"]["precision_gain"],
                     sweep_step_abs_dE_per_site=sweep_step["step"]["abs_dE_per_site"])
    if serving is not None:
        short.update(serving_problems_per_s=serving["group_mixed"]["problems_per_s"],
                     serving_problems_per_s_fp64=serving["group_lanczos"]["problems_per_s"])
    kernel = ("kron_fused_kernel (both passes per output tile, cluster reduction; one launch)"
              if tuned_cfg >= 6 else
              "kron_persistent_kernel (both passes of one matvec in one launch)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        **short,
        "data": "synthetic (seeded N(0,1) sector blocks)",
        "config": dict(workload_config(prob, args.workload),
                       precision=args.precision,
                       l2="flushed between timed steps (256 MiB write outside the events)",
                       parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 8 * D,
                "d2h_bytes_per_step": 8 * D,
                "ms_per_step": t_e2e / args.steps * 1e3,
                "path": "dmrgpp_kron_apply(host x, host y) through the C ABI, pinned buffers"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": UNIT,
                     "frac": achieved / peak if peak else None,
                     "traffic": read_traffic(args.workload,
                                             "kron_fused" if tuned_cfg >= 6 else "kron_persistent"),
                     "kernel": kernel,
                     "peak_source": "measured live: cuBLAS DGEMM 8192^3 FP64 (no FP64 entry "
                                    "in MEASURED_PEAKS.json)"},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
        "tuning": {"tile_config": tuned_cfg, "autotune_best_us": tuned_us},
    }
    if mixed_c2 is not None:
        line["mixed_precision"] = mixed_c2
    if sweep_step is not None:
        line["sweep_step"] = sweep_step
    if serving is not None:
        line["serving"] = serving
    if not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(prob, f_alg)
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


def profile_case(argv) -> int:
    """The workloads of the ncu summaries under profiles/ (see the module
    docstring): a fixed number of applies or one solve, nothing else."""
    p = argparse.ArgumentParser(prog="bench.py --profile-case")
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
    from dmrgpp_b200 import plugin
    from dmrgpp_b200 import superblock as sb

    if a.workload == "mlp":
        import numpy as np
        from dmrgpp_b200.mlp import MLPPreconditioner
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
        from dmrgpp_b200.wft import WaveFunctionTransform
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
        from dmrgpp_b200.truncation import density_truncate
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
    if len(sys.argv) > 1 and sys.argv[1] == "--profile-case":
        sys.exit(profile_case(sys.argv[2:]))
    sys.exit(main())
