"""Per-step superblock energies of whole DMRG runs with the reference's own
sector solver (PsimagLite::LanczosSolver over Dmrg::BatchedGemmCpu, compiled
into oracle/_ref), for the GPU tests that repeat the runs with the CUDA
solver.  Run here:  python tests/golden/make_dmrg_golden.py

* dmrg_heisenberg_L32_m128.json -- spin-1/2 Heisenberg chain, L=32, open
  boundaries, Sz=0, m=128, infinite growth + 2 finite sweeps, Lanczos
  eps 1e-10 (the plain-method configuration); the reference's own test of
  this chain expects -13.9973 within 2e-5 (dmrg/CMakeLists.txt:343-344,
  TestSuite/inputs/input3100.ain).
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import dmrg_driver as dd  # noqa: E402


def heisenberg_L32():
    d = dd.DMRG(dd.Heisenberg(), L=32, m=128, solver=dd.reference_solver(tolerance=1e-10))
    e = d.run(sweeps=2)
    out = {"model": "heisenberg", "L": 32, "m": 128, "sweeps": 2, "seed": 7,
           "lanczos_eps": 1e-10, "energy": e, "energies": d.energies,
           "reference_test_energy": -13.9973, "reference_test_tolerance": 2e-5,
           "source": "dmrg/CMakeLists.txt:343-344 (input3100)"}
    with open(os.path.join(HERE, "dmrg_heisenberg_L32_m128.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("Heisenberg L=32 m=128:", e, "steps", len(d.energies))


if __name__ == "__main__":
    oracle.build()
    heisenberg_L32()
