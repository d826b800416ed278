"""Generates the golden fixtures in this folder from the reference tree.

Run here (it needs the reference sources and the oracle harness built from
them):  python tests/golden/make_golden.py

* batchedgemm_1patch.json -- the known-answer case of the reference unit test
  dmrg/Engine/tests/test_BatchedGemm.cpp:171-259: one patch, one operator,
  A 2x2, B 3x3, vin of 6 entries, all drawn from std::mt19937_64(123456789)
  with std::uniform_real_distribution<double>(-1,1) in the test's order; the
  expected Y = B X A^T is recomputed by the test's own loops and by the
  reference BatchedGemmCpu compiled from its sources.
* kron_data31.npz -- the H*v dump TestSuite/inputs/kron_data31_0_ref.txt
  (KronLogger format, read by dmrgpp_b200.kronlog.read_kronlog; Heisenberg
  L=8) as plugin tables.  The file has no output vector; y is computed by the
  reference BatchedGemmCpu and stored with the fixture.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("DMRGPP_REFERENCE_TREE", "/root/reference")  # read-only source tree
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from dmrgpp_b200.superblock import KronProblem  # noqa: E402

RNG_PROGRAM = r"""
#include <cstdio>
#include <random>
int main() {
  std::mt19937_64 rng(123456789);
  std::uniform_real_distribution<double> dist(-1.0, 1.0);
  double A[2][2], B[3][3], v[6];
  for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) A[i][j] = dist(rng);
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) B[i][j] = dist(rng);
  for (int i = 0; i < 6; i++) v[i] = dist(rng);
  for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) std::printf("%.17g\n", A[i][j]);
  for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) std::printf("%.17g\n", B[i][j]);
  for (int i = 0; i < 6; i++) std::printf("%.17g\n", v[i]);
}
"""


def batchedgemm_1patch():
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "rng.cpp")
        exe = os.path.join(d, "rng")
        open(src, "w").write(RNG_PROGRAM)
        subprocess.run(["g++", "-O0", "-o", exe, src], check=True)
        vals = [float(s) for s in subprocess.run([exe], capture_output=True, text=True,
                                                  check=True).stdout.split()]
    A = np.array(vals[0:4]).reshape(2, 2)      # A(i,j) filled row by row
    B = np.array(vals[4:13]).reshape(3, 3)
    vin = np.array(vals[13:19])
    X = vin.reshape(2, 3).T                    # X(row,col) = vin[row + col*3]
    Y = np.zeros((3, 2))
    BX = np.zeros((3, 2))
    for i in range(3):                          # the test's own loops
        for j in range(2):
            BX[i, j] = sum(B[i, k] * X[k, j] for k in range(3))
    for i in range(3):
        for j in range(2):
            Y[i, j] = sum(BX[i, k] * A[j, k] for k in range(2))
    expected = Y.T.reshape(-1)                  # expected[row + col*3]
    prob = KronProblem(np.array([2]), np.array([3]), 1,
                       {(0, 0, 0): np.asfortranarray(A)}, {(0, 0, 0): np.asfortranarray(B)},
                       name="test_BatchedGemm-1patch")
    yref = oracle.RefKron(prob).apply(vin)
    assert np.allclose(yref, expected, rtol=1e-14, atol=1e-15)
    out = {"source": "dmrg/Engine/tests/test_BatchedGemm.cpp:171-259",
           "A": A.tolist(), "B": B.tolist(), "vin": vin.tolist(),
           "expected": expected.tolist(), "reference_batched_gemm_cpu": yref.tolist()}
    with open(os.path.join(HERE, "batchedgemm_1patch.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("batchedgemm_1patch.json: max |ref - expected| =", np.abs(yref - expected).max())


def kron_data31():
    from dmrgpp_b200.kronlog import read_kronlog
    path = os.path.join(REF, "TestSuite", "inputs", "kron_data31_0_ref.txt")
    prob, vin = read_kronlog(path, name="kron_data31")
    Ad, Bd = prob.A, prob.B
    y = oracle.RefKron(prob).apply(vin)
    rq = float(vin @ y / (vin @ vin))
    keys = sorted(Ad)
    np.savez_compressed(
        os.path.join(HERE, "kron_data31.npz"), lsz=prob.lsz, rsz=prob.rsz,
        noperator=prob.noperator, vin=vin, y_reference=y, rayleigh=rq,
        keys=np.array(keys, dtype=np.int64),
        A=np.concatenate([Ad[k].ravel(order="F") for k in keys]),
        B=np.concatenate([Bd[k].ravel(order="F") for k in keys]),
        source=np.array("TestSuite/inputs/kron_data31_0_ref.txt"))
    print("kron_data31.npz: patches", prob.npatches, "records", len(keys), "dim", prob.dim,
          "Rayleigh quotient", rq)


def load_kron_data31():
    z = np.load(os.path.join(HERE, "kron_data31.npz"))
    lsz, rsz = z["lsz"], z["rsz"]
    Ad, Bd = {}, {}
    pa = pb = 0
    for i, j, k in z["keys"]:
        i, j, k = int(i), int(j), int(k)
        na, nb = lsz[i] * lsz[j], rsz[i] * rsz[j]
        Ad[(i, j, k)] = np.asfortranarray(z["A"][pa:pa + na].reshape(lsz[j], lsz[i]).T)
        Bd[(i, j, k)] = np.asfortranarray(z["B"][pb:pb + nb].reshape(rsz[j], rsz[i]).T)
        pa += na
        pb += nb
    prob = KronProblem(lsz, rsz, int(z["noperator"]), Ad, Bd, name="kron_data31")
    return prob, z["vin"], z["y_reference"], float(z["rayleigh"])


if __name__ == "__main__":
    oracle.build()
    batchedgemm_1patch()
    kron_data31()
    prob, vin, y, rq = load_kron_data31()
    assert np.allclose(oracle.kron_apply(prob, vin), y, rtol=1e-13, atol=1e-15)


def lanczos_fixtures():
    """Lowest eigenpairs by the reference's PsimagLite::LanczosSolver (compiled
    from the reference sources, matvec = the reference BatchedGemmCpu) from
    seeded initial vectors, with reortho, LanczosEps 1e-12, 200 steps."""
    from dmrgpp_b200 import superblock as sb
    out = {}
    cases = {"kron_data31": load_kron_data31()[0],
             "random_sym_6x3": sb.random_problem(6, 3, max_size=14, seed=77, symmetric=True),
             "microbench_1024": sb.c2_problem()}
    for name, prob in cases.items():
        init = np.random.default_rng(2024).standard_normal(prob.dim)
        rk = oracle.RefKron(prob)
        e, z, steps = rk.lanczos(init, steps=200, min_steps=4, tolerance=1e-12, reortho=True)
        exact = None
        if prob.dim <= 3000:
            exact = float(np.linalg.eigvalsh(prob.dense())[0])
        out[name] = {"energy": e, "steps": steps, "dim": prob.dim, "exact": exact,
                     "init_seed": 2024, "z_head": z[:8].tolist(),
                     "z_norm": float(np.linalg.norm(z))}
        print(name, "E =", repr(e), "steps", steps, "exact", exact)
    with open(os.path.join(HERE, "lanczos_reference.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__" and "--lanczos" in sys.argv:
    lanczos_fixtures()
