"""ORACLE -- test infrastructure only.  numpy restatement of the sector
H*x for complex blocks (the reference's BatchedGemm<std::complex<double>>,
BatchedGemm.cpp:117-119, and the per-block method 1 of den_kron_mult.cpp:
75-180, both templated on ComplexOrRealType): Y_i = sum_{j,k} B_k(i,j) X_j
A_k(i,j)^T with plain (unconjugated) transposes, patch blocks r x l
column-major in patch order."""
import numpy as np


def kron_apply(lsz, rsz, A, B, x):
    """A, B: dicts (i, j, k) -> complex blocks; x: complex sector vector."""
    lsz = np.asarray(lsz, dtype=np.int64)
    rsz = np.asarray(rsz, dtype=np.int64)
    xs = np.concatenate([[0], np.cumsum(lsz * rsz)])
    y = np.zeros(int(xs[-1]), dtype=np.complex128)
    for (i, j, k), a in A.items():
        b = B.get((i, j, k))
        if b is None:
            continue
        X = np.asarray(x[xs[j]:xs[j + 1]]).reshape(int(lsz[j]), int(rsz[j])).T
        Y = np.asarray(b) @ X @ np.asarray(a).T
        y[xs[i]:xs[i + 1]] += Y.T.ravel()
    return y
