"""CRS operators sliced into per-patch dense blocks, restated in numpy.

TEST INFRASTRUCTURE (oracle): only tests/ use it, as the checker of
dmrgpp_kron_create_crs.  It restates the reference's InitKron set-up:
InitKronBase::calculateAhat (InitKronBase.h:393-413: Ahat(a, :) =
A(a, :) * sign * value, sign = -1 for a fermionic term on an odd left state)
and ArrayOfMatStruct (ArrayOfMatStruct.h:105-448: the operator restricted to
the rows of patch i's group and the columns of patch j's group), densified as
the batched path does (BatchedGemmKokkos.h:354-370), into the plugin's block
tables.
"""
from __future__ import annotations

import numpy as np

from dmrgpp_b200.superblock import KronProblem


def ahat_values(indptr, data, value=1.0, fermion=False, parity=None):
    """calculateAhat on the CRS values: a * sign * value, in that order."""
    out = np.array(data, dtype=np.float64, copy=True)
    for a in range(len(indptr) - 1):
        sign = -1.0 if (fermion and parity[a]) else 1.0
        for e in range(indptr[a], indptr[a + 1]):
            out[e] = out[e] * sign * value
    return out


def dense_block(indptr, indices, data, r0, nr, c0, nc):
    """Rows [r0, r0 + nr) x columns [c0, c0 + nc) of a CRS matrix, dense,
    column-major."""
    blk = np.zeros((nr, nc), order="F")
    for a in range(r0, r0 + nr):
        for e in range(indptr[a], indptr[a + 1]):
            b = indices[e]
            if c0 <= b < c0 + nc:
                blk[a - r0, b - c0] = data[e]
    return blk


def problem_from_crs(loff, lsz, roff, rsz, A, B, value=None, fermion=None, parity=None,
                     name="crs-sector"):
    """KronProblem of the blocks; A and B are lists of (indptr, indices, data)
    over the left and right bases.  Blocks that are all zero are left out (as
    the plugin's all-zero test leaves them out)."""
    K = len(A)
    np_ = len(lsz)
    At, Bt = {}, {}
    for k in range(K):
        v = 1.0 if value is None else float(value[k])
        f = bool(fermion[k]) if fermion is not None else False
        ip, ix, dv = A[k]
        ah = ahat_values(ip, dv, v, f, parity)
        bp, bx, bv = B[k]
        for i in range(np_):
            for j in range(np_):
                a = dense_block(ip, ix, ah, loff[i], lsz[i], loff[j], lsz[j])
                b = dense_block(bp, bx, bv, roff[i], rsz[i], roff[j], rsz[j])
                if np.any(a != 0.0) and np.any(b != 0.0):
                    At[(i, j, k)] = a
                    Bt[(i, j, k)] = b
    return KronProblem(np.asarray(lsz, dtype=np.int64), np.asarray(rsz, dtype=np.int64), K, At, Bt,
                       name=name)
