"""KronLogger files: the reference's text dump of one superblock H*v (the
input vector and every (outPatch, inPatch, connection) pair of A and B
blocks), read into plugin tables so real superblocks recorded by DMRG++ can
be replayed through this library, and written from plugin tables in the same
format.

Format (dmrg/Engine/MatrixVectorKron/KronLogger.hh:112-174): a line
"Vector", the vector length, the entries one per line; then per logged
connection a header line "# nc, total, outPatch, inPatch, ic, applyAdjoint,
performTranspose, offsetX, offsetY", its nine integers, "## A: <format>" and
the block, "## B: <format>" and the block.  A block is either dense ("rows
cols" then one row per line) or MatrixMarket (coordinate, 1-based).  Records
with performTranspose (the stored lower block, KronConnections.h:141-172) or
applyAdjoint carry the block of the transposed pair and are applied
transposed.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .superblock import KronProblem


def _read_matrix(lines: List[str], pos: int):
    head = lines[pos].strip()
    if head.startswith("%%MatrixMarket"):
        q = pos + 1
        while lines[q].lstrip().startswith("%"):
            q += 1
        rows, cols, nnz = map(int, lines[q].split())
        m = np.zeros((rows, cols))
        for t in range(nnz):
            i, j, v = lines[q + 1 + t].split()
            m[int(i) - 1, int(j) - 1] = float(v)
        return m, q + 1 + nnz
    rows, cols = map(int, head.split())
    m = np.array([[float(x) for x in lines[pos + 1 + r].split()] for r in range(rows)])
    return m.reshape(rows, cols), pos + 1 + rows


def read_kronlog(path: str, name: str = "") -> Tuple[KronProblem, np.ndarray]:
    """(problem, logged vector) of a KronLogger file.  Patch sizes come from
    the block shapes, and the logged offsets are checked against the patch
    layout."""
    lines = open(path).read().splitlines()
    pos = lines.index("Vector")
    n = int(lines[pos + 1])
    vin = np.array([float(lines[pos + 2 + i]) for i in range(n)])
    pos = pos + 2 + n
    recs = []
    npatch = None
    nc = None
    while pos < len(lines):
        if lines[pos].startswith("# nc, total"):
            nc, npatch, outp, inp, ic, adj, tr, offx, offy = (int(x) for x in lines[pos + 1].split())
            if not lines[pos + 2].startswith("## A:"):
                raise ValueError(f"{path}:{pos + 3}: expected '## A:'")
            A, pos = _read_matrix(lines, pos + 3)
            if not lines[pos].startswith("## B:"):
                raise ValueError(f"{path}:{pos + 1}: expected '## B:'")
            B, pos = _read_matrix(lines, pos + 1)
            if tr or adj:
                A, B = A.T, B.T
            recs.append((outp, inp, ic, offx, offy, A, B))
        else:
            pos += 1
    if npatch is None:
        raise ValueError(f"{path}: no connection records")
    lsz = np.zeros(npatch, dtype=np.int64)
    rsz = np.zeros(npatch, dtype=np.int64)
    offs: List[Tuple[int, int]] = []
    Ad, Bd = {}, {}
    for outp, inp, ic, offx, offy, A, B in recs:
        lsz[outp], rsz[outp] = A.shape[0], B.shape[0]
        lsz[inp], rsz[inp] = A.shape[1], B.shape[1]
        offs += [(outp, offx), (inp, offy)]
        Ad[(outp, inp, ic)] = np.asfortranarray(A)
        Bd[(outp, inp, ic)] = np.asfortranarray(B)
    if (lsz == 0).any():
        raise ValueError(f"{path}: patches without any logged block: {np.where(lsz == 0)[0]}")
    prob = KronProblem(lsz, rsz, nc, Ad, Bd, name=name or path)
    if prob.dim != n:
        raise ValueError(f"{path}: vector length {n} != sector dimension {prob.dim}")
    for p, o in offs:
        if prob.xy_start[p] != o:
            raise ValueError(f"{path}: patch {p} offset {o} != {prob.xy_start[p]}")
    return prob, vin


def write_kronlog(prob: KronProblem, v: np.ndarray, path: str) -> None:
    """Writes prob and v in the KronLogger layout (dense blocks, no
    transposition flags), one record per contributing (out, in, k)."""
    with open(path, "w") as f:
        f.write("Vector\n%d\n" % len(v))
        for x in v:
            f.write("%.17g\n" % x)
        xs = prob.xy_start
        for (i, j, k) in sorted(prob.A, key=lambda t: (t[2], t[0], t[1])):
            if (i, j, k) not in prob.B:
                continue
            A, B = prob.A[(i, j, k)], prob.B[(i, j, k)]
            f.write("\n# nc, total, outPatch, inPatch, ic, applyAdjoint, performTranspose, "
                    "offsetX, offsetY\n")
            f.write("%d %d %d %d %d 0 0 %d %d\n" % (prob.noperator, prob.npatches, i, j, k,
                                                    xs[i], xs[j]))
            for tag, m in (("A", A), ("B", B)):
                f.write("## %s: dense\n%d %d\n" % (tag, m.shape[0], m.shape[1]))
                for row in np.asarray(m):
                    f.write(" ".join("%.17g" % x for x in row) + "\n")
