"""Seeded CRS operator sets for the CRS set-up tests (shared by the CPU and
GPU tests): a left and a right basis split into quantum-number groups,
patches pairing left group g with right group G-1-g, K terms H_L x I,
I x H_R and hopping-like links between neighbouring groups (sparse within
their blocks, some fermionic, with factors), as CRS triples."""
import numpy as np


def random_crs_case(seed, ngroups=5, maxg=30, K=5, density=0.35):
    rng = np.random.default_rng(seed)
    gl = rng.integers(1, maxg + 1, ngroups)
    gr = rng.integers(1, maxg + 1, ngroups)
    loff = np.concatenate([[0], np.cumsum(gl)])
    roff = np.concatenate([[0], np.cumsum(gr)])
    nL, nR = int(loff[-1]), int(roff[-1])
    # patches: left group g with right group ngroups-1-g, all but one group
    pats = [g for g in range(ngroups) if g != ngroups // 2] if ngroups > 2 else list(range(ngroups))
    lo = [int(loff[g]) for g in pats]
    ls = [int(gl[g]) for g in pats]
    ro = [int(roff[ngroups - 1 - g]) for g in pats]
    rs = [int(gr[ngroups - 1 - g]) for g in pats]

    def csr(dense):
        ip, ix, dv = [0], [], []
        for a in range(dense.shape[0]):
            nz = np.nonzero(dense[a])[0]
            ix.extend(int(b) for b in nz)
            dv.extend(float(dense[a, b]) for b in nz)
            ip.append(len(ix))
        return (np.array(ip, dtype=np.int32), np.array(ix, dtype=np.int32), np.array(dv))

    def block_op(n, off, sizes, couple, sym):
        M = np.zeros((n, n))
        for g in range(len(sizes)):
            for h in range(len(sizes)):
                if not couple(g, h):
                    continue
                blk = rng.standard_normal((sizes[g], sizes[h]))
                blk[rng.random(blk.shape) > density] = 0.0
                M[off[g]:off[g + 1], off[h]:off[h + 1]] = blk
        return M + M.T if sym else M

    A, B, val, fer = [], [], [], []
    A.append(csr(block_op(nL, loff, gl, lambda g, h: g == h, True)))      # H_L x I
    B.append(csr(np.eye(nR)))
    val.append(1.0)
    fer.append(0)
    A.append(csr(np.eye(nL)))                                              # I x H_R
    B.append(csr(block_op(nR, roff, gr, lambda g, h: g == h, True)))
    val.append(1.0)
    fer.append(0)
    for k in range(2, K):                                                  # links
        d = 1 if k % 2 else -1
        A.append(csr(block_op(nL, loff, gl, lambda g, h: h == g + d, False)))
        B.append(csr(block_op(nR, roff, gr, lambda g, h: h == g - d, False)))
        val.append(float(rng.choice([0.5, -1.0, 1.7])))
        fer.append(int(k % 3 == 0))
    parity = rng.integers(0, 2, nL).astype(np.uint8)
    return dict(loff=lo, lsz=ls, roff=ro, rsz=rs, A=A, B=B, value=val, fermion=fer,
                parity=parity, nL=nL, nR=nR)
