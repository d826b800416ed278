"""ORACLE -- test infrastructure only.  FP64 numpy restatement of the
patch-wise wave-function transformation (the GEMM core of the reference's
WftAccelPatches::operator(), Wft/WftAccelPatches.h:43-66, through
BlockDiagWf::transform, BlockDiagWf.h:525-557, and
ParallelBlockTransform::doTask, BlockDiagWf.h:131-260: per patch
Ynew = opL(W_L) * Yold * opR(W_R)).  In the sector layout of this library a
patch block is r x l column-major, so the same product reads
Y_q = WR_q X_p WL_q^T with WL = opL(W_L) and WR = opR(W_R)^T; output patches
without a source are zero.  Used by tests/ and bench.py's CPU baseline only."""
import numpy as np


def transform(x, l_in, r_in, l_out, r_out, src, WL, WR, trans_WL=False, trans_WR=False):
    """x: input sector vector (patch blocks r_in[p] x l_in[p], column-major);
    WL[q], WR[q]: the applied blocks (stored transposed when trans_*).
    Returns the output sector vector."""
    xs = np.concatenate([[0], np.cumsum(np.asarray(l_in, dtype=np.int64) * np.asarray(r_in, dtype=np.int64))])
    ys = np.concatenate([[0], np.cumsum(np.asarray(l_out, dtype=np.int64) * np.asarray(r_out, dtype=np.int64))])
    y = np.zeros(int(ys[-1]))
    for q, p in enumerate(src):
        if p < 0:
            continue
        X = np.asarray(x[xs[p]:xs[p + 1]]).reshape(int(l_in[p]), int(r_in[p])).T   # r_in x l_in
        wl = np.asarray(WL[q]).T if trans_WL else np.asarray(WL[q])                 # l_out x l_in
        wr = np.asarray(WR[q]).T if trans_WR else np.asarray(WR[q])                 # r_out x r_in
        Y = wr @ X @ wl.T                                                           # r_out x l_out
        y[ys[q]:ys[q + 1]] = Y.T.ravel()
    return y


def flops(l_in, r_in, l_out, r_out, src):
    return float(sum(2.0 * r_out[q] * l_in[p] * (r_in[p] + l_out[q])
                     for q, p in enumerate(src) if p >= 0))
