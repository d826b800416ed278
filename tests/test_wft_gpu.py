"""Parity of the patch-wise wave-function transformation (dmrgpp_wft_*)
with the numpy oracle (oracle/wft_oracle.py), FP64 bar 1e-12 relative; host
and device pointers; truncating (rectangular) transforms; output patches
without a source; the full 16000-state ladder layout."""
import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _layout(rng, npi, npo, maxs, empty_rate=0.15):
    l_in = rng.integers(1, maxs + 1, npi)
    r_in = rng.integers(1, maxs + 1, npi)
    l_out = rng.integers(1, maxs + 1, npo)
    r_out = rng.integers(1, maxs + 1, npo)
    src = [int(rng.integers(0, npi)) if rng.random() > empty_rate else -1 for _ in range(npo)]
    return l_in, r_in, l_out, r_out, src


def _blocks(rng, l_in, r_in, l_out, r_out, src, tl, tr):
    WL, WR = [], []
    for q, p in enumerate(src):
        if p < 0:
            WL.append(None)
            WR.append(None)
            continue
        wl = rng.standard_normal((l_out[q], l_in[p]))
        wr = rng.standard_normal((r_out[q], r_in[p]))
        WL.append(wl.T.copy() if tl else wl)
        WR.append(wr.T.copy() if tr else wr)
    return WL, WR


def rel_err(y, ref):
    return float(np.abs(y - ref).max() / max(np.abs(ref).max(), 1e-300))


@pytest.mark.parametrize("seed,npi,npo,maxs,tl,tr", [
    (0, 1, 1, 1, 0, 0), (1, 4, 5, 20, 0, 0), (2, 6, 6, 70, 1, 0), (3, 5, 7, 33, 0, 1),
    (4, 3, 3, 200, 1, 1), (5, 10, 12, 50, 0, 0), (6, 2, 4, 130, 1, 1)])
def test_random_layouts_match_oracle(cuda_lib, cuda_device, seed, npi, npo, maxs, tl, tr):
    from dmrgpp_b200.wft import WaveFunctionTransform
    from oracle import wft_oracle
    rng = np.random.default_rng(seed)
    lay = _layout(rng, npi, npo, maxs)
    WL, WR = _blocks(rng, *lay, tl, tr)
    w = WaveFunctionTransform(*lay, WL, WR, trans_WL=bool(tl), trans_WR=bool(tr))
    x = rng.standard_normal(w.dim_in)
    y = w(x)
    ref = wft_oracle.transform(x, *lay, WL, WR, trans_WL=bool(tl), trans_WR=bool(tr))
    assert rel_err(y, ref) < RTOL
    assert w.flops == pytest.approx(wft_oracle.flops(*lay))
    for q, p in enumerate(lay[4]):   # outputs without a source are zero
        if p < 0:
            ys = np.concatenate([[0], np.cumsum(lay[2] * lay[3])])
            assert not np.any(y[ys[q]:ys[q + 1]])
    w.close()


def test_device_pointers_match_host_pointers(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200.wft import WaveFunctionTransform
    rng = np.random.default_rng(11)
    lay = _layout(rng, 8, 8, 90, empty_rate=0.0)
    WL, WR = _blocks(rng, *lay, 0, 0)
    w = WaveFunctionTransform(*lay, WL, WR)
    x = rng.standard_normal(w.dim_in)
    y_host = w(x)
    y_dev = w(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(y_dev.cpu().numpy(), y_host)
    w.close()


def test_ladder_layout_orthogonal_and_truncating(cuda_lib, cuda_device):
    """Full 16000-state ladder layout (241 patches): orthogonal square
    transforms keep the norm; a truncating transform (each left group cut to
    80% of its states, rows of an orthogonal matrix) matches the oracle."""
    from dmrgpp_b200.wft import WaveFunctionTransform
    from oracle import wft_oracle
    prob = sb.ladder_problem()
    rng = np.random.default_rng(3)
    l, r = prob.lsz, prob.rsz
    src = list(range(prob.npatches))

    def orth(n):
        q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        return q
    WL = [orth(int(n)) for n in l]
    WR = [orth(int(n)) for n in r]
    w = WaveFunctionTransform(l, r, l, r, src, WL, WR)
    x = rng.standard_normal(w.dim_in)
    y = w(x)
    assert abs(np.linalg.norm(y) / np.linalg.norm(x) - 1.0) < 1e-12
    w.close()
    l_out = np.maximum(1, (8 * l) // 10)
    WLt = [WL[p][:int(l_out[p]), :] for p in range(prob.npatches)]
    w = WaveFunctionTransform(l, r, l_out, r, src, WLt, WR)
    y = w(x)
    assert rel_err(y, wft_oracle.transform(x, l, r, l_out, r, src, WLt, WR)) < RTOL
    assert np.linalg.norm(y) <= np.linalg.norm(x) * (1 + 1e-12)
    w.close()
