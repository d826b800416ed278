"""dmrgpp_kron_apply_noalloc: the one-shot H*x for callers that cannot call
cudaMalloc (its scratch is a fixed device array inside the library).

Checked through the C ABI against the allocating path (dmrgpp_kron_create +
dmrgpp_kron_apply) on two calls in a row with different sectors, so that a
second call cannot lean on what the first left in the shared array.  This
file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

RTOL = 1e-12


def _desc(prob, stream=None):
    from dmrgpp_b200 import plugin
    A, ldA, B, ldB = prob.tables()
    return plugin._DescTables(prob.noperator, prob.npatches, prob.lsz, prob.rsz, A, ldA, B, ldB,
                              0, stream, -1)


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _sparse_second_sector():
    """A sector smaller than the microbench one, with all-zero blocks and an
    output patch that no term reaches (its part of y must come out 0)."""
    prob = sb.random_problem(npatches=7, noperator=4, max_size=90, seed=21, zero_block_rate=0.3)
    for key in [k for k in prob.A if k[0] == 3]:
        del prob.A[key]
        del prob.B[key]
    some = sorted(prob.A)[:3]
    for key in some:                       # present but all zero: not a term
        prob.A[key] = np.zeros_like(prob.A[key], order="F")
    return prob


def _noalloc_apply(cuda_lib, cuda_device, prob, x, stream):
    import torch
    from dmrgpp_b200 import _capi
    t = _desc(prob, stream)
    xd = torch.from_numpy(x).to(cuda_device)
    yd = torch.full_like(xd, float("nan"))
    rc = cuda_lib.dmrgpp_kron_apply_noalloc(ctypes.byref(t.desc), ctypes.c_void_p(xd.data_ptr()),
                                            ctypes.c_void_p(yd.data_ptr()))
    assert rc == _capi.OK, cuda_lib.dmrgpp_kron_noalloc_last_error()
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(cuda_lib, cuda_device):
    """Two calls in a row: the microbench sector, then a smaller sector with
    all-zero blocks and an output patch without terms, which starts from the
    scratch the larger call left behind (y prefilled with NaN each time)."""
    import torch
    from dmrgpp_b200 import plugin

    stream = torch.cuda.current_stream().cuda_stream
    second = _sparse_second_sector()
    for prob, seed in ((sb.c2_problem(seed=3), 1), (second, 2)):
        x = sb.random_unit_vector(prob.dim, seed=seed)
        bg = plugin.BatchedGemm.from_problem(prob, stream=stream)
        y_alloc = bg(x)
        bg.close()
        y_noalloc = _noalloc_apply(cuda_lib, cuda_device, prob, x, stream)
        assert np.isfinite(y_noalloc).all()
        assert _rel(y_noalloc, y_alloc) < RTOL
    s3 = second.xy_start
    assert np.all(y_noalloc[s3[3]:s3[4]] == 0.0)


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream(cuda_lib, cuda_device):
    """Its uploads read host memory freed when the call returns, so a call on
    a stream under capture is refused before any device work; the capture
    itself stays valid."""
    import torch
    from dmrgpp_b200 import _capi
    prob = sb.c2_problem(seed=3)
    x = torch.from_numpy(sb.random_unit_vector(prob.dim, seed=1)).to(cuda_device)
    y = torch.zeros_like(x)
    side = torch.cuda.Stream(cuda_device)
    t = _desc(prob, side.cuda_stream)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        y.add_(x)
        rc = cuda_lib.dmrgpp_kron_apply_noalloc(ctypes.byref(t.desc), ctypes.c_void_p(x.data_ptr()),
                                                ctypes.c_void_p(y.data_ptr()))
    assert rc == _capi.NOT_SUPPORTED
    assert "captured" in cuda_lib.dmrgpp_kron_noalloc_last_error().decode()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, x)
    del g


def test_noalloc_rejects_sectors_beyond_its_scratch(cuda_lib):
    """Size check happens before any device work."""
    from dmrgpp_b200 import _capi
    big = sb.spin_chain_like(sb.gaussian_sector_sizes(2048, 21, 4.0), seed=5)
    t = _desc(big)
    rc = cuda_lib.dmrgpp_kron_apply_noalloc(ctypes.byref(t.desc), ctypes.c_void_p(16),
                                            ctypes.c_void_p(16))
    assert rc == _capi.INVALID_ARG
    msg = cuda_lib.dmrgpp_kron_noalloc_last_error().decode()
    assert "scratch" in msg and str(_capi.NOALLOC_SCRATCH_BYTES) in msg
