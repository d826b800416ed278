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


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_twice(cuda_lib, cuda_device):
    import torch
    from dmrgpp_b200 import _capi, plugin

    stream = torch.cuda.current_stream().cuda_stream
    first = sb.c2_problem(seed=3)
    second = sb.random_problem(npatches=7, noperator=4, max_size=90, seed=21,
                               zero_block_rate=0.0)
    for prob, seed in ((first, 1), (second, 2)):
        x = sb.random_unit_vector(prob.dim, seed=seed)
        bg = plugin.BatchedGemm.from_problem(prob, stream=stream)
        y_alloc = bg(x)
        bg.close()

        t = _desc(prob, stream)
        xd = torch.from_numpy(x).to(cuda_device)
        yd = torch.full_like(xd, float("nan"))
        rc = cuda_lib.dmrgpp_kron_apply_noalloc(ctypes.byref(t.desc), ctypes.c_void_p(xd.data_ptr()),
                                                ctypes.c_void_p(yd.data_ptr()))
        assert rc == _capi.OK, cuda_lib.dmrgpp_kron_noalloc_last_error()
        torch.cuda.synchronize()
        y_noalloc = yd.cpu().numpy()
        assert np.isfinite(y_noalloc).all()
        assert _rel(y_noalloc, y_alloc) < RTOL


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
