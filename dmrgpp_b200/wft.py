"""Patch-wise wave-function transformation on the GPU (dmrgpp_wft_* in
include/dmrgpp_kron.h): Y_q = WR_q X_p WL_q^T for every output patch q with
source patch p, patch blocks r x l column-major as in the Kronecker sector
layout.  The GEMM core of the reference's WftAccelPatches
(Wft/WftAccelPatches.h:43-66, BlockDiagWf.h:131-260)."""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _capi


class WaveFunctionTransform:
    """WaveFunctionTransform(l_in, r_in, l_out, r_out, src, WL, WR) with WL[q]
    (l_out[q] x l_in[src[q]]) and WR[q] (r_out[q] x r_in[src[q]]) numpy
    blocks (None where src[q] < 0); trans_WL / trans_WR: the blocks are given
    transposed.  Calling it on x (numpy or torch CUDA) returns y."""

    def __init__(self, l_in: Sequence[int], r_in: Sequence[int], l_out: Sequence[int],
                 r_out: Sequence[int], src: Sequence[int], WL, WR, trans_WL: bool = False,
                 trans_WR: bool = False, stream: Optional[int] = None, device: int = -1):
        L = _capi.lib()
        sz = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.uint64))
        self._keep = []
        self.l_in, self.r_in, self.l_out, self.r_out = sz(l_in), sz(r_in), sz(l_out), sz(r_out)
        self.src = np.ascontiguousarray(np.asarray(src, dtype=np.int64))
        nq = len(self.l_out)
        if len(self.r_out) != nq or len(self.src) != nq or len(WL) != nq or len(WR) != nq:
            raise ValueError("l_out, r_out, src, WL and WR need one entry per output patch")

        def table(blocks):
            ptrs, lds = (ctypes.c_void_p * nq)(), np.zeros(nq, dtype=np.uint64)
            for q, m in enumerate(blocks):
                if m is None:
                    continue
                a = np.asfortranarray(np.asarray(m, dtype=np.float64))
                self._keep.append(a)
                ptrs[q] = a.ctypes.data
                lds[q] = a.shape[0]
            return ptrs, lds
        self._WL, self._ldWL = table(WL)
        self._WR, self._ldWR = table(WR)
        szp = ctypes.POINTER(ctypes.c_size_t)
        d = _capi.WftDesc(len(self.l_in), self.l_in.ctypes.data_as(szp), self.r_in.ctypes.data_as(szp),
                          nq, self.l_out.ctypes.data_as(szp), self.r_out.ctypes.data_as(szp),
                          self.src.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                          ctypes.cast(self._WL, ctypes.POINTER(ctypes.c_void_p)),
                          self._ldWL.ctypes.data_as(szp),
                          ctypes.cast(self._WR, ctypes.POINTER(ctypes.c_void_p)),
                          self._ldWR.ctypes.data_as(szp), int(trans_WL), int(trans_WR), stream,
                          int(device))
        h = ctypes.c_void_p()
        rc = L.dmrgpp_wft_create(ctypes.byref(d), ctypes.byref(h))
        if rc != _capi.OK:
            raise _capi.DmrgppError(rc, L.dmrgpp_wft_last_error(None).decode())
        self._h, self._lib = h, L
        self._keep = []   # the blocks were copied at create
        di, do = ctypes.c_size_t(), ctypes.c_size_t()
        self._check(L.dmrgpp_wft_dims(h, ctypes.byref(di), ctypes.byref(do)))
        self.dim_in, self.dim_out = int(di.value), int(do.value)
        f = ctypes.c_double()
        self._check(L.dmrgpp_wft_flops(h, ctypes.byref(f)))
        self.flops = float(f.value)

    def _check(self, rc):
        if rc != _capi.OK:
            raise _capi.DmrgppError(rc, self._lib.dmrgpp_wft_last_error(self._h).decode())

    def __call__(self, x, y=None):
        if hasattr(x, "data_ptr"):
            import torch
            if x.numel() != self.dim_in:
                raise ValueError(f"x has {x.numel()} entries, the input layout {self.dim_in}")
            y = torch.empty(self.dim_out, dtype=torch.float64, device=x.device) if y is None else y
            self._check(self._lib.dmrgpp_wft_apply(self._h, x.data_ptr(), y.data_ptr(), 1))
            return y
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.dim_in:
            raise ValueError(f"x has {x.size} entries, the input layout {self.dim_in}")
        y = np.empty(self.dim_out) if y is None else y
        self._check(self._lib.dmrgpp_wft_apply(self._h, x.ctypes.data, y.ctypes.data, 0))
        return y

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dmrgpp_wft_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
