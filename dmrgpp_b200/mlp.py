"""Learned Davidson preconditioner: Python side of the network in
``csrc/mlp.cu`` (all arithmetic runs in that CUDA library).

* ``MLPPreconditioner`` owns one network (4 -> 256 -> 256 -> 1, tanh hidden
  layers; FP32 master weights, BF16 inference weights).
* ``correction_pairs`` produces training data from the solver itself: the
  Davidson solver (Jacobi preconditioner) first converges the sector to
  FP64 accuracy (lowest eigenvalue lambda0); then it is rerun and stopped
  after k iterations, the FP64 residual r of its Ritz pair (theta, u) is
  formed, and the exact correction is the solution of the projected
  correction equation (I-uu^T)(H-sigma)(I-uu^T) t = -r with the shift sigma
  just below lambda0 (conjugate gradients in FP64 through the library) --
  the preconditioned step an exact preconditioner H - sigma would give
  (inverse iteration).  With theta itself as the shift the operator is
  indefinite while theta is above the second eigenvalue, which holds for
  most early iterates.  Features come from (diag(H), r, theta); the target
  is the direction of t* (t* / rms(t*)): Davidson orthonormalises the
  correction, so only its direction matters.
* ``train`` fits the network with the library's forward/backward kernels
  and Adam.
"""
from __future__ import annotations

import ctypes
import math
from typing import Iterable, List, Optional, Tuple

import numpy as np

from . import _capi


class MLPPreconditioner:
    FEATURES = 4

    def __init__(self, seed: int = 0, params: Optional[np.ndarray] = None):
        self._lib = _capi.lib()
        h = ctypes.c_void_p()
        _capi.check(self._lib.dmrgpp_mlp_create(seed, ctypes.byref(h)))
        self._h = h
        self.n_params = int(self._lib.dmrgpp_mlp_num_params())
        if params is not None:
            self.set_params(params)

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        if rc != _capi.OK:
            msg = self._lib.dmrgpp_mlp_last_error(self._h)
            raise _capi.DmrgppError(rc, msg.decode() if msg else "")

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        self._check(self._lib.dmrgpp_mlp_get_params(
            self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        self._check(self._lib.dmrgpp_mlp_set_params(
            self._h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params))

    def get_grads(self) -> np.ndarray:
        g = np.empty(self.n_params, dtype=np.float32)
        self._check(self._lib.dmrgpp_mlp_get_grads(
            self._h, g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), self.n_params))
        return g

    def features(self, diag, r, theta: float, rnorm: float, stream=None):
        import torch
        x = torch.empty((r.numel(), self.FEATURES), dtype=torch.float32, device=r.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self._lib.dmrgpp_mlp_features(diag.data_ptr(), r.data_ptr(), theta, rnorm,
                                                  r.numel(), x.data_ptr(), s))
        return x

    def forward(self, x, stream=None):
        import torch
        out = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self._lib.dmrgpp_mlp_forward(self._h, x.data_ptr(), x.shape[0],
                                                 out.data_ptr(), s))
        return out

    def backward(self, x, y, weight=None, stream=None) -> float:
        import torch
        loss = ctypes.c_double()
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self._lib.dmrgpp_mlp_backward(
            self._h, x.data_ptr(), y.data_ptr(), weight.data_ptr() if weight is not None else None,
            ctypes.byref(loss), s))
        return loss.value

    def adam_step(self, lr: float, stream=None) -> None:
        import torch
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self._lib.dmrgpp_mlp_adam_step(self._h, lr, s))

    TENSOR_CORES, CUDA_CORES = 0, 1

    def set_inference(self, mode: int) -> None:
        """TENSOR_CORES (default): fused tcgen05 kernel, first hidden layer
        in BF16; CUDA_CORES: the FP32 GEMM kernels of training."""
        self._check(self._lib.dmrgpp_mlp_set_inference(self._h, int(mode)))

    def precondition(self, diag, r, theta: float, rnorm: float, stream=None):
        import torch
        t = torch.empty_like(r)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self._lib.dmrgpp_mlp_precondition(self._h, diag.data_ptr(), r.data_ptr(),
                                                      theta, rnorm, t.data_ptr(), r.numel(), s))
        return t

    def precondition_group(self, diag, r, sector_start, theta, rnorm, stream=None):
        """Learned correction of the concatenated residuals of several sectors
        (dmrgpp_mlp_precondition_group): sector_start (int64, nsectors + 1),
        theta and rnorm (float64, one per sector) are torch CUDA tensors."""
        import torch
        t = torch.empty_like(r)
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        self._check(self._lib.dmrgpp_mlp_precondition_group(
            self._h, diag.data_ptr(), r.data_ptr(), sector_start.data_ptr(), theta.data_ptr(),
            rnorm.data_ptr(), int(theta.numel()), t.data_ptr(), r.numel(), s))
        return t

    def save(self, path: str) -> None:
        np.savez_compressed(path, params=self.get_params())

    @classmethod
    def load(cls, path: str) -> "MLPPreconditioner":
        return cls(params=np.load(path)["params"])

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dmrgpp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def correction_pairs(bg, init, checkpoints: Iterable[int] = (1, 2, 3, 5, 8, 12, 18, 26),
                     cg_iterations: int = 600, shift: float = 1e-2) -> List[Tuple]:
    """Solver-generated (features, scaled exact correction) pairs of one
    sector (see the module docstring).  bg: an FP64 plugin.BatchedGemm;
    init: torch CUDA start vector."""
    import torch
    mlp_features = MLPPreconditioner.__new__(MLPPreconditioner)  # feature map only
    mlp_features._lib = _capi.lib()
    mlp_features._h = None
    diag = bg.diagonal()
    D = bg.dim
    lam0, _, st0 = bg.davidson_lowest(init, preconditioner=_capi.PRECOND_JACOBI, tolerance=1e-10,
                                      max_iterations=4000, raise_on_no_convergence=False)
    sigma = lam0 - shift * max(1.0, abs(lam0))
    pairs = []
    for k in checkpoints:
        e, u, st = bg.davidson_lowest(init, preconditioner=_capi.PRECOND_JACOBI, max_iterations=k,
                                      raise_on_no_convergence=False)
        hu = bg(u)
        r = hu - e * u
        r = r - u * torch.dot(u, r)  # remove the (round-off) component along u
        rn = float(torch.linalg.vector_norm(r))
        if rn < 1e-12 * max(1.0, abs(e)):
            break
        t, its, res = bg.correction_solve(u, sigma, r, max_iterations=cg_iterations,
                                          rel_tolerance=1e-8)
        x = mlp_features.features(diag, r, e, rn)
        t_rms = float(torch.linalg.vector_norm(t)) / math.sqrt(D)
        if t_rms == 0.0:
            continue
        y = (t / t_rms).float()
        jac = r / (e - diag)
        cos_jacobi = float(torch.dot(jac, t) / (torch.linalg.vector_norm(jac)
                                                 * torch.linalg.vector_norm(t)))
        cos_resid = float(torch.dot(r, t) / (rn * torch.linalg.vector_norm(t)))
        pairs.append((x, y, {"iteration": k, "theta": e, "rnorm": rn, "cg_iterations": its,
                             "cg_rel_residual": res, "cos_jacobi": cos_jacobi,
                             "cos_residual": cos_resid}))
    return pairs


def train(mlp: MLPPreconditioner, X, Y, steps: int = 600, batch: int = 8192, lr: float = 2e-3,
          seed: int = 0, log_every: int = 0) -> List[float]:
    """Adam on the weighted MSE with the library's kernels; X (rows x 4) and Y
    (rows) are torch CUDA tensors.  Returns the loss history."""
    import torch
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    rows = X.shape[0]
    losses = []
    for step in range(steps):
        idx = torch.randint(0, rows, (min(batch, rows),), generator=g, device=X.device)
        xb = X[idx].contiguous()
        yb = Y[idx].contiguous()
        mlp.forward(xb)
        loss = mlp.backward(xb, yb)
        rate = lr * 0.5 * (1 + math.cos(math.pi * step / steps))  # cosine decay
        mlp.adam_step(rate)
        losses.append(loss)
        if log_every and step % log_every == 0:
            print(f"step {step} loss {loss:.4e}", flush=True)
    return losses
