"""Host-side mirror of the DMRG++ GPU plugin interface.

``BatchedGemm`` has the constructor arguments and the ``apply_Htarget``
method of ``template<class T> class BatchedGemm`` in
``dmrg/GPUPlugin/BatchedGemm.h:11-56`` (instantiated for double,
``BatchedGemm.cpp:117``).  Every call goes through the C ABI of
``include/dmrgpp_kron.h`` into the sm_100a kernels; a CUDA-side failure
raises ``DmrgppError`` instead of the reference's assert/printf.
"""
from __future__ import annotations

import ctypes
import time
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import FP64, SPLIT_BF16, TF32X3, DmrgppError  # noqa: F401


def _size_array(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.uint64))


class _DescTables:
    """Keeps the ctypes descriptor and everything it points to alive."""

    def __init__(self, noperator, npatches, left_patch_size, right_patch_size, Amatrix,
                 ld_Amatrix, Bmatrix, ld_Bmatrix, precision, stream, device, complex_blocks=False):
        tot = npatches * npatches * noperator
        if len(Amatrix) != tot or len(Bmatrix) != tot:
            raise ValueError(f"tables must have npatches^2*noperator = {tot} entries")
        self.l = _size_array(left_patch_size)
        self.r = _size_array(right_patch_size)
        if len(self.l) != npatches or len(self.r) != npatches:
            raise ValueError("patch-size arrays must have npatches entries")
        self.keep = []

        def ptr(m):
            if m is None:
                return None
            if isinstance(m, int):
                return m
            a = np.asarray(m)
            if a.dtype != (np.complex128 if complex_blocks else np.float64):
                raise TypeError("blocks must be complex128" if complex_blocks else "blocks must be float64")
            if a.ndim == 2 and not a.flags.f_contiguous:
                a = np.asfortranarray(a)
            self.keep.append(a)
            return a.ctypes.data

        self.A = (ctypes.c_void_p * tot)(*[ptr(m) for m in Amatrix])
        self.B = (ctypes.c_void_p * tot)(*[ptr(m) for m in Bmatrix])
        self.ldA = _size_array(ld_Amatrix)
        self.ldB = _size_array(ld_Bmatrix)
        if len(self.ldA) != tot or len(self.ldB) != tot:
            raise ValueError("leading-dimension arrays must match the tables")
        szp = ctypes.POINTER(ctypes.c_size_t)
        self.desc = _capi.KronDesc(
            noperator, npatches, self.l.ctypes.data_as(szp), self.r.ctypes.data_as(szp),
            ctypes.cast(self.A, ctypes.POINTER(ctypes.c_void_p)), self.ldA.ctypes.data_as(szp),
            ctypes.cast(self.B, ctypes.POINTER(ctypes.c_void_p)), self.ldB.ctypes.data_as(szp),
            int(precision), stream, int(device))


def cached_memory(device: int = -1):
    """(reserved, in-use) bytes of the library's device memory pool."""
    r, u = ctypes.c_size_t(), ctypes.c_size_t()
    _capi.check(_capi.lib().dmrgpp_cached_memory(device, ctypes.byref(r), ctypes.byref(u)))
    return int(r.value), int(u.value)


def release_cached_memory(device: int = -1) -> None:
    """Returns the pool's unused device memory (kept for the next handle
    otherwise) to the device."""
    _capi.check(_capi.lib().dmrgpp_release_cached_memory(device))


class BatchedGemm:
    """y = H x for one superblock sector on the GPU.

    Arguments follow ``BatchedGemm(noperator, npatches, left_patch_size,
    right_patch_size, Amatrix, ld_Amatrix, Bmatrix, ld_Bmatrix)``: tables of
    ``npatches*npatches*noperator`` column-major blocks indexed
    ``outPatch + inPatch*npatches + k*npatches^2`` (None = absent).
    """

    def __init__(self, noperator: int, npatches: int, left_patch_size: Sequence[int],
                 right_patch_size: Sequence[int], Amatrix, ld_Amatrix, Bmatrix, ld_Bmatrix,
                 precision: int = FP64, stream: Optional[int] = None, device: int = -1):
        L = _capi.lib()
        # complex blocks (std::complex<double>): dmrgpp_kron_create_complex
        self.is_complex = any(m is not None and not isinstance(m, int) and np.iscomplexobj(m)
                              for m in list(Amatrix) + list(Bmatrix))
        if self.is_complex:
            cast = lambda tab: [None if m is None else np.asarray(m, dtype=np.complex128) for m in tab]
            Amatrix, Bmatrix = cast(Amatrix), cast(Bmatrix)
        t = _DescTables(noperator, npatches, left_patch_size, right_patch_size, Amatrix,
                        ld_Amatrix, Bmatrix, ld_Bmatrix, precision, stream, device,
                        complex_blocks=self.is_complex)
        h = ctypes.c_void_p()
        t0 = time.perf_counter()
        create = L.dmrgpp_kron_create_complex if self.is_complex else L.dmrgpp_kron_create
        rc = create(ctypes.byref(t.desc), ctypes.byref(h))
        self.create_seconds = time.perf_counter() - t0   # the C create alone (synchronous)
        _capi.check(rc)
        self._h = h
        self._lib = L
        d = ctypes.c_size_t()
        _capi.check(L.dmrgpp_kron_dim(h, ctypes.byref(d)), h)
        self.dim = int(d.value)
        f = ctypes.c_double()
        _capi.check(L.dmrgpp_kron_flops(h, ctypes.byref(f)), h)
        self.f_alg = float(f.value)

    @classmethod
    def from_problem(cls, prob, **kw) -> "BatchedGemm":
        A, ldA, B, ldB = prob.tables()
        return cls(prob.noperator, prob.npatches, prob.lsz, prob.rsz, A, ldA, B, ldB, **kw)

    @classmethod
    def from_crs(cls, left_offset, left_size, right_offset, right_size, A, B, value=None,
                 fermion=None, left_parity=None, precision: int = FP64,
                 stream: Optional[int] = None, device: int = -1) -> "BatchedGemm":
        """A sector built on the device from its CRS operators
        (dmrgpp_kron_create_crs): A and B are lists (one per term) of
        scipy.sparse CSR matrices or (indptr, indices, data) triples over the
        left and right bases; value (per-term factor on A), fermion (per-term
        flag) and left_parity (per left state) as in calculateAhat."""
        L = _capi.lib()
        keep = []

        def crs(m):
            if hasattr(m, "indptr"):
                ip, ix, dv, rows = m.indptr, m.indices, m.data, m.shape[0]
            else:
                ip, ix, dv = m
                rows = len(ip) - 1
            ip = np.ascontiguousarray(ip, dtype=np.int32)
            ix = np.ascontiguousarray(ix, dtype=np.int32)
            dv = np.ascontiguousarray(dv, dtype=np.float64)
            keep.extend([ip, ix, dv])
            return _capi.Crs(rows, ip.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             ix.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             dv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

        K = len(A)
        Ac = (_capi.Crs * K)(*[crs(m) for m in A])
        Bc = (_capi.Crs * K)(*[crs(m) for m in B])
        arrs = [_size_array(x) for x in (left_offset, left_size, right_offset, right_size)]
        d = _capi.KronCrsDesc()
        szp = ctypes.POINTER(ctypes.c_size_t)
        d.noperator, d.npatches = K, len(arrs[1])
        d.left_offset, d.left_patch_size, d.right_offset, d.right_patch_size = \
            [a.ctypes.data_as(szp) for a in arrs]
        d.A, d.B = Ac, Bc
        vals = fer = par = None
        if value is not None:
            vals = np.ascontiguousarray(value, dtype=np.float64)
            d.value = vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if fermion is not None:
            fer = np.ascontiguousarray(fermion, dtype=np.int32)
            d.fermion = fer.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        if left_parity is not None:
            par = np.ascontiguousarray(left_parity, dtype=np.uint8)
            d.left_parity = par.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))
        d.precision, d.stream, d.device = precision, stream, device
        h = ctypes.c_void_p()
        t0 = time.perf_counter()
        rc = L.dmrgpp_kron_create_crs(ctypes.byref(d), ctypes.byref(h))
        create_seconds = time.perf_counter() - t0
        _capi.check(rc)
        self = cls.__new__(cls)
        self._h, self._lib = h, L
        self.is_complex = False
        self.create_seconds = create_seconds
        n = ctypes.c_size_t()
        _capi.check(L.dmrgpp_kron_dim(h, ctypes.byref(n)), h)
        self.dim = int(n.value)
        f = ctypes.c_double()
        _capi.check(L.dmrgpp_kron_flops(h, ctypes.byref(f)), h)
        self.f_alg = float(f.value)
        return self

    @classmethod
    def from_problems(cls, probs, precision: int = FP64, stream: Optional[int] = None,
                      device: int = -1) -> "BatchedGemm":
        """Many independent sectors in one handle (dmrgpp_kron_create_group):
        H is block-diagonal over the sectors, one apply runs them all in one
        launch on the concatenated vector; sector_offsets() gives the layout."""
        L = _capi.lib()
        tabs = []
        for prob in probs:
            A, ldA, B, ldB = prob.tables()
            tabs.append(_DescTables(prob.noperator, prob.npatches, prob.lsz, prob.rsz, A, ldA,
                                    B, ldB, precision, stream, device))
        descs = (_capi.KronDesc * len(tabs))(*[t.desc for t in tabs])
        h = ctypes.c_void_p()
        _capi.check(L.dmrgpp_kron_create_group(descs, len(tabs), ctypes.byref(h)))
        self = cls.__new__(cls)
        self._h, self._lib = h, L
        d = ctypes.c_size_t()
        _capi.check(L.dmrgpp_kron_dim(h, ctypes.byref(d)), h)
        self.dim = int(d.value)
        f = ctypes.c_double()
        _capi.check(L.dmrgpp_kron_flops(h, ctypes.byref(f)), h)
        self.f_alg = float(f.value)
        return self

    SETUP_PHASES = ("plan", "alloc", "upload", "upload_fill", "diagonal", "mixed", "total")

    def setup_profile(self) -> dict:
        """Seconds spent in each phase of this handle's create
        (dmrgpp_kron_setup_profile)."""
        n = len(self.SETUP_PHASES)
        t = (ctypes.c_double * n)()
        _capi.check(self._lib.dmrgpp_kron_setup_profile(self._h, t, n), self._h)
        return {k: float(v) for k, v in zip(self.SETUP_PHASES, t)}

    def sector_offsets(self) -> np.ndarray:
        """Start offsets of the handle's sectors in x (nsectors + 1 entries)."""
        n = ctypes.c_size_t()
        _capi.check(self._lib.dmrgpp_kron_group_sectors(self._h, ctypes.byref(n), None), self._h)
        offs = np.zeros(n.value + 1, dtype=np.int64)
        _capi.check(self._lib.dmrgpp_kron_group_sectors(
            self._h, ctypes.byref(n), offs.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))),
            self._h)
        return offs

    def lanczos_lowest_group(self, init, steps: int = 200, min_steps: int = 4,
                             tolerance: float = 1e-12, eigs_for_stop: int = 1,
                             reortho: bool = True, check_every: int = 8, mask=None):
        """Lowest eigenpair of every sector of a group handle, all sectors in
        lockstep (dmrgpp_lanczos_lowest_group).  Returns (energies array,
        concatenated Ritz vectors, steps array); numpy or torch CUDA like
        lanczos_lowest.  mask (one bool per sector) restricts the solve to
        the sectors set in it (dmrgpp_lanczos_lowest_group_masked): the
        others get NaN energies and zero vectors at no cost."""
        L = self._lib
        p = _capi.LanczosParams()
        L.dmrgpp_lanczos_params_init(ctypes.byref(p))
        p.steps, p.min_steps, p.tolerance = steps, min_steps, tolerance
        p.eigs_for_stop, p.reortho, p.check_every = eigs_for_stop, int(reortho), check_every
        nsec = len(self.sector_offsets()) - 1
        e = np.zeros(nsec)
        n = np.zeros(nsec, dtype=np.uint64)
        dp = ctypes.POINTER(ctypes.c_double)
        szp = ctypes.POINTER(ctypes.c_size_t)
        m = None
        if mask is not None:
            m = np.ascontiguousarray(np.asarray(mask, dtype=bool).astype(np.int32))
            if m.size != nsec:
                raise ValueError(f"mask needs {nsec} entries")
        mp = m.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if m is not None else None
        if hasattr(init, "data_ptr"):
            import torch
            z = torch.empty_like(init)
            self._pointers(init, z)
            rc = L.dmrgpp_lanczos_lowest_group_masked(self._h, ctypes.byref(p), init.data_ptr(), 1,
                                                      mp, e.ctypes.data_as(dp), z.data_ptr(),
                                                      n.ctypes.data_as(szp))
        else:
            init = np.ascontiguousarray(init, dtype=np.float64)
            z = np.empty(self.dim)
            self._pointers(init, z)
            rc = L.dmrgpp_lanczos_lowest_group_masked(self._h, ctypes.byref(p), init.ctypes.data, 0,
                                                      mp, e.ctypes.data_as(dp), z.ctypes.data,
                                                      n.ctypes.data_as(szp))
        _capi.check(rc, self._h)
        return e, z, n.astype(np.int64)

    @property
    def handle(self):
        return self._h

    def apply_Htarget(self, vin, vout) -> None:
        """vout = H vin in patch order.  numpy arrays are host buffers (copied
        in and out); torch CUDA tensors are used in place on the device."""
        on_dev, px, py = self._pointers(vin, vout)
        _capi.check(self._lib.dmrgpp_kron_apply(self._h, px, py, on_dev), self._h)

    def __call__(self, x):
        if hasattr(x, "is_cuda") and x.is_cuda:
            import torch
            y = torch.empty_like(x)
        else:
            y = np.empty(self.dim, dtype=np.complex128 if getattr(self, "is_complex", False)
                         else np.float64)
        self.apply_Htarget(x, y)
        return y

    def _pointers(self, vin, vout):
        cplx = getattr(self, "is_complex", False)
        if hasattr(vin, "data_ptr"):
            want = "torch.complex128" if cplx else "torch.float64"
            for v in (vin, vout):
                if not (v.is_cuda and v.is_contiguous() and str(v.dtype) == want
                        and v.numel() == self.dim):
                    raise ValueError(f"device vectors must be contiguous {want[6:]} CUDA tensors "
                                     f"of length {self.dim}")
            return 1, vin.data_ptr(), vout.data_ptr()
        want = np.complex128 if cplx else np.float64
        for v in (vin, vout):
            if not (isinstance(v, np.ndarray) and v.dtype == want and v.flags.c_contiguous
                    and v.size == self.dim):
                raise ValueError(f"host vectors must be contiguous {np.dtype(want).name} of "
                                 f"length {self.dim}")
        return 0, vin.ctypes.data, vout.ctypes.data

    def lanczos_lowest(self, init, steps: int = 200, min_steps: int = 4,
                       tolerance: float = 1e-12, eigs_for_stop: int = 1, reortho: bool = True,
                       check_every: int = 8, use_graph: bool = True,
                       residual_gap_ratio: float = 0.0):
        """Lowest eigenpair by the device Lanczos (the reference's
        LanczosSolver::computeAllStatesBelow for one state).  Returns
        (energy, ritz_vector, steps).  numpy init -> numpy vector; a torch
        CUDA tensor -> a torch CUDA tensor."""
        L = self._lib
        p = _capi.LanczosParams()
        L.dmrgpp_lanczos_params_init(ctypes.byref(p))
        p.steps, p.min_steps, p.tolerance = steps, min_steps, tolerance
        p.eigs_for_stop, p.reortho, p.check_every = eigs_for_stop, int(reortho), check_every
        p.use_graph = int(use_graph)
        p.residual_gap_ratio = residual_gap_ratio
        e = ctypes.c_double()
        n = ctypes.c_size_t()
        if hasattr(init, "data_ptr"):
            import torch
            z = torch.empty_like(init)
            self._pointers(init, z)
            rc = L.dmrgpp_lanczos_lowest(self._h, ctypes.byref(p), init.data_ptr(), 1,
                                         ctypes.byref(e), z.data_ptr(), ctypes.byref(n))
        else:
            init = np.ascontiguousarray(init, dtype=np.float64)
            z = np.empty(self.dim)
            self._pointers(init, z)
            rc = L.dmrgpp_lanczos_lowest(self._h, ctypes.byref(p), init.ctypes.data, 0,
                                         ctypes.byref(e), z.ctypes.data, ctypes.byref(n))
        _capi.check(rc, self._h)
        return e.value, z, int(n.value)

    def davidson_lowest(self, init, preconditioner: int = 1, mlp=None, tolerance: float = 1e-8,
                        max_iterations: int = 500, max_subspace: int = 32,
                        mixed_tolerance: float = 1e-4, denominator_floor: float = 1e-3,
                        raise_on_no_convergence: bool = True):
        """Lowest eigenpair by the device Davidson.  preconditioner: 0 none,
        1 Jacobi, 2 learned (mlp = dmrgpp_b200.mlp.MLPPreconditioner).
        Returns (energy, ritz_vector, stats dict)."""
        L = self._lib
        p = _capi.DavidsonParams()
        L.dmrgpp_davidson_params_init(ctypes.byref(p))
        p.max_iterations, p.max_subspace, p.tolerance = max_iterations, max_subspace, tolerance
        p.preconditioner = preconditioner
        p.mlp = mlp.handle if mlp is not None else None
        p.mixed_tolerance, p.denominator_floor = mixed_tolerance, denominator_floor
        st = _capi.DavidsonStats()
        e = ctypes.c_double()
        if hasattr(init, "data_ptr"):
            import torch
            z = torch.empty_like(init)
            self._pointers(init, z)
            rc = L.dmrgpp_davidson_lowest(self._h, ctypes.byref(p), init.data_ptr(), 1,
                                          ctypes.byref(e), z.data_ptr(), ctypes.byref(st))
        else:
            init = np.ascontiguousarray(init, dtype=np.float64)
            z = np.empty(self.dim)
            self._pointers(init, z)
            rc = L.dmrgpp_davidson_lowest(self._h, ctypes.byref(p), init.ctypes.data, 0,
                                          ctypes.byref(e), z.ctypes.data, ctypes.byref(st))
        if rc != _capi.NOT_CONVERGED or raise_on_no_convergence:
            _capi.check(rc, self._h)
        stats = {f: getattr(st, f) for f, _ in _capi.DavidsonStats._fields_}
        return e.value, z, stats

    def davidson_lowest_group(self, init, preconditioner: int = 1, mlp=None,
                              tolerance: float = 1e-8, max_iterations: int = 500,
                              max_subspace: int = 32, denominator_floor: float = 1e-3,
                              raise_on_no_convergence: bool = True):
        """Lowest eigenpair of every sector of a group handle by the lockstep
        group Davidson (dmrgpp_davidson_lowest_group), in the handle's
        precision.  Returns (energies array, concatenated Ritz vectors,
        converged array, stats dict); numpy or torch CUDA like
        davidson_lowest."""
        L = self._lib
        p = _capi.DavidsonParams()
        L.dmrgpp_davidson_params_init(ctypes.byref(p))
        p.max_iterations, p.max_subspace, p.tolerance = max_iterations, max_subspace, tolerance
        p.preconditioner = preconditioner
        p.mlp = mlp.handle if mlp is not None else None
        p.denominator_floor = denominator_floor
        nsec = len(self.sector_offsets()) - 1
        e = np.zeros(nsec)
        conv = np.zeros(nsec, dtype=np.int32)
        st = _capi.DavidsonStats()
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        if hasattr(init, "data_ptr"):
            import torch
            z = torch.empty_like(init)
            self._pointers(init, z)
            rc = L.dmrgpp_davidson_lowest_group(self._h, ctypes.byref(p), init.data_ptr(), 1,
                                                e.ctypes.data_as(dp), z.data_ptr(),
                                                conv.ctypes.data_as(ip), ctypes.byref(st))
        else:
            init = np.ascontiguousarray(init, dtype=np.float64)
            z = np.empty(self.dim)
            self._pointers(init, z)
            rc = L.dmrgpp_davidson_lowest_group(self._h, ctypes.byref(p), init.ctypes.data, 0,
                                                e.ctypes.data_as(dp), z.ctypes.data,
                                                conv.ctypes.data_as(ip), ctypes.byref(st))
        if rc != _capi.NOT_CONVERGED or raise_on_no_convergence:
            _capi.check(rc, self._h)
        stats = {f: getattr(st, f) for f, _ in _capi.DavidsonStats._fields_}
        return e, z, conv.astype(bool), stats

    def refine_lowest(self, psi, max_outer: int = 6, tolerance: float = 1e-9,
                      inner_iterations: int = 200, inner_tolerance: float = 1e-4,
                      raise_on_no_convergence: bool = True):
        """FP64 residual refinement of psi (torch CUDA tensor, updated in place);
        the correction solves use the handle's current precision.  Returns
        (energy, stats dict)."""
        st = _capi.RefineStats()
        e = ctypes.c_double()
        self._pointers(psi, psi)
        rc = self._lib.dmrgpp_refine_lowest(self._h, psi.data_ptr(), max_outer, tolerance,
                                            inner_iterations, inner_tolerance, ctypes.byref(e),
                                            ctypes.byref(st))
        if rc != _capi.NOT_CONVERGED or raise_on_no_convergence:
            _capi.check(rc, self._h)
        return e.value, {f: getattr(st, f) for f, _ in _capi.RefineStats._fields_}

    def solve_lowest(self, init, tolerance: float = 1e-10, method: str = "auto",
                     mixed_steps: int = 150, mixed_tolerance: float = 1e-7,
                     fp64_steps: int = 400, tf32x3_gain: float = 1.5,
                     correction: str = "jacobi"):
        """Lowest eigenpair of a real sector (init: torch CUDA tensor) by
          "fp64"  -- FP64 Lanczos, full reorthogonalisation, eigenvalue-change
                     tolerance `tolerance` (the reference's method);
          "mixed" -- Lanczos in the handle's TF32x3 form without
                     reorthogonalisation (it only supplies a start vector; up
                     to mixed_steps steps or a mixed_tolerance Ritz-value
                     change), then the FP64 refinement to |r| <= tolerance
                     max(1, |E|); if the refinement reports no convergence (a
                     start above the first excitation of a nearly gapless
                     sector), FP64 Lanczos finishes from the refined state;
          "auto"  -- "mixed" on a TF32x3 handle unless the last autotune timed
                     its TF32x3 H*x less than tf32x3_gain times faster than the
                     tuned FP64 one (sectors of small patches), else "fp64".
        correction: the refinement's correction solves, "jacobi"
        (preconditioned by the diagonal of H, see set_correction_preconditioner;
        on Hubbard-chain sectors 35% fewer correction matvecs) or "none"
        (plain conjugate gradients).
        Returns (energy, vector, stats dict; stats["method"] is the one used).
        The handle's precision and correction preconditioner are left as they
        were."""
        if method not in ("auto", "fp64", "mixed"):
            raise ValueError(f"unknown method {method!r}")
        if correction not in ("none", "jacobi"):
            raise ValueError(f"unknown correction {correction!r}")
        t64, t32 = self.tuned_times()
        user = self.get_precision()
        if method == "auto":
            has_mixed = user == TF32X3 or t32 > 0
            slow = t32 > 0 and t64 > 0 and t64 < tf32x3_gain * t32
            method = "mixed" if has_mixed and not slow else "fp64"
        clock = time.perf_counter   # each phase ends in a host read of its result
        try:
            if method == "fp64":
                self.set_precision(FP64)
                t0 = clock()
                e, z, n = self.lanczos_lowest(init, steps=fp64_steps, tolerance=tolerance)
                return e, z, dict(method="fp64", fp64_lanczos_steps=n, converged=1,
                                  fp64_lanczos_seconds=clock() - t0)
            self.set_precision(TF32X3)
            t0 = clock()
            e1, z, n1 = self.lanczos_lowest(init, steps=mixed_steps, tolerance=mixed_tolerance,
                                            reortho=False)
            t1 = clock()
            if correction == "jacobi":
                self.set_correction_preconditioner(_capi.PRECOND_JACOBI)
            try:
                e, st = self.refine_lowest(z, max_outer=12, tolerance=tolerance,
                                           inner_iterations=80, inner_tolerance=1e-2,
                                           raise_on_no_convergence=False)
            finally:
                if correction == "jacobi":
                    self.set_correction_preconditioner(_capi.PRECOND_NONE)
            st = dict(st, method="mixed", mixed_lanczos_steps=n1, fallback=0,
                      mixed_lanczos_seconds=t1 - t0, refine_seconds=clock() - t1)
            if not st["converged"]:
                # from the refined state plus a small seeded perturbation (see
                # solve_lowest_group)
                import torch
                g = torch.from_numpy(np.random.default_rng(7).standard_normal(self.dim)).to(z.device)
                z = z + 1e-3 * torch.linalg.vector_norm(z) * g / torch.linalg.vector_norm(g)
                self.set_precision(FP64)
                t0 = clock()
                e, z, n2 = self.lanczos_lowest(z, steps=fp64_steps, tolerance=tolerance)
                st.update(fallback=1, converged=1, fp64_lanczos_steps=n2,
                          fp64_lanczos_seconds=clock() - t0)
            return e, z, st
        finally:
            self.set_precision(user)

    def solve_lowest_group(self, init, tolerance: float = 1e-10, mixed_tolerance: float = 1e-5,
                           mixed_steps: int = 200, correction: str = "jacobi",
                           fp64_steps: int = 200):
        """Lowest eigenpair of every sector of a group handle created with
        TF32x3 (init: torch CUDA tensor, the concatenated start vectors):
        the TF32x3 group Lanczos without reorthogonalisation (it only supplies
        start vectors; up to mixed_steps steps or a mixed_tolerance Ritz-value
        change), then the lockstep FP64 group refinement to
        |r| <= tolerance max(1, |E|) with the given correction solves ("jacobi"
        or "none"); a sector whose refinement did not converge (its start above
        the first excitation of a nearly gapless sector) is then finished by an
        FP64 group Lanczos started from the refined vectors, whose result is
        taken for those sectors only.  Returns (energies, vectors, stats dict:
        lanczos_steps, refine stats, fallbacks and the seconds of each phase).
        The handle's precision and correction preconditioner are left as they
        were."""
        import torch
        if correction not in ("none", "jacobi"):
            raise ValueError(f"unknown correction {correction!r}")
        user = self.get_precision()
        clock = time.perf_counter   # each phase ends in a host read of its result
        try:
            self.set_precision(TF32X3)
            t0 = clock()
            _, z, steps = self.lanczos_lowest_group(init, steps=mixed_steps,
                                                    tolerance=mixed_tolerance, reortho=False)
            t1 = clock()
            if correction == "jacobi":
                self.set_correction_preconditioner(_capi.PRECOND_JACOBI)
            try:
                e, conv, st = self.refine_lowest_group(z, max_outer=12, tolerance=tolerance,
                                                       inner_iterations=80, inner_tolerance=1e-2,
                                                       raise_on_no_convergence=False)
            finally:
                if correction == "jacobi":
                    self.set_correction_preconditioner(_capi.PRECOND_NONE)
            t2 = clock()
            st = dict(st, lanczos_steps=steps, fallbacks=int((~conv).sum()),
                      mixed_lanczos_seconds=t1 - t0, refine_seconds=t2 - t1,
                      fallback_seconds=0.0)
            if not conv.all():
                # only the unconverged sectors, each from its refined vector
                # plus a seeded perturbation of relative size 1e-3 (a start
                # that already is an eigenvector makes the first Lanczos step
                # break down; the reference's Lanczos, mirrored here, keeps
                # the pre-reorthogonalisation beta)
                offs = self.sector_offsets()
                g = torch.from_numpy(np.random.default_rng(7).standard_normal(self.dim)).to(z.device)
                start = z.clone()
                for q in np.flatnonzero(~conv):
                    gs = g[offs[q]:offs[q + 1]]
                    start[offs[q]:offs[q + 1]] += 1e-3 * gs / torch.linalg.vector_norm(gs)
                self.set_precision(FP64)
                e64, z64, _ = self.lanczos_lowest_group(start, steps=fp64_steps, tolerance=1e-12,
                                                        mask=~conv)
                for q in np.flatnonzero(~conv):
                    e[q] = e64[q]
                    z[offs[q]:offs[q + 1]] = z64[offs[q]:offs[q + 1]]
                if z.is_cuda:
                    torch.cuda.synchronize(z.device)
                st["fallback_seconds"] = clock() - t2
            st["converged"] = 1
            return e, z, st
        finally:
            self.set_precision(user)

    def refine_lowest_group(self, psi, max_outer: int = 6, tolerance: float = 1e-9,
                            inner_iterations: int = 200, inner_tolerance: float = 1e-4,
                            raise_on_no_convergence: bool = True):
        """FP64 refinement of every sector of a group handle at once
        (dmrgpp_refine_lowest_group); psi is the concatenated sector vectors
        (torch CUDA tensor, updated in place).  Returns (energies array,
        converged array, stats dict)."""
        nsec = len(self.sector_offsets()) - 1
        e = np.zeros(nsec)
        conv = np.zeros(nsec, dtype=np.int32)
        st = _capi.RefineStats()
        self._pointers(psi, psi)
        rc = self._lib.dmrgpp_refine_lowest_group(
            self._h, psi.data_ptr(), max_outer, tolerance, inner_iterations, inner_tolerance,
            e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            conv.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.byref(st))
        if rc != _capi.NOT_CONVERGED or raise_on_no_convergence:
            _capi.check(rc, self._h)
        return e, conv.astype(bool), {f: getattr(st, f) for f, _ in _capi.RefineStats._fields_}

    def diagonal(self):
        """Diagonal of H (torch CUDA tensor, patch order)."""
        import torch
        d = torch.empty(self.dim, dtype=torch.float64, device="cuda")
        _capi.check(self._lib.dmrgpp_kron_diagonal(self._h, d.data_ptr()), self._h)
        torch.cuda.synchronize()
        return d

    def correction_solve(self, u, theta: float, r, max_iterations: int = 500,
                         rel_tolerance: float = 1e-10):
        """Exact correction t (torch CUDA tensors) of (I-uu^T)(H-theta)(I-uu^T) t = -r."""
        import torch
        t = torch.empty_like(u)
        its = ctypes.c_int()
        res = ctypes.c_double()
        _capi.check(self._lib.dmrgpp_correction_solve(self._h, u.data_ptr(), theta, r.data_ptr(),
                                                      t.data_ptr(), max_iterations, rel_tolerance,
                                                      ctypes.byref(its), ctypes.byref(res)), self._h)
        return t, its.value, res.value

    def autotune(self, cache_path: Optional[str] = None, reps: int = 10):
        """Picks the fastest tile configuration / work split for this sector
        (cached by sector shape in cache_path).  Returns (cfg, microseconds)."""
        cfg = ctypes.c_int()
        us = ctypes.c_double()
        path = cache_path.encode() if cache_path else None
        _capi.check(self._lib.dmrgpp_kron_autotune(self._h, path, reps, ctypes.byref(cfg),
                                                   ctypes.byref(us)), self._h)
        return cfg.value, us.value

    def tuned_times(self):
        """(FP64 apply, TF32x3 apply) microseconds of the last autotune (-1
        when not measured)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        _capi.check(self._lib.dmrgpp_kron_tuned_times(self._h, ctypes.byref(a), ctypes.byref(b)),
                    self._h)
        return a.value, b.value

    def set_correction_preconditioner(self, preconditioner: int) -> None:
        """PRECOND_NONE (default) or PRECOND_JACOBI for this handle's correction
        solves (refine_lowest, correction_solve)."""
        _capi.check(self._lib.dmrgpp_set_correction_preconditioner(self._h, int(preconditioner)),
                    self._h)

    def get_precision(self) -> int:
        v = ctypes.c_int()
        _capi.check(self._lib.dmrgpp_kron_get_precision(self._h, ctypes.byref(v)), self._h)
        return v.value

    def set_precision(self, precision: int) -> None:
        """FP64 or the mixed mode the handle was created with."""
        _capi.check(self._lib.dmrgpp_kron_set_precision(self._h, precision), self._h)

    def set_config(self, cfg: int, items_per_cta: int = 2) -> None:
        _capi.check(self._lib.dmrgpp_kron_set_config(self._h, cfg, items_per_cta), self._h)

    def get_config(self):
        c, i = ctypes.c_int(), ctypes.c_int()
        _capi.check(self._lib.dmrgpp_kron_get_config(self._h, ctypes.byref(c), ctypes.byref(i)),
                    self._h)
        return c.value, i.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.dmrgpp_kron_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tridiag_eigen(diag, offdiag, vectors: bool = True):
    """Eigenvalues (ascending) and eigenvectors of a symmetric tridiagonal
    matrix by the library's host solver."""
    d = np.ascontiguousarray(diag, dtype=np.float64)
    e = np.ascontiguousarray(offdiag, dtype=np.float64)
    n = len(d)
    w = np.empty(n)
    Z = np.empty((n, n), order="F") if vectors else None
    dp = ctypes.POINTER(ctypes.c_double)
    rc = _capi.lib().dmrgpp_tridiag_eigen(n, d.ctypes.data_as(dp),
                                          e.ctypes.data_as(dp) if n > 1 else None,
                                          w.ctypes.data_as(dp),
                                          Z.ctypes.data_as(dp) if vectors else None)
    _capi.check(rc)
    return (w, Z) if vectors else w


def plan_info(prob, precision: int = FP64) -> dict:
    """Host-only planning statistics of a sector (no GPU needed)."""
    A, ldA, B, ldB = prob.tables()
    t = _DescTables(prob.noperator, prob.npatches, prob.lsz, prob.rsz, A, ldA, B, ldB,
                    precision, None, -1)
    info = _capi.PlanInfo()
    _capi.check(_capi.lib().dmrgpp_kron_plan_info_get(ctypes.byref(t.desc), ctypes.byref(info)))
    return {f: getattr(info, f) for f, _ in _capi.PlanInfo._fields_}


def sector_gather_index(patch_left, patch_right, left_partition, right_partition, perm_inverse,
                        offset: int, sector_size: int) -> np.ndarray:
    """The sector's copyIn / copyOut index (dmrgpp_kron_gather_index, host
    only): patch_left / patch_right are the patches' left and right groups
    (GenIjPatch), left_partition / right_partition the blocks' group offsets
    (Basis::partition, groups + 1 entries), perm_inverse the superblock's
    permutationInverse (nl x nr), offset and sector_size the target sector in
    super-basis order.  Returns int64 idx with yin = vin[idx] (dmrgpp_gather)
    and vout[idx] = xout (dmrgpp_scatter)."""
    pl, pr = _size_array(patch_left), _size_array(patch_right)
    lp, rp = _size_array(left_partition), _size_array(right_partition)
    perm = _size_array(perm_inverse)
    d = _capi.GatherIndexDesc()
    szp = ctypes.POINTER(ctypes.c_size_t)
    d.npatches = len(pl)
    d.patch_left, d.patch_right = pl.ctypes.data_as(szp), pr.ctypes.data_as(szp)
    d.left_groups, d.right_groups = len(lp) - 1, len(rp) - 1
    d.left_partition, d.right_partition = lp.ctypes.data_as(szp), rp.ctypes.data_as(szp)
    d.perm_inverse = perm.ctypes.data_as(szp)
    d.offset, d.sector_size = int(offset), int(sector_size)
    idx = np.empty(int(sector_size), dtype=np.int64)
    _capi.check(_capi.lib().dmrgpp_kron_gather_index(
        ctypes.byref(d), idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
    return idx


def sector_patches(left_qns, right_qns, target):
    """The sector's patches (dmrgpp_kron_patch_list, host only): left_qns and
    right_qns are the blocks' group quantum numbers (tuples of additive
    integers, one per group), target the sector's.  Returns (patch_left,
    patch_right) arrays, left group outer, right group inner."""
    q = len(target)
    lq = np.ascontiguousarray(np.asarray(left_qns, dtype=np.int64).reshape(-1, q))
    rq = np.ascontiguousarray(np.asarray(right_qns, dtype=np.int64).reshape(-1, q))
    t = np.ascontiguousarray(np.asarray(target, dtype=np.int64))
    cap = len(lq) * max(len(rq), 1)
    pl = np.empty(max(cap, 1), dtype=np.uint64)
    pr = np.empty(max(cap, 1), dtype=np.uint64)
    n = ctypes.c_size_t()
    i64 = ctypes.POINTER(ctypes.c_int64)
    szp = ctypes.POINTER(ctypes.c_size_t)
    _capi.check(_capi.lib().dmrgpp_kron_patch_list(
        len(lq), lq.ctypes.data_as(i64), len(rq), rq.ctypes.data_as(i64), q, t.ctypes.data_as(i64),
        cap, pl.ctypes.data_as(szp), pr.ctypes.data_as(szp), ctypes.byref(n)))
    return pl[:n.value].astype(np.int64), pr[:n.value].astype(np.int64)
