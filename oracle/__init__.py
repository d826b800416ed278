"""ORACLE -- test infrastructure only.

CPU checkers for the Kronecker H*psi path:

* ``liboracle_kron.so`` (``kron_oracle.c``): a scalar C restatement of the
  reference plugin's two-pass product, its flop count and the sector gather
  index.
* ``_ref/libref_kron.so`` (``ref_harness.cpp``): the reference's own
  ``Dmrg::BatchedGemmCpu`` and ``PsimagLite::LanczosSolver`` compiled from
  the reference sources (built here only when the reference tree exists; the
  built file travels with the repository snapshot).
* ``_ref/libref_kronconn.so`` (``kronconn_harness.cpp``): the reference's
  default non-batched H*x, ``KronConnections::doTask`` over the output
  patches with the reference's ``den_kron_mult`` per block.
* ``lanczos_oracle``: a numpy restatement of PsimagLite's Lanczos.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_kron.so")
REF_SO = os.path.join(HERE, "_ref", "libref_kron.so")
REF_KC_SO = os.path.join(HERE, "_ref", "libref_kronconn.so")
# the reference source tree (read-only); only the build recipe reads it
REFERENCE_TREE = os.environ.get("DMRGPP_REFERENCE_TREE", "/root/reference")

_sz = ctypes.c_size_t
_szp = ctypes.POINTER(ctypes.c_size_t)
_dp = ctypes.POINTER(ctypes.c_double)
_vpp = ctypes.POINTER(ctypes.c_void_p)


def build(force: bool = False) -> None:
    """Compile the C restatement and, when the reference tree is present,
    the reference harness."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", HERE, "liboracle_kron.so"], check=True)
    if os.path.isdir(REFERENCE_TREE) and (force or not os.path.exists(REF_SO)
                                          or not os.path.exists(REF_KC_SO)):
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + REFERENCE_TREE], check=True)


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return ctypes.CDLL(path)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = _load(ORACLE_SO)
        args = [_sz, _sz, _szp, _szp, _vpp, _szp, _vpp, _szp]
        lib.oracle_kron_apply.argtypes = args + [_dp, _dp]
        lib.oracle_kron_apply.restype = ctypes.c_int
        lib.oracle_kron_flops.argtypes = args
        lib.oracle_kron_flops.restype = ctypes.c_double
        lib.oracle_gather_index.argtypes = [_sz, _szp, _szp, _szp, _szp, _sz, _szp, _sz,
                                            ctypes.POINTER(ctypes.c_longlong)]
        lib.oracle_gather_index.restype = _sz
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


MATVEC_CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p, _dp, _dp)


def ref_lib():
    global _ref
    if _ref is None:
        # the OpenBLAS shipped in the Python env finds its libgfortran only
        # when it is already loaded
        import glob
        import sys
        libdir = os.path.join(sys.prefix, "lib", "python%d.%d" % sys.version_info[:2],
                              "site-packages", "opencv_python_headless.libs")
        for pat in ("libquadmath*.so*", "libgfortran*.so*"):
            for f in glob.glob(os.path.join(libdir, pat)):
                ctypes.CDLL(f, mode=ctypes.RTLD_GLOBAL)
        lib = _load(REF_SO)
        lib.ref_kron_create.argtypes = [_sz, _sz, _szp, _szp, _vpp, _szp, _vpp, _szp]
        lib.ref_kron_create.restype = ctypes.c_void_p
        lib.ref_kron_apply.argtypes = [ctypes.c_void_p, _dp, _dp]
        lib.ref_kron_apply.restype = None
        lib.ref_kron_destroy.argtypes = [ctypes.c_void_p]
        lib.ref_kron_dim.argtypes = [ctypes.c_void_p]
        lib.ref_kron_dim.restype = _sz
        lib.ref_lanczos.argtypes = [_sz, ctypes.c_void_p, ctypes.c_void_p, _dp, _sz, _sz,
                                    ctypes.c_double, ctypes.c_int, _dp, _dp]
        lib.ref_lanczos.restype = _sz
        _ref = lib
    return _ref


class _Tables:
    """ctypes views of a KronProblem's plugin tables (keeps arrays alive)."""

    def __init__(self, prob):
        A, ldA, B, ldB = prob.tables()
        tot = len(A)
        self.keep = [a for a in A if a is not None] + [b for b in B if b is not None]
        self.A = (ctypes.c_void_p * tot)(*[None if a is None else a.ctypes.data for a in A])
        self.B = (ctypes.c_void_p * tot)(*[None if b is None else b.ctypes.data for b in B])
        self.ldA = np.ascontiguousarray(ldA, dtype=np.uint64)
        self.ldB = np.ascontiguousarray(ldB, dtype=np.uint64)
        self.l = np.ascontiguousarray(prob.lsz, dtype=np.uint64)
        self.r = np.ascontiguousarray(prob.rsz, dtype=np.uint64)
        self.K = prob.noperator
        self.np = prob.npatches

    def args(self):
        return (self.K, self.np, self.l.ctypes.data_as(_szp), self.r.ctypes.data_as(_szp),
                ctypes.cast(self.A, _vpp), self.ldA.ctypes.data_as(_szp),
                ctypes.cast(self.B, _vpp), self.ldB.ctypes.data_as(_szp))


def kron_apply(prob, x: np.ndarray) -> np.ndarray:
    """y = H*x by the C restatement."""
    t = _Tables(prob)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty(prob.dim)
    rc = oracle_lib().oracle_kron_apply(*t.args(), x.ctypes.data_as(_dp), y.ctypes.data_as(_dp))
    assert rc == 0
    return y


def kron_flops(prob) -> float:
    t = _Tables(prob)
    return float(oracle_lib().oracle_kron_flops(*t.args()))


def gather_index(npatches, left_part, right_part, patch_left, patch_right, nl, perm_inverse,
                 offset, dim) -> np.ndarray:
    u = lambda a: np.ascontiguousarray(a, dtype=np.uint64)
    lp, rp, pl, pr, pi = map(u, (left_part, right_part, patch_left, patch_right, perm_inverse))
    idx = np.empty(dim, dtype=np.int64)
    n = oracle_lib().oracle_gather_index(
        npatches, lp.ctypes.data_as(_szp), rp.ctypes.data_as(_szp), pl.ctypes.data_as(_szp),
        pr.ctypes.data_as(_szp), nl, pi.ctypes.data_as(_szp), offset,
        idx.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
    assert n == dim
    return idx


_ref_kc = None


def ref_kronconn_lib():
    global _ref_kc
    if _ref_kc is None:
        ref_lib()          # loads the BLAS's Fortran runtime first
        lib = _load(REF_KC_SO)
        lib.ref_kronconn_create.argtypes = [_sz, _sz, _szp, _szp, _vpp, _szp, _vpp, _szp]
        lib.ref_kronconn_create.restype = ctypes.c_void_p
        lib.ref_kronconn_apply.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        lib.ref_kronconn_apply.restype = None
        lib.ref_kronconn_destroy.argtypes = [ctypes.c_void_p]
        _ref_kc = lib
    return _ref_kc


class RefKronConn:
    """The reference's default non-batched H*x for one sector
    (KronConnections::doTask with den_kron_mult per block, oracle/_ref);
    fits sectors whose BatchedGemmCpu slabs would not."""

    def __init__(self, prob):
        t = _Tables(prob)
        self.dim = prob.dim
        self.lib = ref_kronconn_lib()
        self.h = self.lib.ref_kronconn_create(*t.args())   # copies the blocks

    def apply(self, x: np.ndarray, threads: int = 1, y: Optional[np.ndarray] = None) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if y is None:
            y = np.empty(self.dim)
        self.lib.ref_kronconn_apply(self.h, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp),
                                    int(threads))
        return y

    def close(self):
        if self.h:
            self.lib.ref_kronconn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefKron:
    """The reference's Dmrg::BatchedGemmCpu for one sector (oracle/_ref)."""

    def __init__(self, prob, quiet: bool = True):
        self.t = _Tables(prob)
        self.dim = prob.dim
        lib = ref_lib()
        with _quiet_stdout(quiet):
            self.h = lib.ref_kron_create(*self.t.args())
        self.lib = lib

    def apply(self, x: np.ndarray, y: Optional[np.ndarray] = None) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        if y is None:
            y = np.empty(self.dim)
        self.lib.ref_kron_apply(self.h, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp))
        return y

    def lanczos(self, init, steps=200, min_steps=4, tolerance=1e-12, reortho=True,
                quiet: bool = True):
        """Lowest eigenpair by PsimagLite::LanczosSolver with this matvec."""
        n = self.dim
        init = np.ascontiguousarray(init, dtype=np.float64)
        z = np.zeros(n)
        e = ctypes.c_double(0.0)
        cb = ctypes.cast(self.lib.ref_kron_matvec_cb, ctypes.c_void_p)
        with _quiet_stdout(quiet):
            it = self.lib.ref_lanczos(n, cb, self.h, init.ctypes.data_as(_dp), steps, min_steps,
                                      tolerance, int(reortho), ctypes.byref(e),
                                      z.ctypes.data_as(_dp))
        return e.value, z, int(it)

    def __del__(self):
        try:
            self.lib.ref_kron_destroy(self.h)
        except Exception:
            pass


class _quiet_stdout:
    """Silence C-level stdout (the reference prints progress lines)."""

    def __init__(self, on=True):
        self.on = on

    def __enter__(self):
        if not self.on:
            return
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.devnull, 1)

    def __exit__(self, *a):
        if not self.on:
            return
        libc = ctypes.CDLL(None)
        try:
            libc.fflush(None)
        except Exception:
            pass
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.devnull)
