"""Build recipe of the in-tree CUDA library ``dmrgpp_b200/_lib/libdmrgpp_kron.so``.

Every source under ``dmrgpp_b200/csrc`` is compiled by nvcc for sm_100a only
and linked into one shared library that exports the C ABI of
``include/dmrgpp_kron.h``.  Run ``python -m dmrgpp_b200.build`` (add
``--verbose-ptxas`` to print register and shared-memory use).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(LIBDIR, "libdmrgpp_kron.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags(verbose_ptxas: bool):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
                "--expt-relaxed-constexpr"]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) \
        + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False, quiet: bool = True) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()
    srcs = sources()
    objs = [os.path.join(OBJDIR, os.path.basename(s) + ".o") for s in srcs]
    jobs = []
    for s, o in zip(srcs, objs):
        if force or verbose_ptxas or _stale(o, s):
            cmd = [cc] + _flags(verbose_ptxas) + ["-c", s, "-o", o]
            if s.endswith(".cpp"):
                cmd = [cc] + _flags(False) + ["-x", "cu", "-c", s, "-o", o]
            jobs.append(cmd)
    relink = bool(jobs) or force or not os.path.exists(LIB)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
            if verbose_ptxas or not quiet:
                sys.stderr.write(r.stderr)
    if relink:
        tmp = LIB + ".tmp"
        cmd = [cc] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart_static", "-lrt", "-ldl",
                                                             "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--verbose-ptxas" in sys.argv,
          quiet=False)
    print(LIB)
