"""The C-ABI library without a GPU: it loads, exports every declared symbol,
plans sectors on the host exactly like the oracle, and rejects bad input
with status codes (all checks happen before any device work)."""
import ctypes
import os
import re

import numpy as np
import pytest

from dmrgpp_b200 import superblock as sb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(dmrgpp_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol(cuda_lib):
    names = declared_symbols()
    assert "dmrgpp_kron_create" in names and "dmrgpp_kron_apply" in names
    missing = [n for n in names if not hasattr(cuda_lib, n)]
    assert not missing, missing


def test_version(cuda_lib):
    from dmrgpp_b200 import _capi
    assert _capi.lib().dmrgpp_version().startswith(b"dmrgpp-b200")


@pytest.mark.parametrize("seed", range(5))
def test_host_plan_matches_oracle(cuda_lib, oracle_built, seed):
    from dmrgpp_b200 import plugin
    prob = sb.random_problem(npatches=3 + seed, noperator=1 + seed % 4, max_size=40, seed=seed,
                             zero_block_rate=0.25)
    info = plugin.plan_info(prob)
    assert info["ntriples"] == len(prob.triples())
    assert info["dim"] == prob.dim
    assert info["f_alg"] == oracle_built.kron_flops(prob)


def test_plan_of_microbench_sector(cuda_lib):
    from dmrgpp_b200 import plugin
    info = plugin.plan_info(sb.c2_problem())
    assert info["ntriples"] == 103
    assert info["dim"] == 76406
    assert info["f_alg"] == 130138856.0


def _desc_for(prob):
    from dmrgpp_b200 import plugin
    A, ldA, B, ldB = prob.tables()
    return plugin._DescTables(prob.noperator, prob.npatches, prob.lsz, prob.rsz, A, ldA, B, ldB,
                              0, None, -1)


def test_invalid_inputs_are_rejected_with_status(cuda_lib):
    from dmrgpp_b200 import _capi, plugin
    prob = sb.random_problem(3, 2, seed=2)
    # empty patch (the reference asserts 1 <= size, setup_sparse_batch.cpp:70-71)
    bad = sb.random_problem(3, 2, seed=2)
    bad.lsz = bad.lsz.copy()
    bad.lsz[1] = 0
    t = _desc_for(bad)
    h = ctypes.c_void_p()
    rc = cuda_lib.dmrgpp_kron_create(ctypes.byref(t.desc), ctypes.byref(h))
    assert rc == _capi.INVALID_ARG and not h.value
    assert b"empty" in cuda_lib.dmrgpp_kron_last_error(None)
    # leading dimension smaller than the block
    t = _desc_for(prob)
    k = next(i for i in range(len(t.ldA)) if t.A[i])
    t.ldA[k] = 0
    rc = cuda_lib.dmrgpp_kron_create(ctypes.byref(t.desc), ctypes.byref(h))
    assert rc == _capi.INVALID_ARG
    # unknown precision mode
    t = _desc_for(prob)
    t.desc.precision = 7
    assert cuda_lib.dmrgpp_kron_create(ctypes.byref(t.desc), ctypes.byref(h)) == _capi.INVALID_ARG
    # null descriptor / output
    assert cuda_lib.dmrgpp_kron_create(None, ctypes.byref(h)) == _capi.INVALID_ARG
    assert cuda_lib.dmrgpp_kron_create(ctypes.byref(t.desc), None) == _capi.INVALID_ARG
    # destroy(NULL) is a no-op
    assert cuda_lib.dmrgpp_kron_destroy(None) == _capi.OK
    with pytest.raises(ValueError):
        plugin.BatchedGemm(1, 2, [1, 1], [1, 1], [None], [0], [None], [0])


def test_group_create_rejects_bad_sector_lists(cuda_lib):
    """dmrgpp_kron_create_group validates every sector before any device work."""
    from dmrgpp_b200 import _capi
    a, b = _desc_for(sb.random_problem(3, 2, seed=2)), _desc_for(sb.random_problem(2, 1, seed=3))
    h = ctypes.c_void_p()
    descs = (_capi.KronDesc * 2)(a.desc, b.desc)
    assert cuda_lib.dmrgpp_kron_create_group(descs, 0, ctypes.byref(h)) == _capi.INVALID_ARG
    assert cuda_lib.dmrgpp_kron_create_group(None, 2, ctypes.byref(h)) == _capi.INVALID_ARG
    assert cuda_lib.dmrgpp_kron_create_group(descs, 2, None) == _capi.INVALID_ARG
    descs[1].precision = 2                       # precisions differ
    assert cuda_lib.dmrgpp_kron_create_group(descs, 2, ctypes.byref(h)) == _capi.INVALID_ARG
    assert b"same precision" in cuda_lib.dmrgpp_kron_last_error(None)
    bad = sb.random_problem(2, 1, seed=3)
    bad.lsz = bad.lsz.copy()
    bad.lsz[0] = 0
    c = _desc_for(bad)
    descs = (_capi.KronDesc * 2)(a.desc, c.desc)
    assert cuda_lib.dmrgpp_kron_create_group(descs, 2, ctypes.byref(h)) == _capi.INVALID_ARG
    assert b"sector 1" in cuda_lib.dmrgpp_kron_last_error(None) and not h.value


def test_tridiagonal_helpers_of_the_group_solver(tmp_path):
    """Sturm bisection and inverse iteration (tridiag.cpp) against the QL
    solver on random, graded and nearly degenerate tridiagonals."""
    import subprocess
    exe = str(tmp_path / "tridiag_check")
    csrc = os.path.join(ROOT, "dmrgpp_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + csrc,
                    os.path.join(ROOT, "tests", "tridiag_check.cpp"),
                    os.path.join(csrc, "tridiag.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout


def test_missing_library_fails_loudly(monkeypatch):
    from dmrgpp_b200 import _capi
    monkeypatch.setattr(_capi, "LIB_PATH", "/nonexistent/libdmrgpp_kron.so")
    monkeypatch.setattr(_capi, "_lib", None)
    with pytest.raises(ImportError):
        _capi.lib()


CPP_SHIM_PROGRAM = r"""
#include "BatchedGemm.h"
#include <complex>
#include <cstdio>
#include <vector>
int main() {
  std::vector<std::size_t> l = {2, 0}, r = {3, 1}, ld(8, 0);   // patch 1 has an empty left group
  std::vector<double*> A(8, nullptr), B(8, nullptr);
  std::vector<std::complex<double>*> Ac(8, nullptr), Bc(8, nullptr);
  int caught = 0;
  try {
    BatchedGemm<double> bg(2, 2, l, r, A, ld, B, ld);
  } catch (const std::runtime_error& e) {
    std::printf("caught: %s\n", e.what());
    ++caught;
  }
  try {   // the reference's second instantiation
    BatchedGemm<std::complex<double>> bg(2, 2, l, r, Ac, ld, Bc, ld);
  } catch (const std::runtime_error& e) {
    std::printf("caught complex: %s\n", e.what());
    ++caught;
  }
  return caught == 2 ? 0 : 1;
}
"""


def test_cpp_dropin_header_compiles_links_and_throws(cuda_lib, tmp_path):
    """include/BatchedGemm.h (the C++ drop-in for dmrg/GPUPlugin/BatchedGemm.h)
    builds against the library and turns a status code into an exception."""
    import subprocess
    from dmrgpp_b200 import _capi
    src = tmp_path / "shim.cpp"
    exe = tmp_path / "shim"
    src.write_text(CPP_SHIM_PROGRAM)
    libdir = os.path.dirname(_capi.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src),
                    "-L" + libdir, "-ldmrgpp_kron", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caught: dmrgpp-b200:" in r.stdout and "empty" in r.stdout
    assert "caught complex: dmrgpp-b200:" in r.stdout


def test_wft_create_rejects_bad_descriptors(cuda_lib):
    """Descriptor checks of the wave-function transformation happen before
    any device work, with the reason in dmrgpp_wft_last_error(NULL)."""
    from dmrgpp_b200 import _capi
    from dmrgpp_b200 import wft as wft_mod
    ok = dict(l_in=[2, 3], r_in=[3, 1], l_out=[2], r_out=[2], src=[1],
              WL=[np.ones((2, 3))], WR=[np.ones((2, 1))])
    for change, words in [({"src": [2]}, "out of range"),
                          ({"WL": [None]}, "null transformation block"),
                          ({"l_in": [2, 0]}, "empty"),
                          ({"WR": [np.ones((1, 1))]}, "leading dimension")]:
        kw = dict(ok, **change)
        with pytest.raises(_capi.DmrgppError) as e:
            wft_mod.WaveFunctionTransform(**kw)
        assert e.value.status == _capi.INVALID_ARG and words in str(e.value), str(e.value)
    h = ctypes.c_void_p()
    assert cuda_lib.dmrgpp_wft_create(None, ctypes.byref(h)) == _capi.INVALID_ARG
    assert cuda_lib.dmrgpp_wft_destroy(None) == _capi.OK
