"""The C++ drop-in header (include/BatchedGemm.h, the class the reference's
BatchedGemmPluginSc constructs, dmrg/GPUPlugin/BatchedGemm.h:11-56) computing
on the GPU.

A C++ program written here from the golden fixtures builds the two
instantiations of the plugin class exactly as the reference's caller does
(std::vector<T*> block tables indexed out + in*np + k*np*np, VectorSizeType
sizes and leading dimensions) and calls apply_Htarget with host vectors:
  * BatchedGemm<double> on the known-answer case of the plugin's unit test
    (dmrg/Engine/tests/test_BatchedGemm.cpp:171-259, 1e-12 as there);
  * BatchedGemm<std::complex<double>> on the complex known answer of
    dmrg/Engine/tests/test_KronConnections.cpp:132-178 (H*input = {7+14i,
    2+4i}).
Compiled twice: with PsimagLite's default SizeType (unsigned long) and with
USE_SHORT (uint32_t), so the caller's VectorSizeType& arguments bind either
way."""
import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")


def _lit(values):
    return ", ".join(repr(float(v)) for v in values)


def _program():
    g = json.load(open(os.path.join(GOLDEN, "batchedgemm_1patch.json")))
    A = np.asfortranarray(np.array(g["A"]))
    B = np.asfortranarray(np.array(g["B"]))
    c = json.load(open(os.path.join(GOLDEN, "kron_connections_complex.json")))
    np_c = 1 + max(max(b["out"], b["in"]) for b in c["blocks"])
    slots = ["nullptr"] * (np_c * np_c)
    decl = []
    for q, b in enumerate(c["blocks"]):
        decl.append(f"\tstd::complex<double> ca{q}({b['A'][0]!r}, {b['A'][1]!r}), "
                    f"cb{q}({b['B'][0]!r}, {b['B'][1]!r});")
        slots[b["out"] + b["in"] * np_c] = str(q)
    a_tab = ", ".join("nullptr" if s == "nullptr" else f"&ca{s}" for s in slots)
    b_tab = ", ".join("nullptr" if s == "nullptr" else f"&cb{s}" for s in slots)
    cin = ", ".join(f"std::complex<double>({v[0]!r}, {v[1]!r})" for v in c["input"])
    return f"""
#include "BatchedGemm.h"

#include <complex>
#include <cstdio>
#include <vector>

int main()
{{
	using BG = BatchedGemm<double>;
	std::vector<double> A = {{{_lit(A.flatten(order="F"))}}};
	std::vector<double> B = {{{_lit(B.flatten(order="F"))}}};
	BG::VectorSizeType  l {{{A.shape[0]}}}, r {{{B.shape[0]}}}, ldA {{{A.shape[0]}}}, ldB {{{B.shape[0]}}};
	std::vector<double*> Am {{A.data()}}, Bm {{B.data()}};
	BG                   bg(1, 1, l, r, Am, ldA, Bm, ldB);
	std::vector<double>  vin = {{{_lit(g["vin"])}}}, vout(vin.size(), -1.0);
	bg.apply_Htarget(vin.data(), vout.data());
	std::printf("real");
	for (double v : vout)
		std::printf(" %.17g", v);
	std::printf("\\n");

	using CG = BatchedGemm<std::complex<double>>;
{chr(10).join(decl)}
	std::vector<std::complex<double>*> Ac {{{a_tab}}}, Bc {{{b_tab}}};
	CG::VectorSizeType sizes({np_c}, 1), ld({np_c * np_c}, 1);  // one ld per table entry
	CG cg(1, {np_c}, sizes, sizes, Ac, ld, Bc, ld);
	std::vector<std::complex<double>> cin = {{{cin}}}, cout(cin.size());
	cg.apply_Htarget(cin.data(), cout.data());
	std::printf("complex");
	for (auto v : cout)
		std::printf(" %.17g %.17g", v.real(), v.imag());
	std::printf("\\n");
	return 0;
}}
"""


@pytest.mark.parametrize("short_size", [False, True])
def test_cpp_dropin_known_answers(cuda_lib, cuda_device, tmp_path, short_size):
    from dmrgpp_b200 import _capi
    src = tmp_path / "dropin.cpp"
    exe = tmp_path / "dropin"
    src.write_text(_program())
    libdir = os.path.dirname(_capi.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-I" + os.path.join(ROOT, "include"), str(src), "-L" + libdir,
           "-ldmrgpp_kron", "-Wl,-rpath," + libdir, "-o", str(exe)]
    if short_size:
        cmd.insert(2, "-DUSE_SHORT")
    subprocess.run(cmd, check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = {ln.split()[0]: [float(v) for v in ln.split()[1:]] for ln in out.stdout.splitlines()}
    g = json.load(open(os.path.join(GOLDEN, "batchedgemm_1patch.json")))
    np.testing.assert_allclose(lines["real"], g["expected"], rtol=1e-12, atol=0)
    c = json.load(open(os.path.join(GOLDEN, "kron_connections_complex.json")))
    got = np.array(lines["complex"]).reshape(-1, 2)
    np.testing.assert_allclose(got, np.array(c["expected_H_input"]), rtol=0, atol=1e-12)
