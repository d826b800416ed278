"""Generates kron_connections_complex.json from the reference's complex
known-answer test, read as text:
dmrg/Engine/tests/test_KronConnections.cpp:132-178 (two 1x1 patches, one
connection; setBlock(out, in, left, right) puts the scalar `left` in the
system (A) table and `right` in the environment (B) table; the test checks
H*input = {7+14i, 2+4i} and x_out + H*input with x_out = {3+i, -1+2i} equal to
{10+15i, 1+6i}).  Run here: python tests/golden/make_complex_golden.py
"""
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(os.environ.get("DMRGPP_REFERENCE_TREE", "/root/reference"),
                   "dmrg", "Engine", "tests", "test_KronConnections.cpp")
CPLX = r"ComplexType\(\s*([-0-9.]+)\s*,\s*([-0-9.]+)\s*\)"


def cplx(m):
    return [float(m[0]), float(m[1])]


def main():
    text = open(SRC).read()
    body = text[text.index('TEST_CASE("KronConnections applies a complex'):]
    blocks = []
    for m in re.finditer(r"setBlock\(initKron,\s*(\d+),\s*(\d+),\s*" + CPLX + r",\s*" + CPLX + r"\)", body):
        blocks.append({"out": int(m.group(1)), "in": int(m.group(2)),
                       "A": cplx(m.group(3, 4)), "B": cplx(m.group(5, 6))})
    inp = re.search(r"const VectorType\s+input\s*\{\s*" + CPLX + r",\s*" + CPLX + r"\s*\}", body)
    checks = re.findall(r"checkVector\(multiply\(matrix, input\),\s*\{\s*" + CPLX + r",\s*" + CPLX + r"\s*\}", body)
    xout = re.search(r"initKron\.xout_ = \{\s*" + CPLX + r",\s*" + CPLX + r"\s*\}", body)
    fwd = re.search(r"checkVector\(initKron\.xout_,\s*\{\s*" + CPLX + r",\s*" + CPLX + r"\s*\}\)", body)
    out = {"source": "dmrg/Engine/tests/test_KronConnections.cpp:132-178",
           "blocks": blocks,
           "input": [cplx(inp.group(1, 2)), cplx(inp.group(3, 4))],
           "expected_H_input": [cplx(checks[0][0:2]), cplx(checks[0][2:4])],
           "x_out_before": [cplx(xout.group(1, 2)), cplx(xout.group(3, 4))],
           "expected_x_out_plus_H_input": [cplx(fwd.group(1, 2)), cplx(fwd.group(3, 4))]}
    assert len(blocks) == 4
    json.dump(out, open(os.path.join(HERE, "kron_connections_complex.json"), "w"), indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
