"""CPU check of the wave-function transformation plan (no GPU): the host
emulation in wft_plan_check.cpp replays both grouped GEMM passes from the
plan's lists and packed blocks and compares with the direct per-patch
products (see that file for the list of checks)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "dmrgpp_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("wft") / "wft_plan_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "wft_plan_check.cpp"), os.path.join(CSRC, "wft_plan.cpp"),
                    "-o", exe, "-lpthread"], check=True)
    return exe


@pytest.mark.parametrize("seed,npi,npo,maxs,tl,tr", [
    (1, 1, 1, 1, 0, 0), (2, 3, 4, 9, 0, 0), (3, 5, 5, 40, 1, 0), (4, 4, 6, 70, 0, 1),
    (5, 6, 3, 33, 1, 1), (6, 2, 2, 200, 0, 0), (7, 8, 8, 25, 1, 1), (8, 3, 5, 130, 1, 0)])
def test_transformation_plan(checker, seed, npi, npo, maxs, tl, tr):
    out = subprocess.run([checker, str(seed), str(npi), str(npo), str(maxs), str(tl), str(tr)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
