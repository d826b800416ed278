"""CPU check of the fused H*x schedule (no GPU): the host emulation in
fused_schedule_check.cpp replays every item of the fused launch for several
tile shapes, cluster sizes and work splits, checks the cluster placement of
the parts, the bounds of every operand load and store, and recomputes H*x
from the packed operators (see that file for the list of checks)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "dmrgpp_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("fused") / "fused_schedule_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "fused_schedule_check.cpp"),
                    os.path.join(CSRC, "kron_plan.cpp"), "-o", exe, "-lpthread"], check=True)
    return exe


@pytest.mark.parametrize("seed,np_,nop,maxs", [
    (1, 1, 1, 1), (2, 3, 2, 9), (3, 5, 3, 40), (4, 4, 2, 150), (5, 6, 4, 70),
    (6, 2, 2, 260), (7, 8, 5, 33), (8, 12, 5, 110), (9, 21, 5, 120)])
def test_fused_items_loads_stores_and_result(checker, seed, np_, nop, maxs):
    out = subprocess.run([checker, str(seed), str(np_), str(nop), str(maxs)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
