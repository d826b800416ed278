"""CPU check of the TF32x3 operand layout and copy plan (no GPU): the host
emulation in mixed_layout_check.cpp replays every bulk copy and store the
tensor-core kernel would issue for a sector and recomputes H*x from the
copied blocks (see that file for the list of checks)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "dmrgpp_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("mixed") / "mixed_layout_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "mixed_layout_check.cpp"),
                    os.path.join(CSRC, "kron_plan.cpp"), "-o", exe, "-lpthread"], check=True)
    return exe


@pytest.mark.parametrize("seed,np_,nop,maxs,bn", [
    (1, 1, 1, 1, 64), (2, 3, 2, 9, 64), (3, 5, 3, 40, 64), (4, 4, 2, 150, 128),
    (5, 6, 4, 70, 128), (6, 2, 2, 260, 128), (7, 8, 5, 33, 64), (8, 3, 3, 129, 64),
    (9, 12, 5, 110, 64), (10, 8, 4, 150, 128)])
def test_copies_stores_and_result(checker, seed, np_, nop, maxs, bn):
    out = subprocess.run([checker, str(seed), str(np_), str(nop), str(maxs), str(bn)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr


def test_small_sectors_get_k_split_tiles(checker):
    """Sectors with few pass-2 tiles are cut along K (several parts per tile)."""
    out = subprocess.run([checker, "9", "12", "5", "110", "64"], capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout
    assert int(out.stdout.split()[-1]) > 0
