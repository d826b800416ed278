"""CPU check of the persistent FP64 H*x schedule (no GPU): the host emulation
in persistent_schedule_check.cpp replays every work item of the persistent
launch (pass-1 tiles of BX_j, pass-2 output tiles whole or cut along K) for
every tile shape and K-chunk of the launch configurations and several grid
sizes, checks the bounds of every operand load and store, that each pass-2
load reads only BX rows its dependency's pass-1 items wrote, that every BX
and Y element is written once, and recomputes H*x from the packed operators
(see that file for the list of checks)."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "dmrgpp_b200", "csrc")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("persistent") / "persistent_schedule_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "persistent_schedule_check.cpp"),
                    os.path.join(CSRC, "kron_plan.cpp"), "-o", exe, "-lpthread"], check=True)
    return exe


@pytest.mark.parametrize("seed,np_,nop,maxs", [
    (1, 1, 1, 1), (2, 3, 2, 9), (3, 6, 3, 40), (4, 4, 2, 130), (5, 12, 5, 70),
    (6, 2, 2, 200), (7, 20, 4, 20), (11, 40, 3, 3), (12, 2, 2, 300)])
def test_persistent_items_loads_stores_and_result(checker, seed, np_, nop, maxs):
    out = subprocess.run([checker, str(seed), str(np_), str(nop), str(maxs)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr


@pytest.fixture(scope="module")
def group_checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("group") / "group_schedule_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "group_schedule_check.cpp"),
                    os.path.join(CSRC, "kron_plan.cpp"), "-o", exe, "-lpthread"], check=True)
    return exe


@pytest.mark.parametrize("seed,nsec,maxp,maxk,maxs", [
    (1, 1, 4, 3, 30), (2, 4, 5, 3, 30), (3, 7, 3, 4, 20), (4, 2, 8, 5, 60), (5, 12, 2, 2, 12),
    (23, 50, 1, 1, 1)])
def test_group_items_stay_in_their_sector(group_checker, seed, nsec, maxp, maxk, maxs):
    """Sectors of a group launch are isolated: pass-2 segments depend only on
    their own sector's patches, and with any one sector's items skipped (as
    the masked group solvers do) the others still give their own H*x while
    the skipped sector's output stays as it was (group_schedule_check.cpp)."""
    out = subprocess.run([group_checker, str(seed), str(nsec), str(maxp), str(maxk), str(maxs)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
