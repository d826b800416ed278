"""The library's environment switches (kron_plan.h): the host thread count
(host_threads: DMRGPP_HOST_THREADS when set, otherwise the CPUs of the
process's affinity mask, at most 32) and the debug-mode check
(validation_requested: DMRGPP_VALIDATE set to a nonzero number)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "dmrgpp_b200", "csrc")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("threads") / "host_threads_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "host_threads_check.cpp"), os.path.join(CSRC, "kron_plan.cpp"),
                    "-o", out, "-lpthread"], check=True)
    return out


def _both(cmd, **env):
    e = dict(os.environ)
    e.pop("DMRGPP_HOST_THREADS", None)
    e.pop("DMRGPP_VALIDATE", None)
    e.update(env)
    out = subprocess.run(cmd, capture_output=True, text=True, env=e, check=True).stdout.split()
    return int(out[0]), int(out[1])


def _run(cmd, **env):
    return _both(cmd, **env)[0]


def test_environment_override(exe):
    assert _run([exe], DMRGPP_HOST_THREADS="3") == 3
    assert _run([exe], DMRGPP_HOST_THREADS="1000") == 256
    # not a positive count: ignored
    assert _run([exe], DMRGPP_HOST_THREADS="0") == _run([exe])


def test_affinity_mask(exe):
    n = _run([exe])
    assert 1 <= n <= 32 and n <= len(os.sched_getaffinity(0))
    if shutil.which("taskset") and len(os.sched_getaffinity(0)) >= 2:
        cpus = sorted(os.sched_getaffinity(0))[:2]
        assert _run(["taskset", "-c", ",".join(map(str, cpus)), exe]) == 2


def test_validation_switch(exe):
    assert _both([exe])[1] == 0
    assert _both([exe], DMRGPP_VALIDATE="1")[1] == 1
    assert _both([exe], DMRGPP_VALIDATE="0")[1] == 0
