"""The library's host thread count (host_threads in kron_plan.h):
DMRGPP_HOST_THREADS when set, otherwise the CPUs of the process's affinity
mask (taskset), at most 32."""
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
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + CSRC, os.path.join(HERE, "host_threads_check.cpp"),
                    "-o", out, "-lpthread"], check=True)
    return out


def _run(cmd, **env):
    e = dict(os.environ)
    e.pop("DMRGPP_HOST_THREADS", None)
    e.update(env)
    return int(subprocess.run(cmd, capture_output=True, text=True, env=e, check=True).stdout)


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
