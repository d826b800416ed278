"""The autotuner's cache key on the CPU: tuning_key_check.cpp builds
spin-chain-like sector plans (kron_plan.cpp) and checks that a sweep step's
small patch-size changes keep the key while another sector shape, term count
or GPU changes it."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "dmrgpp_b200", "csrc")


def test_tuning_key(tmp_path):
    exe = str(tmp_path / "tuning_key_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
                    os.path.join(HERE, "tuning_key_check.cpp"), os.path.join(CSRC, "kron_plan.cpp"),
                    "-o", exe, "-lpthread"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.startswith("ok"), out.stdout + out.stderr
