"""The benchmark's multi-rank plumbing without a GPU: the MAX-over-ranks
timing reduction and the barrier on two gloo ranks, and the reference arm's
rank behaviour (rank 0 prints one line, other ranks exit 0 silently)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.rank_barrier(dist, world)
        got = bench.reduce_max(dist, world, 1.5 + rank, "cpu")
        bench.rank_barrier(dist, world)
    finally:
        dist.destroy_process_group()
    with open(f"{out}.{rank}", "w") as f:
        f.write(repr(got))


def test_max_over_ranks_on_two_gloo_ranks(tmp_path):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "res")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert [float(open(f"{out}.{r}").read()) for r in range(2)] == [2.5, 2.5]


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_prints_on_rank_zero_only(rank):
    import oracle
    oracle.build()
    if not oracle.ref_available():
        pytest.skip("reference CPU build not present")
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    if rank != 0:
        assert lines == []
        return
    line = json.loads(lines[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    for key in ("metric", "value", "unit", "cpu_baseline", "e2e", "config"):
        assert key in line
    assert line["e2e"]["h2d_bytes_per_step"] == 0
