"""bench.py's multi-GPU plumbing on CPU: two ranks under torch.distributed.run (gloo,
127.0.0.1), as the driver launches the bench for N > 1 - the max-over-ranks timing, the
whole-job rate and the reference arm's rank-0-only rule."""
import json
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_slowest_rank(tmp_path):
    cmd = ["timeout", "-k", "10", "180", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node=2", "--master-addr=127.0.0.1", f"--master-port={_free_port()}",
           os.path.join(HERE, "multirank_worker.py"), str(tmp_path)]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    got = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(2)]
    for g in got:
        assert g["ws"] == 2
        assert g["slowest"] == 2.5                       # every rank sees the slowest rank's time
        assert abs(g["rate"] - 2 * 1000.0 * 4 / 2.5) < 1e-9
    assert got[1]["reference_rc"] == 0                   # the reference arm exits at once off rank 0
