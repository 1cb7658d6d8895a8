"""The bench's multi-process plumbing on CPU: two gloo ranks rendezvous on
127.0.0.1, barrier, and agree on the max of their step times (the replica path of
`bench.py --gpus N`, whose data path has no exchange)."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import os, sys, json
sys.path.insert(0, {root!r})
import bench
world, rank, local = bench.dist_setup(None, backend="gloo")
bench.barrier(world)
m = bench.max_over_ranks(1.5 + rank, world)
bench.barrier(world)
with open(os.path.join({out!r}, "rank%d.json" % rank), "w") as f:
    f.write(json.dumps({{"rank": rank, "world": world, "max": m}}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_max_and_barrier(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(SCRIPT.format(root=ROOT, out=str(tmp_path)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(script)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env={**os.environ, "OMP_NUM_THREADS": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    import json
    res = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert {r["rank"] for r in res} == {0, 1}
    assert all(r["world"] == 2 and r["max"] == 2.5 for r in res)
