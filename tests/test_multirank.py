"""The multi-GPU form of bench.py on CPU: two ranks over gloo (one process each, as torchrun starts them) take the
same collective the benchmark takes after its timed steps, and get the slowest rank's time and the rows of both.
The device path itself does not span GPUs (frames shard with no exchange), so this aggregation is the whole of the
N > 1 logic."""
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys
sys.path.insert(0, sys.argv[1])
import torch, torch.distributed as dist
import bench
rank = int(os.environ["RANK"])
dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
ms, rows = bench.over_ranks(dist, torch, 10.0 + 5.0 * rank, 1000 + rank, "cpu")
print("RESULT", rank, ms, rows, flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo():
    port = _port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    for rank, out in enumerate(outs):
        line = [l for l in out.splitlines() if l.startswith("RESULT")][0].split()
        assert int(line[1]) == rank and float(line[2]) == 15.0 and float(line[3]) == 2001.0
