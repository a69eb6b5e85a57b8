"""The N > 1 plumbing of bench.py (plasticity_b200/replicas.py) on the CPU:
two rank processes over gloo (127.0.0.1) share a barrier and the maximum of
their times; a rank whose peer never joins ends with an error within the
group's short timeout instead of waiting for good."""
import os
import socket
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_CODE = r"""
import sys
sys.path.insert(0, {root!r})
from plasticity_b200.replicas import Replicas
r = Replicas("gloo", timeout_s={timeout})
r.barrier()
print("MAX", r.max_over_ranks(10.0 + 5.0 * r.rank), flush=True)
r.close()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(rank, world, port, timeout):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    return subprocess.Popen([sys.executable, "-c", RANK_CODE.format(root=ROOT, timeout=timeout)], env=env,
                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)


def test_two_replicas_barrier_and_max_over_ranks():
    port = _free_port()
    procs = [_launch(r, 2, port, 60) for r in range(2)]
    outs = [p.communicate(timeout=120) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
        assert "MAX 15.0" in o, (o, e)


def test_missing_peer_fails_within_the_timeout():
    port = _free_port()
    t0 = time.time()
    p = _launch(0, 2, port, 5)
    o, e = p.communicate(timeout=120)
    assert p.returncode != 0
    assert time.time() - t0 < 90
