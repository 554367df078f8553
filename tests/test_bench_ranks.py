"""bench.py's multi-rank plumbing on CPU: two gloo ranks (as torchrun starts
them) meet at the barrier and agree on the maximum of their step times, and
the replica value is the whole-job aggregate."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, %r)
    import bench
    world, rank, local, pg = bench.dist_setup(2)
    bench.barrier(pg)
    mine = 10.0 + 5.0 * rank
    ms = bench.max_over_ranks(pg, mine)
    cells, steps = 1000, 4
    value = world * cells * steps / (ms / 1e3)
    print(json.dumps({"rank": rank, "world": world, "ms": ms, "value": value}))
    pg.destroy_process_group()
""") % ROOT


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_take_the_max_time():
    import json
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["ms"] == 15.0
        assert abs(o["value"] - 2 * 1000 * 4 / 0.015) < 1e-6
