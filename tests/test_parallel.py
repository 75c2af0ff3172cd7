"""Multi-process host logic on CPU: two gloo ranks exercise the barrier, the
max/sum over ranks used for timing, and the cost-balanced batch sharding
(every matrix owned by exactly one rank, loads balanced)."""
import os
import socket
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


WORKER = r"""
import os, sys, json, datetime
sys.path.insert(0, {root!r})
import numpy as np, torch.distributed as dist
from mex_linear_algebra_b200 import parallel, gen
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ws, rank, _ = parallel.world()
parallel.barrier(ws)
mx = parallel.max_over_ranks(ws, 10.0 + rank)
sm = parallel.sum_over_ranks(ws, 1.0 + rank)
shapes = np.array([gen.ldpc_shape(3, b) for b in range(200)])
mine = parallel.shard_batch(shapes, ws, rank)
cost = parallel.batch_cost(shapes)[mine].sum()
tot = parallel.sum_over_ranks(ws, cost)
cnt = parallel.sum_over_ranks(ws, len(mine))
print(json.dumps({{"rank": rank, "max": mx, "sum": sm, "mine": mine.tolist(), "cost": cost,
                  "total_cost": tot, "count": cnt}}))
dist.destroy_process_group()
"""


def test_two_gloo_ranks():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=120)
        assert p.returncode == 0, e
        import json
        outs.append(json.loads(o.strip().splitlines()[-1]))
    assert all(o["max"] == 11.0 and o["sum"] == 3.0 for o in outs)
    owned = sorted(outs[0]["mine"] + outs[1]["mine"])
    assert owned == list(range(200))            # each matrix on exactly one rank
    assert outs[0]["count"] == 200
    c0, c1 = outs[0]["cost"], outs[1]["cost"]
    assert abs(c0 - c1) / (c0 + c1) < 0.02       # balanced by estimated cost


def test_shard_single_rank_owns_all():
    from mex_linear_algebra_b200 import parallel
    sh = np.array([[100, 200], [64, 130], [1000, 2000]])
    assert list(parallel.shard_batch(sh, 1, 0)) == [0, 1, 2]
