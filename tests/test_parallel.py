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


SHARDED_WORKER = r"""
import os, sys, json, datetime
sys.path.insert(0, {root!r})
sys.path.insert(0, os.path.join({root!r}, "oracle"))
import numpy as np, torch.distributed as dist
import oracle as O
from mex_linear_algebra_b200 import parallel, gen
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ws, rank, _ = parallel.world()
shapes = np.array([gen.ldpc_shape(3, b) for b in range(120)])
calls = []

def compute(idx):
    # this rank's share, by the oracle on the CPU (the GPU run uses the batch engine)
    out = {{}}
    for i in idx:
        calls.append(int(i))
        m, n, P = gen.ldpc_packed(3, int(i))
        out[int(i)] = int(O.rank(P, m, n, 10))
    return out

merged, owners = parallel.run_sharded(shapes, ws, rank, compute)
print(json.dumps({{"rank": rank, "calls": calls, "owners": owners,
                  "ranks": [merged[i] for i in range(len(shapes))]}}))
dist.destroy_process_group()
"""


def test_sharded_batch_two_gloo_ranks():
    """A parity-check batch split over two ranks: every matrix computed by
    exactly one rank, the gathered results complete on both ranks and equal
    to a single-process run."""
    import json
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from mex_linear_algebra_b200 import gen
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", SHARDED_WORKER.format(root=ROOT)], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e
        outs.append(json.loads(o.strip().splitlines()[-1]))
    calls = sorted(outs[0]["calls"] + outs[1]["calls"])
    assert calls == list(range(120))                       # each matrix computed once
    assert outs[0]["owners"] == outs[1]["owners"]
    want = [int(O.rank(gen.ldpc_packed(3, b)[2], *gen.ldpc_shape(3, b), 10)) for b in range(120)]
    assert outs[0]["ranks"] == want and outs[1]["ranks"] == want


def test_run_sharded_detects_gaps():
    import pytest
    from mex_linear_algebra_b200 import parallel
    sh = np.array([[10, 20]] * 5)
    merged, owners = parallel.run_sharded(sh, 1, 0, lambda idx: {int(i): int(i) * 2 for i in idx})
    assert merged == {i: 2 * i for i in range(5)} and owners == [[0, 1, 2, 3, 4]]
    with pytest.raises(RuntimeError):
        parallel.run_sharded(sh, 1, 0, lambda idx: {int(i): 0 for i in idx[:-1]})


def test_shard_single_rank_owns_all():
    from mex_linear_algebra_b200 import parallel
    sh = np.array([[100, 200], [64, 130], [1000, 2000]])
    assert list(parallel.shard_batch(sh, 1, 0)) == [0, 1, 2]
