"""Host side of the data-parallel (sharded-by-points) sampler, on CPU: the shard partition and the
exchange callbacks that the native sampler calls (dpmm_allreduce_fn), over a world_size-2 gloo process
group and over threads of one process.  The device side is covered by tests/test_gpu_shard.py."""
import ctypes
import os
import socket
import subprocess
import sys
import threading

import numpy as np
import pytest

from conftest import ROOT
from dpmmsubclusters_gpu_b200.shard import LocalGroupExchange, TorchDistributedExchange, shard_bounds


@pytest.mark.parametrize("n,world", [(10, 1), (10, 3), (1000003, 8), (16, 16), (7, 2)])
def test_shard_bounds_partition_every_point_once(n, world):
    seen = np.zeros(n, np.int32)
    prev_end = 0
    for r in range(world):
        off, cnt = shard_bounds(n, world, r)
        assert off == prev_end and cnt >= n // world
        seen[off:off + cnt] += 1
        prev_end = off + cnt
    assert prev_end == n and np.all(seen == 1)
    with pytest.raises(ValueError):
        shard_bounds(n, world, world)


def _call(ex, a):
    """Invoke the exchange the way the native sampler does: through its C function pointer."""
    return ex.callback(None, a.ctypes.data_as(ctypes.c_void_p), a.size, None)


def test_local_group_exchange_threads_sum_in_rank_order():
    world = 3
    g = LocalGroupExchange(world, device=False)
    rng = np.random.default_rng(0)
    # values whose sum depends on the order of the additions: every rank must get the rank-order sum
    parts = [rng.normal(size=1000) * 10.0 ** rng.integers(-8, 8, size=1000) for _ in range(world)]
    out = [None] * world
    rcs = [None] * world

    def run(r):
        bufs = []
        for step in range(3):                 # several exchanges of different sizes, in the same order
            a = parts[r][: 1000 - 100 * step].copy()
            rcs[r] = _call(g.ranks[r], a)
            bufs.append(a)
        out[r] = bufs

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=60)
    assert rcs == [0] * world
    for step in range(3):
        n = 1000 - 100 * step
        expect = parts[0][:n].copy()
        for p in parts[1:]:
            expect += p[:n]
        for r in range(world):
            assert np.array_equal(out[r][step], expect)      # bit-identical on every rank


_GLOO_CHILD = r"""
import ctypes, os, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
from dpmmsubclusters_gpu_b200.shard import TorchDistributedExchange, shard_bounds
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="tcp://127.0.0.1:" + sys.argv[2], rank=rank, world_size=world)
ex = TorchDistributedExchange(device=False)
# the statistics exchange of a sharded data set: each rank holds the per-cluster count / sum / scatter
# of its own points; after the exchange every rank holds the whole data set's
rng = np.random.default_rng(42)
N, D, K = 5000, 3, 4
x = rng.normal(size=(N, D))
z = rng.integers(0, K, size=N)
off, n = shard_bounds(N, world, rank)
xs, zs = x[off:off + n], z[off:off + n]
stats = np.concatenate([np.concatenate([[np.sum(zs == k)], xs[zs == k].sum(0), (xs[zs == k].T @ xs[zs == k]).ravel()])
                        for k in range(K)])
rc = ex.callback(None, stats.ctypes.data_as(ctypes.c_void_p), stats.size, None)
full = np.concatenate([np.concatenate([[np.sum(z == k)], x[z == k].sum(0), (x[z == k].T @ x[z == k]).ravel()])
                       for k in range(K)])
assert rc == 0
assert np.allclose(stats, full, rtol=1e-12, atol=1e-9), np.abs(stats - full).max()
# every rank must hold the same bits
g = [None] * world
dist.all_gather_object(g, stats.tobytes())
assert all(b == g[0] for b in g)
assert ex.calls == 1 and ex.values == stats.size
dist.destroy_process_group()
print("OK", rank)
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_torch_distributed_exchange_gloo_world_size_2():
    port = str(_free_port())
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
        procs.append(subprocess.Popen([sys.executable, "-c", _GLOO_CHILD, ROOT, port], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=240) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, o + e
        assert "OK" in o


def test_exchange_failure_is_reported_to_the_caller():
    class Broken(TorchDistributedExchange):
        def allreduce(self, buf, count, stream):
            raise RuntimeError("peer lost")
    ex = Broken(device=False)
    a = np.ones(4)
    assert _call(ex, a) == 1 and "peer lost" in str(ex.error)
