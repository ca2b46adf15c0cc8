"""The N > 1 host path of bench.py on CPU: two gloo ranks (one process each, as torchrun
launches them) agree on barrier and max-over-ranks, get distinct replica seeds, and the
reference arm prints only on rank 0."""
import os
import socket
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import bench
g = bench.RankGroup("gloo")
g.barrier()
m = g.max(10.0 * (g.rank + 1))
cfg = bench.make_case("small", bench.replica_seed(g.rank))
print(json.dumps({{"rank": g.rank, "world": g.world, "max": m, "seed": int(cfg.seed)}}), flush=True)
g.close()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _launch(code, world=2, extra_env=None, timeout=120):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, e
        outs.append(o)
    return outs


def test_two_gloo_ranks_reduce_and_seed_replicas():
    import json
    outs = _launch(WORKER.format(root=ROOT))
    rows = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(r["rank"] for r in rows) == [0, 1]
    assert all(r["world"] == 2 for r in rows)
    assert all(r["max"] == 20.0 for r in rows)
    assert rows[0]["seed"] != rows[1]["seed"]


def test_reference_arm_prints_on_rank_zero_only(tmp_path):
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); sys.argv = ['bench.py', '--impl', 'reference', "
            "'--case', 'small', '--steps', '2', '--warmup', '1']; import bench; sys.exit(bench.main())")
    outs = _launch(code, timeout=300)
    import json
    line = json.loads(outs[0].strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert outs[1].strip() == ""


SLAB_WORKER = r"""
import json, os, sys
sys.path.insert(0, {root!r})
import torch, torch.distributed as dist
from mrlbm_2d_b200.slabs import SlabExchange
dist.init_process_group("gloo")
r, w = dist.get_rank(), dist.get_world_size()
got = {{}}
def pack(side, t):
    t.fill_(100.0 * r + side)                  # this rank's face `side`
def unpack(side, t):
    got[side] = float(t[0])
ex = SlabExchange(r, w, pack, unpack, 12, torch.float64, torch.device("cpu"))
ex.exchange()
print(json.dumps({{"rank": r, "got": got}}), flush=True)
dist.destroy_process_group()
"""


def test_slab_halo_exchange_between_three_gloo_ranks():
    """Each slab receives its left neighbour's right face into side 0 and its right neighbour's
    left face into side 1; the end slabs have one neighbour."""
    import json
    outs = _launch(SLAB_WORKER.format(root=ROOT), world=3)
    rows = {json.loads(o.strip().splitlines()[-1])["rank"]: json.loads(o.strip().splitlines()[-1])["got"] for o in outs}
    assert rows[0] == {"1": 100.0}
    assert rows[1] == {"0": 1.0, "1": 200.0}
    assert rows[2] == {"0": 101.0}


def test_partition_keeps_the_cylinder_whole():
    from mrlbm_2d_b200.slabs import partition
    assert partition(400, 3, (65, 95)) == [(1, 133), (134, 266), (267, 400)]
    parts = partition(400, 4, (90, 110))
    assert any(a < 90 and 110 < b for (a, b) in parts)          # strictly inside one slab
    for (a, b), (c, d) in zip(parts, parts[1:]):
        assert b + 1 == c
    assert parts[0][0] == 1 and parts[-1][1] == 400
