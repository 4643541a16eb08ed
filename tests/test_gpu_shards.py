"""The multi-GPU path on one GPU: two processes (gloo for the host plumbing) each step their own shard of one
world set, split by body count, on cuda:0. Their kernels never wait on each other, so the two processes may
share the device. Every world's state, gathered to rank 0, is bit for bit the state a single process reaches
stepping the whole set as one batch."""
import os
import pickle
import socket
import subprocess
import sys

import numpy as np
import pytest

from twofold_b200 import scenes
from twofold_b200.world import Batch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_WORLDS, STEPS = 48, 12

RANK_SCRIPT = r'''
import os, pickle, sys
sys.path.insert(0, os.environ["TF_ROOT"])
import bench
from twofold_b200 import scenes, shard
from twofold_b200.world import Batch
d = bench.Dist(backend="gloo", timeout_s=120)
n_worlds, steps = int(os.environ["TF_WORLDS"]), int(os.environ["TF_STEPS"])
shards = shard.lpt_partition(scenes.config4_bodies(n_worlds), d.world_size)
sc = scenes.config4(n_worlds=n_worlds, only=shards[d.rank])
b = Batch.from_scene(sc, device=0)
b.step_checked(sc.dt, steps, graph=True)
mine = {int(w): b.world_states(k) for k, w in enumerate(shards[d.rank])}
b.close()
d.barrier()
gathered = [None] * d.world_size
d.pg.all_gather_object(gathered, mine)
if d.rank == 0:
    whole = {}
    for g in gathered:
        whole.update(g)
    with open(os.environ["TF_OUT"], "wb") as f:
        pickle.dump(whole, f)
d.close()
'''


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_shards_on_one_gpu_match_one_batch(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    out_file = tmp_path / "states.pkl"
    env = dict(os.environ, TF_ROOT=ROOT, TF_OUT=str(out_file), TF_WORLDS=str(N_WORLDS), TF_STEPS=str(STEPS))
    cmd = ["timeout", "-k", "30", "600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(script)]
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=700)
    assert res.returncode == 0, res.stderr[-3000:]
    with open(out_file, "rb") as f:
        sharded = pickle.load(f)
    assert sorted(sharded) == list(range(N_WORLDS))
    sc = scenes.config4(n_worlds=N_WORLDS)
    b = Batch.from_scene(sc)
    b.step_checked(sc.dt, STEPS, graph=True)
    for w in range(N_WORLDS):
        one = b.world_states(w)
        for k in ("p", "q", "v", "w"):
            assert np.array_equal(np.asarray(one[k]).view(np.uint32), np.asarray(sharded[w][k]).view(np.uint32)), \
                f"world {w} {k}"
