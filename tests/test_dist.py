"""The multi-process path of bench.py on CPU: two ranks over gloo, launched the way the driver launches the
bench (torchrun, one process per rank, 127.0.0.1). The ranks' reductions give the max of their times and the
sum of their work, every rank takes the same collective steps, one world set is split over the ranks by body
count and gathered back whole, and the reference arm prints one line from rank 0 while rank 1 exits without
work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r'''
import json, os, sys
sys.path.insert(0, os.environ["TF_ROOT"])
import numpy as np
import bench
from twofold_b200 import scenes, shard
d = bench.Dist(backend="gloo", timeout_s=60)
rank = d.rank
d.barrier()
mx = d.reduce(10.0 + rank, "MAX")
sm = d.reduce(100.0 * (rank + 1), "SUM")
d.barrier()
# One world set of 64 worlds, split by body count; each rank builds only its own worlds.
counts = scenes.config4_bodies(64)
shards = shard.lpt_partition(counts, d.world_size)
mine = scenes.config4(n_worlds=64, only=shards[rank])
digest = {int(w): float(np.abs(x.bodies["position"].astype(np.float64)).sum() + len(x.bodies))
          for w, x in zip(shards[rank], mine.worlds)}
gathered = [None] * d.world_size
d.pg.all_gather_object(gathered, digest)
union = {}
for g in gathered:
    union.update({str(k): v for k, v in g.items()})
# Long lines from two processes interleave on one pipe: each rank writes its own file.
with open(os.path.join(os.environ["TF_OUT"], f"rank{rank}.json"), "w") as f:
    json.dump({"rank": rank, "world_size": d.world_size, "max": mx, "sum": sm,
               "shard": shards[rank], "loads": shard.shard_loads(counts, shards), "union": union}, f)
d.close()
'''


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, timeout=240, out_dir=""):
    env = dict(os.environ, TF_ROOT=ROOT, TF_OUT=str(out_dir), CUDA_VISIBLE_DEVICES="")
    cmd = ["timeout", "-k", "30", str(timeout), sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port", str(_free_port())] + args
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout + 60)


def test_two_ranks_reduce_and_partition_over_gloo(tmp_path):
    """Two ranks split one 64-world set by body count, build only their own worlds, and gather a digest of
    each world to every rank: the union is the whole set, world for world equal to one process building all of
    it, and the two ranks' bodies differ by less than the largest world."""
    import numpy as np

    sys.path.insert(0, ROOT)
    from twofold_b200 import scenes

    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    out = _torchrun([str(script)], out_dir=tmp_path)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    for l in lines:
        assert l["world_size"] == 2
        assert l["max"] == 11.0 and l["sum"] == 300.0
    a, b = sorted(lines, key=lambda l: l["rank"])
    assert sorted(a["shard"] + b["shard"]) == list(range(64)) and not set(a["shard"]) & set(b["shard"])
    counts = scenes.config4_bodies(64)
    assert abs(a["loads"][0] - a["loads"][1]) <= int(counts.max())
    whole = scenes.config4(n_worlds=64)
    expect = {str(w): float(np.abs(x.bodies["position"].astype(np.float64)).sum() + len(x.bodies))
              for w, x in enumerate(whole.worlds)}
    assert a["union"] == expect and b["union"] == expect


def test_lpt_partition_is_balanced_and_deterministic():
    sys.path.insert(0, ROOT)
    from twofold_b200 import scenes, shard

    counts = scenes.config4_bodies(4096 * 8)
    for n in (1, 2, 4, 8):
        shards = shard.lpt_partition(counts, n)
        assert sorted(w for s in shards for w in s) == list(range(len(counts)))
        loads = shard.shard_loads(counts, shards)
        assert max(loads) - min(loads) <= int(counts.max())
        assert shards == shard.lpt_partition(counts, n)
    assert shard.lpt_partition([5, 3, 3, 1], 2) == [[0, 3], [1, 2]]


def test_reference_arm_runs_on_rank_zero_only():
    pytest.importorskip("torch")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as R

    if not R.available():
        pytest.skip("oracle library not built")
    out = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--worlds", "8", "--steps", "2", "--warmup", "1"])
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "reference"
