"""The multi-process path of bench.py on CPU: two ranks over gloo, launched the way the driver launches the
bench (torchrun, one process per rank, 127.0.0.1). The ranks' reductions give the max of their times and the
sum of their work, every rank takes the same collective steps, and the reference arm prints one line from rank
0 while rank 1 exits without work."""
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
import bench
d = bench.Dist(backend="gloo", timeout_s=60)
rank = d.rank
d.barrier()
mx = d.reduce(10.0 + rank, "MAX")
sm = d.reduce(100.0 * (rank + 1), "SUM")
d.barrier()
from twofold_b200 import scenes
# Each rank steps its own batch: the batched scene is seeded by the rank.
first = scenes.config4(n_worlds=4, seed=rank).worlds[0]
print(json.dumps({"rank": rank, "world_size": d.world_size, "max": mx, "sum": sm,
                  "bodies": len(first.bodies), "x0": float(first.bodies["position"][1][0])}), flush=True)
d.close()
'''


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _torchrun(args, timeout=240):
    env = dict(os.environ, TF_ROOT=ROOT, CUDA_VISIBLE_DEVICES="")
    cmd = ["timeout", "-k", "30", str(timeout), sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "2", "--master-addr", "127.0.0.1", "--master-port", str(_free_port())] + args
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=timeout + 60)


def test_two_ranks_reduce_and_partition_over_gloo(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    out = _torchrun([str(script)])
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(l) for l in out.stdout.splitlines() if l.startswith("{")]
    assert sorted(l["rank"] for l in lines) == [0, 1]
    for l in lines:
        assert l["world_size"] == 2
        assert l["max"] == 11.0 and l["sum"] == 300.0
    # The ranks' batches differ: each rank's worlds are its own.
    a, b = sorted(lines, key=lambda l: l["rank"])
    assert (a["bodies"], a["x0"]) != (b["bodies"], b["x0"])


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
