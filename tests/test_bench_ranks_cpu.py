"""bench.py's multi-rank path on the host: `--gpus 2` with no launcher in the
environment starts two ranks itself (torch.distributed.run on 127.0.0.1), the
ranks take their weak-scaling Sobol ranges, and the one exchange (the rank's
matrix read into a buffer, then summed over ranks) leaves rank 0 holding the
matrix that one process builds over both ranks' ranges.  The build is
bench.HostStandIn (numpy), the backend gloo; no GPU is involved."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from scp3_b200 import shard  # noqa: E402


def test_two_ranks_launch_and_reduce(tmp_path):
    out = str(tmp_path / "M.npy")
    steps, warmup, n = 2, 3, 64
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--standin",
                        "--steps", str(steps), "--warmup", str(warmup), "--samples", str(n),
                        "--dump-matrix", out], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(x) for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, p.stdout          # rank 0 alone prints
    line = lines[0]
    assert line["n_gpus"] == 2 and line["steps"] == steps and line["config"]["parallelism"] == "dp2 (sample ranges)"
    M2 = np.load(out)
    # one process over both ranks' timed ranges (the warm-up steps are reset away)
    ref = bench.HostStandIn()
    for r in range(2):
        base, _ = shard.sample_range(r, 2, 0, n, "weak")
        for k in range(warmup, warmup + steps):
            ref.accumulate(base + k * n, n)
    scale = np.abs(ref.M).max()
    assert np.abs(M2 - ref.M).max() <= 1e-12 * scale
    # and not what either rank holds alone
    alone = bench.HostStandIn()
    for k in range(warmup, warmup + steps):
        alone.accumulate(k * n, n)
    assert np.abs(M2 - alone.M).max() > 1e-3 * scale


def test_exchange_reads_before_it_reduces(monkeypatch):
    import torch
    calls = []

    class Recorder(bench.HostStandIn):
        def read_dev(self, ptr, ld, mode=0):
            calls.append("read")
            super().read_dev(ptr, ld, mode)

    def reduce(M, group=None):
        calls.append("reduce")
        assert torch.equal(M, torch.from_numpy(hb.M))     # the rank's own matrix is in place
        return M

    monkeypatch.setattr(shard, "reduce_matrix", reduce)
    hb = Recorder()
    hb.accumulate(5, 40)
    M = torch.zeros((hb.nb, hb.nb), dtype=torch.float64)
    bench.exchange(hb, M, None)
    assert calls == ["read", "reduce"]


def test_launcher_refuses_a_rank_count_mismatch(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "3")
    try:
        bench.dist_setup(2, "gloo")
    except SystemExit as e:
        assert "--gpus 2" in str(e)
    else:
        raise AssertionError("dist_setup accepted 3 ranks for --gpus 2")
