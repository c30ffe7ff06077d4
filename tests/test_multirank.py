"""The multi-rank path of bench.py on CPU: two torchrun ranks over gloo.  The ranks exchange only
timings (max / sum / barrier); under --impl reference rank 0 alone times the reference and prints
the JSON line, the other rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

import _oracle as O

HARNESS = os.path.join(O.REPO, "oracle", "_ref", "8x8x8x8", "harness")


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _torchrun(args, timeout=300):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_port())] + args
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    return subprocess.run(cmd, cwd=O.REPO, capture_output=True, text=True, timeout=timeout, env=env)


def test_dist_reductions_over_gloo(tmp_path):
    script = tmp_path / "ranks.py"
    script.write_text(
        "import json, os, sys\n"
        f"sys.path.insert(0, {O.REPO!r})\n"
        "import bench\n"
        "d = bench.Dist()\n"
        "assert d.world == 2 and not d.gpu\n"
        "d.barrier()\n"
        "out = {'rank': d.rank, 'max': d.max(10.0 + d.rank), 'sum': d.sum(1.5)}\n"
        "d.close()\n"
        # one file per rank: the two ranks' stdout lines can interleave under torchrun
        f"open(os.path.join({str(tmp_path)!r}, 'rank%d.json' % out['rank']), 'w').write(json.dumps(out))\n")
    r = _torchrun([str(script)])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    assert all(x["max"] == 11.0 and x["sum"] == 3.0 for x in lines)


def test_reference_arm_under_two_ranks():
    if not os.path.exists(HARNESS):
        pytest.skip("reference harness not built")
    r = _torchrun(["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
                   "--dims", "8,8,8,8"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1   # rank 0 only
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
