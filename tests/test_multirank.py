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


FAKE_ARM = r'''
import json, os, sys
sys.path.insert(0, REPO)
import bench
import masterarbeit_b200.su2g as S

RANK = int(os.environ["RANK"])


class FakeLattice:
    """Host stand-in for a GPU lattice: every timed block of calls takes (5 + rank) ms, and the
    profiled pass reports one event-timed launch per call and kernel class."""

    def __init__(self, dims, **kw):
        self.calls = {"heatbath": 0, "plaquette": 0, "reduce": 0}
        self.profiling = False

    def sweep(self, n_sweeps=1, n_hb=1, n_or=0, acc=False):
        self.calls["heatbath"] += 8 * n_sweeps

    def plaquette(self):
        self.calls["plaquette"] += 1
        return 0.5

    def sweep_plaquette(self, n_sweeps=1, n_hb=1, n_or=0, acc=False):
        self.sweep(n_sweeps, n_hb, n_or)
        self.calls["reduce"] += 1
        return (0.5, 0.98) if acc else 0.5

    def synchronize(self):
        pass

    def timer_begin(self):
        pass

    def timer_end(self):
        return 5.0 + RANK

    def profile(self, on=True):
        self.profiling = on
        self.calls = {k: 0 for k in self.calls}

    def profile_read(self):
        return {k: (n, 0.1 * n) for k, n in self.calls.items()}

    def download(self, out=None):
        return out

    def upload(self, links):
        pass

    def close(self):
        pass


class FakePinned:
    def __init__(self, shape, dtype=None):
        self.array = None

    def free(self):
        pass


S.Lattice, S.PinnedArray = FakeLattice, FakePinned
sys.argv = ["bench.py", "--gpus", "2", "--steps", "4", "--warmup", "3", "--no-extras", "--no-cpu", "--dims", "8,8,8,8"]
args = bench.parse()
d = bench.Dist()
bench.run_ours(args, d, [8, 8, 8, 8])
d.close()
'''


def test_repo_arm_rank_plumbing_under_two_ranks(tmp_path):
    """bench.py's own arm under torchrun with two gloo ranks, the lattice replaced by a host fake:
    rank 0 alone prints one line, timed as the maximum over ranks, with the whole-job aggregate."""
    script = tmp_path / "arm.py"
    script.write_text(f"REPO = {O.REPO!r}\n" + FAKE_ARM)
    r = _torchrun([str(script)])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    vol, K = 8 ** 4, 4
    # the slower rank (rank 1: 6 ms for the K steps) sets the job's time
    assert line["n_gpus"] == 2 and line["steps"] == K and line["warmup"] == 3
    assert line["ms_per_step"] == 6.0 / K
    assert abs(line["value"] - 4 * vol * K * 2 / 6e-3) <= 1e-6 * line["value"]
    assert abs(line["e2e"]["value"] - 4 * vol * K * 2 / 6e-3) <= 1e-6 * line["value"]
    assert line["scaling"] == "weak" and line["config"]["parallelism"] == "replicas x2"
    assert line["roofline"]["launches"] == 8 * K and line["gpu_launches"] == 9 * K
    assert "cpu_baseline" not in line   # rank 0 at N = 1 only
