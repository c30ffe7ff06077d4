"""The native qcd driver (masterarbeit_b200/_lib/su2qcd, driver/su2qcd.cpp): the reference's qcd.c
flow on the GPU.  Its plaquette record equals the library's own graph loop for the same seed, its
configurations pass the reference's own readConfig check (the harness built from the reference's
sources), and the reflection start and the Metropolis / random-order updates run through it."""
import os
import re
import subprocess

import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(O.REPO, "masterarbeit_b200", "_lib", "su2qcd")
HARNESS = os.path.join(O.REPO, "oracle", "_ref", "8x8x8x8", "harness")
QCD_IN = """outFileId     1
outputDir     {odir}
start         {start}
beta          3.09
epsilon       0.5
nconf         30
ntherm        10
ndecorr       1
writeConfFreq 10
seed          1337
"""
BASE = "8x8x8x8_SU2_b3.090000_id1"


def _run(work, extra=(), start=0):
    os.makedirs(work, exist_ok=True)
    inp = os.path.join(work, "qcd.in")
    open(inp, "w").write(QCD_IN.format(odir=work, start=start))
    return subprocess.run([DRIVER, "-i", inp, "-d", "8x8x8x8"] + list(extra), cwd=work, capture_output=True,
                          text=True, timeout=600)


def test_su2qcd_log_configs_and_trace(tmp_path):
    if not os.path.exists(DRIVER):
        pytest.skip("su2qcd not built")
    work = str(tmp_path / "run")
    r = _run(work, ["--or", "2"])
    assert r.returncode == 0, r.stderr
    log = open(os.path.join(work, BASE + ".log")).read()
    assert log.startswith("*******************************\nLATTICE QCD CODE\n")
    plaq = re.findall(r"^plaq\t([0-9.]+)$", log, re.M)
    acc = [float(x) for x in re.findall(r"acc=([0-9.]+)\)", log)]
    assert len(plaq) == 30 and len(acc) == 30 and log.count("update took") == 30
    # the same chain through the library: 30 blocks of 1 heatbath + 2 overrelaxation sweeps
    L = Lattice((8, 8, 8, 8), precision="fp64", beta=3.09, seed=1337, start="cold")
    p, a = L.graph_run(30, 1, 1, 2)
    assert ["%.8f" % x for x in p] == plaq
    # configurations after sweeps 19 and 29 (qcd.c:64), accepted by the reference's readConfig
    cfgs = sorted(f for f in os.listdir(work) if re.fullmatch(BASE + r"_n\d+", f))
    assert cfgs == [BASE + "_n1", BASE + "_n2"]
    if os.path.exists(HARNESS):
        for c in cfgs:
            h = subprocess.run([HARNESS, "plaq", os.path.join(work, c)], capture_output=True, text=True, timeout=120)
            assert h.returncode == 0, h.stdout + h.stderr
    # no overwriting of an existing log (setupOutputFiles, inp_IO.c:158-165)
    r2 = _run(work)
    assert r2.returncode == 1 and "overwrite" in r2.stderr


def test_su2qcd_reflection_start_and_metropolis(tmp_path):
    if not os.path.exists(DRIVER):
        pytest.skip("su2qcd not built")
    small = os.path.join(O.GOLDEN, "cfg_4x4x4x4_base.cfg")
    r = _run(str(tmp_path / "t"), ["-t", small])
    assert r.returncode == 0, r.stderr
    log = open(os.path.join(str(tmp_path / "t"), BASE + ".log")).read()
    assert "Configuration imported for thermalisation" in log
    # the first sweep starts from the mirrored small lattice, whose plaquette is the file's
    _, p0, _ = O.golden_config("cfg_4x4x4x4_base.cfg")
    assert f"calc plaq {p0:.6e}" in r.stdout
    r = _run(str(tmp_path / "m"), ["--utype", "0", "--stype", "1"], start=1)
    assert r.returncode == 0, r.stderr
    log = open(os.path.join(str(tmp_path / "m"), BASE + ".log")).read()
    acc = [float(x) for x in re.findall(r"\(algorithm 0; sweep 1; acc=([0-9.]+)\)", log)]
    assert len(acc) == 30 and all(0.2 < a < 1.0 for a in acc)
