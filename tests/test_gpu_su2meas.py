"""The native measurement driver (masterarbeit_b200/_lib/su2meas, driver/su2meas.cpp) against the
reference's own meas and qtop programs (built from its sources into oracle/_ref) on configurations
the reference wrote: the same WIL lines, QTOP lines equal to the reference's qtop and, for meas
(whose reference build logs QTOP inf, its PI is never set), to the oracle's charge."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu

REPO = O.REPO
DRIVER = os.path.join(REPO, "masterarbeit_b200", "_lib", "su2meas")
REFBIN = os.path.join(REPO, "oracle", "_ref", "8x8x8x8")
BASE = "8x8x8x8_SU2_b3.090000_id1"

MEAS_IN = """outFileId      1
odir           {odir}
beta           3.09
seed           1337
sconf          1
fconf          2
econf          1
mtopcharge     1
smear_tc       5 0.1
mwil           1 6
tLoopExtent    1 2 3 4 5 7
tSmear         2 0.5
rLoopExtent    1 2 3 4 1 6
rSmear         3 0.5
mcorrs         0
kappa          0.1588
source         0 0 0 0
stype          1
nmax           5000
prec           1.0e-08
n2pt           1
gammas         5 5
"""


def _need(*paths):
    for p in paths:
        if not os.path.exists(p):
            pytest.skip(f"{p} not built")


def _setup(work):
    os.makedirs(work, exist_ok=True)
    dims, _, U = O.golden_config("cfg_8x8x8x8_base.cfg")
    shutil.copyfile(os.path.join(O.GOLDEN, "cfg_8x8x8x8_base.cfg"), os.path.join(work, f"{BASE}_n1"))
    L = Lattice(dims, precision="fp64", beta=3.09, seed=3)
    L.upload(U)
    L.sweep(3, 1, 1)
    L.write_config(os.path.join(work, f"{BASE}_n2"))
    inp = os.path.join(work, "meas.in")
    open(inp, "w").write(MEAS_IN.format(odir=work))
    return inp


def _lines(path, key):
    return [line.rstrip("\n") for line in open(path) if line.startswith(key)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("fp32", 2e-5)])
def test_su2meas_matches_reference_meas(tmp_path, precision, tol):
    _need(DRIVER, os.path.join(REFBIN, "meas"))
    ref_dir, gpu_dir = str(tmp_path / "ref"), str(tmp_path / "gpu")
    for d in (ref_dir, gpu_dir):
        inp = _setup(d)
    subprocess.run([os.path.join(REFBIN, "meas"), "-i", os.path.join(ref_dir, "meas.in")], cwd=ref_dir, check=True,
                   capture_output=True, timeout=600)
    subprocess.run([DRIVER, "-i", inp, "-d", "8x8x8x8", "-p", precision], cwd=gpu_dir, check=True,
                   capture_output=True, timeout=600)
    ref_log, gpu_log = os.path.join(ref_dir, f"{BASE}.meas"), os.path.join(gpu_dir, f"{BASE}.meas")
    rw, gw = _lines(ref_log, "WIL"), _lines(gpu_log, "WIL")
    assert len(rw) == len(gw) == 12
    for a, b in zip(rw, gw):
        fa, fb = a.split(), b.split()
        assert fa[:3] == fb[:3] and re.fullmatch(r"WIL \d+ \d+\t-?\d\.\d{8}e[+-]\d\d", b)
        assert abs(float(fa[3]) - float(fb[3])) <= tol * abs(float(fa[3])) + 1e-15
    # the reference's meas logs QTOP inf (PI is never set); the driver's charge against the oracle
    assert all(re.fullmatch(r"QTOP -?inf", line) for line in _lines(ref_log, "QTOP"))
    gq = _lines(gpu_log, "QTOP")
    assert len(gq) == 2 and all(re.fullmatch(r"QTOP -?\d\.\d{8}e[+-]\d\d", x) for x in gq)
    dims = (8, 8, 8, 8)
    for n, line in zip((1, 2), gq):
        _, _, U = O.golden_config(os.path.join(gpu_dir, f"{BASE}_n{n}"))
        q, sabs = O.qtop(dims, O.ape(dims, U, 5, 0.1, "all"))
        assert abs(float(line.split()[1]) - q) <= (1e-8 if precision == "fp64" else tol) * sabs + 1e-8 * abs(q)
    # the same progress lines around the measurements
    text = open(gpu_log).read()
    assert text.count("\nMeasuring on configuration:\n") == 2 and text.count("\nMeasurement complete (took ") == 2


def test_su2meas_qtop_matches_reference_qtop(tmp_path):
    _need(DRIVER, os.path.join(REFBIN, "qtop"))
    out = {}
    for name, cmd in (("ref", [os.path.join(REFBIN, "qtop")]), ("gpu", [DRIVER, "-d", "8x8x8x8", "--qtop"])):
        work = str(tmp_path / name)
        os.makedirs(work)
        shutil.copyfile(os.path.join(O.GOLDEN, "cfg_8x8x8x8_base.cfg"),
                        os.path.join(work, "8x8x8x8_SU2_b2.300000_id1_n1"))
        subprocess.run(cmd + [work], cwd=work, check=True, capture_output=True, timeout=600)
        out[name] = _lines(os.path.join(work, "8x8x8x8_SU2_b2.300000_id1.meas"), "QTOP")
    assert len(out["ref"]) == len(out["gpu"]) == 21
    dims, _, U = O.golden_config("cfg_8x8x8x8_base.cfg")
    W = U.copy()
    for k, (a, b) in enumerate(zip(out["ref"], out["gpu"])):
        fa, fb = a.split(), b.split()
        assert fa[:4] == fb[:4]   # configuration, APE steps, alpha (%e)
        if k:
            W = O.ape(dims, W, 1, 0.1, "all")
        sabs = O.qtop(dims, W)[1]
        assert abs(float(fa[4]) - float(fb[4])) <= 2e-8 * sabs + 1e-8 * abs(float(fa[4]))
