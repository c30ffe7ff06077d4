"""The reference's own drivers linked against libsu2g through masterarbeit_b200/shim/ref_shim.c.

masterarbeit_b200/shim/build_dropin.sh links LGT_Code/main/qcd.c, main_meas/meas.c and
main_qtop/qtop.c, unmodified, against the shim.  oracle/build_ref.sh builds the same drivers with
the reference's own modules as the checker.  Both are built from the reference tree where it is
present and travel with the repository as binaries; tests skip when they are absent.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import _oracle as O

REPO = O.REPO
DIMS = "8x8x8x8"
DROPIN = os.path.join(REPO, "masterarbeit_b200", "shim", "_build", DIMS)
REFBIN = os.path.join(REPO, "oracle", "_ref", DIMS)


def _need(*paths):
    for p in paths:
        if not os.path.exists(p):
            pytest.skip(f"{p} not built (needs the reference tree)")


def test_dropin_links_the_shim():
    """The drop-in drivers take the hot-path symbols from the shim and the library, nothing from the
    reference's update/obs modules."""
    _need(os.path.join(DROPIN, "qcd"), os.path.join(DROPIN, "obj", "ref_shim.o"))
    syms = subprocess.run(["nm", os.path.join(DROPIN, "qcd")], capture_output=True, text=True).stdout
    assert re.search(r" T gaugefieldUpdate$", syms, re.M)
    assert re.search(r" T plaquette$", syms, re.M)
    assert re.search(r" U su2g_sweep_plaquette$", syms, re.M)
    assert not re.search(r" T localHeatbathUpdate$", syms, re.M)
    assert re.search(r" T ref_readConfig$", syms, re.M)
    dyn = subprocess.run(["ldd", os.path.join(DROPIN, "qcd")], capture_output=True, text=True).stdout
    assert "libsu2g.so" in dyn and "not found" not in dyn.split("libsu2g.so", 1)[1].splitlines()[0]


def _qtop_lines(path):
    out = []
    for line in open(path):
        if line.startswith("QTOP"):
            f = line.split()
            out.append((int(f[1]), int(f[2]), float(f[3]), float(f[4])))
    return out


def _run_qtop(binary, workdir, cfg, env=None):
    os.makedirs(workdir, exist_ok=True)
    shutil.copyfile(cfg, os.path.join(workdir, f"{DIMS}_SU2_b2.300000_id1_n1"))
    subprocess.run([binary, workdir], cwd=workdir, check=True, capture_output=True, env=env, timeout=600)
    return _qtop_lines(os.path.join(workdir, f"{DIMS}_SU2_b2.300000_id1.meas"))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 2e-8), ("fp32", 2e-5)])
def test_dropin_qtop_matches_reference_qtop(tmp_path, precision, tol):
    """main_qtop/qtop.c: Q after 0..20 APE_all steps (alpha 0.1) on a configuration written by the
    reference, with the reference's modules and with the shim.  Q is logged as %+.8e."""
    _need(os.path.join(DROPIN, "qtop"), os.path.join(REFBIN, "qtop"))
    cfg = os.path.join(O.GOLDEN, "cfg_8x8x8x8_base.cfg")
    ref = _run_qtop(os.path.join(REFBIN, "qtop"), str(tmp_path / "ref"), cfg)
    env = dict(os.environ, SU2G_PRECISION=precision)
    gpu = _run_qtop(os.path.join(DROPIN, "qtop"), str(tmp_path / "gpu"), cfg, env)
    assert len(ref) == len(gpu) == 21
    # |dQ| against the scale sum_x |q(x)| of each measurement (the oracle gives it)
    dims, _, U = O.golden_config("cfg_8x8x8x8_base.cfg")
    W = U.copy()
    for (c1, n1, a1, q1), (c2, n2, a2, q2) in zip(ref, gpu):
        assert (c1, n1, a1) == (c2, n2, a2)
        if n1 > 0:
            W = O.ape(dims, W, 1, 0.1, "all")
        sabs = O.qtop(dims, W)[1]
        assert abs(q1 - q2) <= tol * sabs + 1e-8 * abs(q1), (n1, q1, q2, sabs)


MEAS_IN = """outFileId      1
odir           {odir}
beta           3.09
seed           1337
sconf          1
fconf          1
econf          1
mtopcharge     0
smear_tc       0 0.3
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


def _run_meas(binary, workdir, cfg, env=None):
    os.makedirs(workdir, exist_ok=True)
    shutil.copyfile(cfg, os.path.join(workdir, f"{DIMS}_SU2_b3.090000_id1_n1"))
    inp = os.path.join(workdir, "meas.in")
    open(inp, "w").write(MEAS_IN.format(odir=workdir))
    subprocess.run([binary, "-i", inp], cwd=workdir, check=True, capture_output=True, env=env, timeout=600)
    w = {}
    for line in open(os.path.join(workdir, f"{DIMS}_SU2_b3.090000_id1.meas")):
        if line.startswith("WIL"):
            f = line.split()
            w[(int(f[1]), int(f[2]))] = float(f[3])
    return w


@pytest.mark.gpu
def test_dropin_meas_matches_reference_meas(tmp_path):
    """main_meas/meas.c: temporal + spatial APE then W(R,T) for an explicit pair list, reference
    modules against the shim (FP64); WIL lines are logged as %.8e."""
    _need(os.path.join(DROPIN, "meas"), os.path.join(REFBIN, "meas"))
    cfg = os.path.join(O.GOLDEN, "cfg_8x8x8x8_base.cfg")
    ref = _run_meas(os.path.join(REFBIN, "meas"), str(tmp_path / "ref"), cfg)
    gpu = _run_meas(os.path.join(DROPIN, "meas"), str(tmp_path / "gpu"), cfg,
                    dict(os.environ, SU2G_PRECISION="fp64"))
    assert set(ref) == set(gpu) and len(ref) == 6
    for k in ref:
        assert abs(ref[k] - gpu[k]) <= 1e-8 * abs(ref[k]) + 1e-15, (k, ref[k], gpu[k])


QCD_IN = """outFileId     1
outputDir     {odir}
start         0
beta          3.09
epsilon       0.15
nconf         30
ntherm        10
ndecorr       1
writeConfFreq 10
seed          1337
"""


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_dropin_qcd_runs_and_writes_reference_readable_configs(tmp_path, precision):
    """main/qcd.c on the GPU: 30 heatbath sweeps from a cold start; the log keeps the reference's
    lines, the plaquette thermalises to the beta=3.09 value, and the configurations it writes pass
    the reference's own readConfig plaquette check (config_IO.c:611-614)."""
    _need(os.path.join(DROPIN, "qcd"), os.path.join(REFBIN, "harness"))
    work = str(tmp_path)
    inp = os.path.join(work, "qcd.in")
    open(inp, "w").write(QCD_IN.format(odir=work))
    env = dict(os.environ, SU2G_PRECISION=precision, SU2G_OR="2")
    subprocess.run([os.path.join(DROPIN, "qcd"), "-i", inp], cwd=work, check=True, capture_output=True, env=env,
                   timeout=600)
    log = open(os.path.join(work, f"{DIMS}_SU2_b3.090000_id1.log")).read()
    plaq = [float(x) for x in re.findall(r"^plaq\t([0-9.]+)$", log, re.M)]
    acc = [float(x) for x in re.findall(r"acc=([0-9.]+)\)", log)]
    assert len(plaq) == 30 and len(acc) == 30
    assert log.count("update took") == 30
    assert 0.97 < min(acc) <= max(acc) <= 1.0
    assert 0.70 < np.mean(plaq[10:]) < 0.76
    cfgs = sorted(p for p in os.listdir(work) if "_n" in p and not p.endswith((".log", ".out", ".in")))
    assert len(cfgs) == 2, cfgs
    for c in cfgs:
        # the reference's readConfig aborts if the stored plaquette does not match its own
        r = subprocess.run([os.path.join(REFBIN, "harness"), "plaq", os.path.join(work, c)], capture_output=True,
                           text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
