#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ from the reference's own C code.

This script is the provenance of every file next to it.  It needs the reference
tree ($SU2_REFERENCE_ROOT, else a `reference` directory beside the repository) and gcc; it
compiles the reference from its sources with oracle/build_ref.sh and runs the
resulting harness binaries (oracle/ref_harness.c).  The GPU box has no
reference tree, which is why the outputs are committed.

Outputs
  cfg_*.cfg      configurations in the reference's binary format
                 (LGT_Code/modules/io/config_IO.c:40-117): written by the
                 reference's writeConfig after its own heatbath chain, APE
                 smearing or Philox-injected heatbath sweeps.
  golden.json    observables computed by the reference's own routines
                 (%.17g): plaquette, APE, W(R,T), Q, injected-heatbath
                 acceptance and plaquette.
  golden.json["reflect"]  readConfigForThermalisation of the 4x4x4x4 and 6x4x4x8 base
                 configurations into lattices of twice the extents, run by the reference
                 and written by its writeConfig: sha256 of the link payload (the bytes after
                 the 32-byte header), the header plaquette and the computed one.  Run
                 `make_golden.py --reflect-only` to refresh this part alone.
  golden.json["metropolis"]  the reference's localMetropolisUpdate (metro.c:78-109) on Philox
                 uniforms in checkerboard order (cfg_*_metroinj.cfg, acceptance, plaquette), and
                 the reference's own RANLUX chains at 8^4, beta 3.09 for Metropolis with
                 sequential and random site order and for heatbath with random order
                 (gaugefieldUpdate utype/stype, update.c:102-175): plaquette mean, error, tau_int.
                 `make_golden.py --metro-only` refreshes this part alone.
  golden.json["stats"]  outputs of the reference's analysis tools on synthetic data that
                 tests/_stats.py regenerates from the recorded seeds:
                 LGT_Code/Autocorrelation/t_int.c (compiled by oracle/build_ref.sh) on two
                 AR(1) series, and Analysis/static potential/static_potential.py (run here,
                 its plotting module replaced by a no-op stand-in, matplotlib being absent) on
                 1000 configurations of W(R<=12, T<=20).  `make_golden.py --stats-only`.
  golden.json["thesis_24x24x24x24_b3.09"]  equilibrium averages of the reference's own thesis
                 chains at 24^4, beta 3.09 (one configuration per heatbath sweep, hot and cold
                 starts), read from the WIL lines of its logs:
                 measurements/Therm/24x24x24x24_SU2_b3.090000_id1_{hot,cold}_1.meas (unsmeared
                 W(1,1), W(1,5), W(5,1), W(5,5); 4999 sweeps) and
                 Thermalisation/24x24x24x24_SU2_b3.090000_id1_{hot,cold}_NAPE_100.meas (W(10,16)
                 after 100 spatial APE steps; 10000 sweeps).  Per chain: the sweeps before
                 `cut` dropped, the mean, the t_int.c Gamma-method error (tests/_stats.py) and a
                 binned error (blocks of 100 sweeps); the test uses the larger.  The two starts
                 are combined by inverse-variance weights, the error scaled by sqrt(chi^2/dof)
                 where they disagree.  `make_golden.py --thesis-only`.
  kp_improved.dat  the reference's Kennedy-Pendleton sampler histogram at
                 alpha=7 (copied from LGT_Code/main_test/improved.dat; 200 bins
                 of N=1e8 draws; column 2 is count*200/N).
"""
import hashlib
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("SU2_REFERENCE_ROOT") or os.path.join(os.path.dirname(REPO), "reference")

LATTICES = {
    # dims T,X,Y,Z : (start, seed, beta, sweeps)
    "4x4x4x4": (1, 3, 2.3, 5),
    "6x4x4x8": (1, 5, 3.09, 10),
    "8x8x8x8": (0, 1, 3.09, 50),
}
LINK_LEVEL = {"4x4x4x4", "6x4x4x8"}  # small enough to commit smeared / updated fields


def harness(dims, inj=False):
    return os.path.join(REPO, "oracle", "_ref", dims, "harness_inj" if inj else "harness")


def run(cmd):
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    res = []
    for line in out.splitlines():
        if line.startswith("RESULT "):
            res.append(line.split()[2:])
    return res


REFLECT = {"4x4x4x4": "8x8x8x8", "6x4x4x8": "12x8x8x16"}   # small base -> full lattice


def reflect_golden(gold):
    subprocess.run([os.path.join(REPO, "oracle", "build_ref.sh"), REF] + sorted(set(REFLECT.values())), check=True)
    out = {}
    for small, big in REFLECT.items():
        path = os.path.join("/tmp", f"reflect_{small}_to_{big}.cfg")
        rr = run([harness(big), "reflect", os.path.join(HERE, f"cfg_{small}_base.cfg"), path])
        with open(path, "rb") as f:
            data = f.read()
        out[big] = {"small": f"cfg_{small}_base.cfg", "plaq": float(rr[0][0]),
                    "payload_sha256": hashlib.sha256(data[32:]).hexdigest(), "bytes": len(data)}
    gold["reflect"] = out


METRO_INJ = {"seed": 777, "beta": 3.09, "eps": 0.5, "sweep0": 3, "sweeps": 2}
METRO_CHAINS = [(0, 0), (0, 1), (1, 1)]   # (utype, stype)
METRO_CHAIN = {"dims": [8, 8, 8, 8], "beta": 3.09, "eps": 0.5, "start": 0, "seed": 11, "sweeps": 6000, "therm": 500}


def metro_golden(gold):
    sys.path.insert(0, os.path.dirname(HERE))
    import _stats
    out = {"inj": {}, "chains": []}
    e = METRO_INJ
    for dims in sorted(LINK_LEVEL):
        cfg = f"cfg_{dims}_metroinj.cfg"
        rr = run([harness(dims, True), "metroinj", os.path.join(HERE, f"cfg_{dims}_base.cfg"), str(e["seed"]),
                  str(e["beta"]), str(e["eps"]), str(e["sweep0"]), str(e["sweeps"]), os.path.join(HERE, cfg)])
        out["inj"][dims] = dict(e, cfg=cfg, acc=[float(x[1]) for x in rr], plaq=[float(x[2]) for x in rr])
    c = METRO_CHAIN
    for utype, stype in METRO_CHAINS:
        rr = run([harness("8x8x8x8"), "genm", str(c["start"]), str(c["seed"]), str(c["beta"]), str(c["eps"]),
                  str(utype), str(stype), str(c["sweeps"])])
        plaq = [float(x[1]) for x in rr]
        m, err, tau = _stats.mean_err(plaq[c["therm"]:])
        out["chains"].append(dict(c, utype=utype, stype=stype, mean=m, err=err, tau_int=tau))
    out["chain_note"] = ("reference gaugefieldUpdate with RANLUX; plaquette after every sweep; "
                         "the first `therm` sweeps discarded; errors by the t_int.c Gamma method")
    gold["metropolis"] = out


class _NoPlot:
    """Stand-in for matplotlib: every attribute, call and index returns the stand-in."""

    def __getattr__(self, name):
        return self

    def __call__(self, *a, **k):
        return self

    def __getitem__(self, i):
        return self

    def __iter__(self):
        return iter((self, self))


def stats_golden(gold):
    import contextlib
    import io
    import runpy
    import tempfile
    import types

    sys.path.insert(0, os.path.dirname(HERE))
    import _stats
    out = {"t_int": [], "veff": {}}
    for seed, phi, n in _stats.AR1_SERIES:
        x = _stats.ar1_series(seed, phi, n)
        with tempfile.TemporaryDirectory() as d:
            f = os.path.join(d, "series.txt")
            np.savetxt(f, x, fmt="%.17g")
            txt = subprocess.run([os.path.join(REPO, "oracle", "_ref", "t_int"), f], check=True, capture_output=True,
                                 text=True).stdout
        m = txt.split("\n")[1].split()
        out["t_int"].append({"seed": seed, "phi": phi, "n": n, "sha256": hashlib.sha256(x.tobytes()).hexdigest(),
                             "mean": float(m[0]), "err": float(m[2]), "two_tau": float(m[6])})
    w = _stats.veff_data()
    script = os.path.join(REF, "Analysis", "static potential", "static_potential.py")
    stub = types.ModuleType("matplotlib")
    stub.pyplot = _NoPlot()
    saved = {k: sys.modules.get(k) for k in ("matplotlib", "matplotlib.pyplot")}
    sys.modules["matplotlib"], sys.modules["matplotlib.pyplot"] = stub, stub.pyplot
    cwd = os.getcwd()
    try:
        with tempfile.TemporaryDirectory() as d:
            with open(os.path.join(d, "24x24x24x24_SU2_b3.09_NAPE_400.meas"), "w") as f:
                f.write(_stats.veff_meas_text(w))
            os.chdir(d)
            buf = io.StringIO()
            with contextlib.redirect_stdout(buf):
                runpy.run_path(script, run_name="__main__")
    finally:
        os.chdir(cwd)
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    veff, vr = [], []
    for line in buf.getvalue().splitlines():
        f = line.split("\t")
        if len(f) == 3:
            veff.append([int(f[0]), int(f[1]), float(f[2])])
        elif len(f) == 4:
            vr.append([int(f[0]), float(f[2]), float(f[3])])
    out["veff"] = {"sha256": hashlib.sha256(w.tobytes()).hexdigest(), "veff": veff, "v": vr,
                   "n_bins": 20, "t_fit_start": [7] * 9 + [8] * 3, "t_fit_end": [17] * 12}
    gold["stats"] = out


# The thesis chains: which log, which loops, and where each start is thermalised.  The hot start's
# W(5,5) and smeared W(10,16) still drift for thousands of sweeps (1000-sweep window means), so
# the cuts are set where the window means of both starts have levelled off.
THESIS = {
    "unsmeared": {"file": "measurements/Therm/24x24x24x24_SU2_b3.090000_id1_%s_1.meas",
                  "loops": [(1, 1), (1, 5), (5, 1), (5, 5)], "cut": {"hot": 2500, "cold": 2500}},
    "ape_spatial_100": {"file": "Thermalisation/24x24x24x24_SU2_b3.090000_id1_%s_NAPE_100.meas",
                        "loops": [(10, 16)], "cut": {"hot": 4000, "cold": 2500}},
}
THESIS_BLOCK = 100


def _wil_lines(path):
    """Per configuration, {(R, T): W} from the WIL lines of a meas log (meas.c:113)."""
    import re
    confs = []
    for block in open(path).read().split("Measuring on configuration:")[1:]:
        confs.append({(int(m.group(1)), int(m.group(2))): float(m.group(3))
                      for m in re.finditer(r"WIL (\d+) (\d+)\s+(\S+)", block)})
    return confs


def binned_err(x, block):
    x = np.asarray(x, dtype=np.float64)
    nb = len(x) // block
    m = x[: nb * block].reshape(nb, block).mean(axis=1)
    return float(m.std(ddof=1) / np.sqrt(nb))


def thesis_golden(gold):
    sys.path.insert(0, os.path.dirname(HERE))
    import _stats
    out = {"dims": [24, 24, 24, 24], "beta": 3.09, "block": THESIS_BLOCK,
           "note": "reference thesis chains, one configuration per heatbath sweep; error = max(Gamma method "
                   "of t_int.c, binned); hot and cold starts combined by inverse-variance weights, the error scaled by "
                   "sqrt(chi^2/dof) where they disagree",
           "sets": {}}
    for name, spec in THESIS.items():
        obs = {}
        for start in ("hot", "cold"):
            rel = spec["file"] % start
            confs = _wil_lines(os.path.join(REF, rel))
            cut = spec["cut"][start]
            for R, T in spec["loops"]:
                x = np.array([c[(R, T)] for c in confs])[cut:]
                m, eg, tau = _stats.mean_err(x)
                eb = binned_err(x, THESIS_BLOCK)
                obs.setdefault(f"{R},{T}", {"R": R, "T": T, "chains": {}})["chains"][start] = {
                    "file": rel, "configurations": len(confs), "cut": cut, "mean": m, "err_gamma": eg,
                    "tau_int": tau, "err_binned": eb, "err": max(eg, eb)}
        for o in obs.values():
            w = {k: 1.0 / c["err"] ** 2 for k, c in o["chains"].items()}
            o["mean"] = sum(w[k] * c["mean"] for k, c in o["chains"].items()) / sum(w.values())
            # where the two starts disagree by more than their errors, the error of the combination is
            # scaled by sqrt(chi^2 / dof) (the scale factor of the Particle Data Group's averages)
            chi2 = sum(w[k] * (c["mean"] - o["mean"]) ** 2 for k, c in o["chains"].items())
            o["scale"] = float(max(1.0, np.sqrt(chi2 / (len(w) - 1))))
            o["err"] = float(o["scale"] / np.sqrt(sum(w.values())))
        out["sets"][name] = list(obs.values())
    gold["thesis_24x24x24x24_b3.09"] = out


def main():
    if "--stats-only" in sys.argv:
        path = os.path.join(HERE, "golden.json")
        with open(path) as f:
            gold = json.load(f)
        stats_golden(gold)
        with open(path, "w") as f:
            json.dump(gold, f, indent=1)
        print("updated", path)
        return 0
    if "--thesis-only" in sys.argv:
        path = os.path.join(HERE, "golden.json")
        with open(path) as f:
            gold = json.load(f)
        thesis_golden(gold)
        with open(path, "w") as f:
            json.dump(gold, f, indent=1)
        print("updated", path)
        return 0
    if "--metro-only" in sys.argv:
        path = os.path.join(HERE, "golden.json")
        with open(path) as f:
            gold = json.load(f)
        metro_golden(gold)
        with open(path, "w") as f:
            json.dump(gold, f, indent=1)
        print("updated", path)
        return 0
    if "--reflect-only" in sys.argv:
        path = os.path.join(HERE, "golden.json")
        with open(path) as f:
            gold = json.load(f)
        reflect_golden(gold)
        with open(path, "w") as f:
            json.dump(gold, f, indent=1)
        print("updated", path)
        return 0
    subprocess.run([os.path.join(REPO, "oracle", "build_ref.sh"), REF] + list(LATTICES), check=True)
    gold = {"reference": "daggerfall247/Masterarbeit LGT_Code, compiled by oracle/build_ref.sh", "lattices": {}}
    for dims, (start, seed, beta, nsw) in LATTICES.items():
        d = [int(x) for x in dims.split("x")]
        base = f"cfg_{dims}_base.cfg"
        r = run([harness(dims), "gen", str(start), str(seed), str(beta), str(nsw), os.path.join(HERE, base)])
        entry = {
            "dims": d,
            "base": base,
            "gen": {"start": start, "seed": seed, "beta": beta, "sweeps": nsw,
                    "plaq_trace": [float(x[1]) for x in r]},
        }
        entry["plaq"] = float(run([harness(dims), "plaq", os.path.join(HERE, base)])[0][0])

        # APE smearing, three modes (smearing.c:74-168)
        entry["ape"] = {}
        for mode in ("all", "spatial", "temporal"):
            ns, alpha = 3, 0.5
            out = os.path.join(HERE if dims in LINK_LEVEL else "/tmp", f"cfg_{dims}_ape_{mode}.cfg")
            rr = run([harness(dims), "ape", os.path.join(HERE, base), mode, str(ns), str(alpha), out])
            e = {"ns": ns, "alpha": alpha, "plaq": float(rr[0][0])}
            if dims in LINK_LEVEL:
                e["cfg"] = os.path.basename(out)
            entry["ape"][mode] = e

        # Wilson loops, explicit list mode (wilson.c:268-324)
        lt = d[0]
        R = [r_ for r_ in range(1, 7) for t_ in range(1, lt)]
        T = [t_ for r_ in range(1, 7) for t_ in range(1, lt)]
        rr = run([harness(dims), "wil", os.path.join(HERE, base), ",".join(map(str, R)), ",".join(map(str, T))])
        entry["wilson"] = [[int(x[0]), int(x[1]), float(x[2])] for x in rr]

        # Topological charge after cumulative APE_all steps (qtop.c:76-91)
        for alpha, Ns in ((0.1, [0, 1, 5]), (0.5, [0, 3])):
            rr = run([harness(dims), "qtop", os.path.join(HERE, base), str(alpha), ",".join(map(str, Ns))])
            entry.setdefault("qtop", []).append({"alpha": alpha, "N": Ns, "Q": [float(x[1]) for x in rr]})

        # Reference heatbath on injected Philox uniforms, checkerboard order
        hb_seed, hb_beta, sweep0, nhb = 12345, 3.09, 7, 2
        out = os.path.join(HERE if dims in LINK_LEVEL else "/tmp", f"cfg_{dims}_hbinj.cfg")
        rr = run([harness(dims, True), "hbinj", os.path.join(HERE, base), str(hb_seed), str(hb_beta), str(sweep0),
                  str(nhb), out])
        e = {"seed": hb_seed, "beta": hb_beta, "sweep0": sweep0, "sweeps": nhb,
             "acc": [float(x[1]) for x in rr], "plaq": [float(x[2]) for x in rr]}
        if dims in LINK_LEVEL:
            e["cfg"] = os.path.basename(out)
        entry["hbinj"] = e

        # Hot start of initGaugeField on injected Philox uniforms
        if dims in LINK_LEVEL:
            out = os.path.join(HERE, f"cfg_{dims}_hotinj.cfg")
            rr = run([harness(dims, True), "hotinj", "99", out])
            entry["hotinj"] = {"seed": 99, "plaq": float(rr[0][0]), "cfg": os.path.basename(out)}
        gold["lattices"][dims] = entry

    # The reference's own heatbath chain (RANLUX) for the statistical comparison: qcd.c's loop at
    # 8^4, beta = 3.09, cold start, plaquette every sweep, W(R,T) every 10 sweeps; the first
    # THERM sweeps are discarded; errors by the t_int.c Gamma method (tests/_stats.py).
    sys.path.insert(0, os.path.dirname(HERE))
    import _stats
    nsw, every, therm = 6000, 10, 500
    R, T = [1, 2, 1, 2, 3], [1, 2, 2, 1, 3]
    out = subprocess.run([harness("8x8x8x8"), "genw", "0", "1", "3.09", str(nsw), str(every), ",".join(map(str, R)),
                          ",".join(map(str, T))], check=True, capture_output=True, text=True).stdout
    plaq, wil = [], {}
    for line in out.splitlines():
        f = line.split()
        if line.startswith("RESULT plaq"):
            plaq.append((int(f[2]), float(f[3])))
        elif line.startswith("RESULT wil"):
            wil.setdefault((int(f[3]), int(f[4])), []).append((int(f[2]), float(f[5])))
    chain = {"dims": [8, 8, 8, 8], "beta": 3.09, "start": "cold", "seed": 1, "sweeps": nsw, "therm": therm,
             "sweep": "reference heatbath (lexicographic Gauss-Seidel), one sweep between plaquettes"}
    m, e, t = _stats.mean_err([p for n, p in plaq if n > therm])
    chain["plaquette"] = {"mean": m, "err": e, "tau_int": t}
    chain["wilson"] = []
    for (r_, t_), series in sorted(wil.items()):
        m, e, t = _stats.mean_err([w for n, w in series if n > therm])
        chain["wilson"].append({"R": r_, "T": t_, "every": every, "mean": m, "err": e, "tau_int": t})
    gold["chain_8x8x8x8_b3.09"] = chain

    reflect_golden(gold)
    metro_golden(gold)
    stats_golden(gold)
    thesis_golden(gold)
    shutil.copyfile(os.path.join(REF, "LGT_Code", "main_test", "improved.dat"), os.path.join(HERE, "kp_improved.dat"))
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(gold, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    sys.exit(main())
