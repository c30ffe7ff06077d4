"""Parity at 24^4, beta = 3.09 with the reference's own thesis chains, and the error of the FP32
path against FP64 on a thermalised 24^4 field.

Statistical parity.  The thesis ran the reference's heatbath (lexicographic order, RANLUX) at 24^4
and logged W(1,1), W(1,5), W(5,1), W(5,5) after every sweep, and W(10,16) after 100 spatial APE
steps (LGT_Code/modules/obs/smearing.c:107-138, wilson.c:268-324).  Their equilibrium means and
errors (t_int.c Gamma method or blocks of 100 sweeps, the larger; hot and cold starts combined)
are in tests/golden/golden.json["thesis_24x24x24x24_b3.09"] (tests/golden/make_golden.py
--thesis-only).  Two GPU chains from a Haar-random start are compared with them: FP32 1 heatbath +
4 overrelaxation sweeps, and the FP64 heatbath alone.  The ten comparisons (five loops, two chains)
form one family, tested at a family-wise false-alarm rate of 1e-3 by the Bonferroni bound:
|z| < z(1 - 1e-3 / 20) = 3.89 for each, z = (GPU - reference) / sqrt(err_GPU^2 + err_ref^2).  The
z values are printed (the north-star reading, "within 2 sigma combined", is reported beside it).

FP32 against FP64.  One thermalised FP64 field is uploaded into an FP32 and an FP64 handle, and the
observables of the thesis' measurement programs are computed in both: the plaquette; W(R <= 10,
T <= 16) after 100, 200 and 400 spatial APE steps (alpha 0.5); Q after 15 and 30 APE_all steps
(alpha 0.5).  Bounds, asserted:
  - plaquette: 1e-6 relative (well conditioned: a mean of 6V terms of one sign);
  - W(R, T): |dW| <= 1e-6 relative, or 1e-9 absolute for a loop whose mean falls below 1e-3 (a sum
    of site terms of both signs, each |w_x| <= 1);
  - Q: |dQ| <= 1e-6 * sum_x |q_x| / (32 pi^2) (Q sums site densities of both signs).
"""
import math
from statistics import NormalDist

import numpy as np
import pytest

import _stats
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu

DIMS = (24, 24, 24, 24)
BETA = 3.09
FWER = 1e-3


def _err(x, block):
    """max(t_int.c Gamma-method error, binned error)."""
    m, eg, tau = _stats.mean_err(x)
    nb = len(x) // block
    b = np.asarray(x[: nb * block]).reshape(nb, block).mean(axis=1)
    return m, max(eg, float(b.std(ddof=1) / math.sqrt(nb))), tau


def _chain(precision, n_or, therm, sweeps, smear_every, seed):
    """Haar start, `therm` sweeps, then `sweeps` sweeps with the unsmeared loops after every sweep
    and W(10,16) after 100 spatial APE steps (on a copy of the field) every `smear_every` sweeps."""
    L = Lattice(DIMS, precision=precision, beta=BETA, seed=seed, start="haar")
    L.sweep(therm, 1, n_or)
    R, T = [1, 1, 5, 5], [1, 5, 1, 5]
    unsm, sm = [], []
    for i in range(sweeps):
        L.sweep(1, 1, n_or)
        unsm.append(L.wilson(R, T))
        if (i + 1) % smear_every == 0:
            sm.append(L.measure(R=[10], T=[16], ns_s=100, alpha_s=0.5)[1][0])
    L.close()
    return np.array(unsm), np.array(sm)


def test_chains_agree_with_thesis_chains(golden):
    ref = golden["thesis_24x24x24x24_b3.09"]["sets"]
    chains = {
        "fp32 1HB+4OR": _chain("fp32", 4, 2000, 10000, 10, 24001),
        "fp64 HB": _chain("fp64", 0, 4000, 10000, 10, 24002),
    }
    rows = []
    for name, (unsm, sm) in chains.items():
        for j, o in enumerate(ref["unsmeared"]):
            m, e, tau = _err(unsm[:, j], 100)
            rows.append((name, f"W({o['R']},{o['T']})", m, e, tau, o["mean"], o["err"]))
        o = ref["ape_spatial_100"][0]
        m, e, tau = _err(sm, 20)
        rows.append((name, "W(10,16) after 100 spatial APE", m, e, tau, o["mean"], o["err"]))
    zc = NormalDist().inv_cdf(1.0 - FWER / (2 * len(rows)))
    zs = []
    for name, obs, m, e, tau, rm, re_ in rows:
        z = (m - rm) / math.hypot(e, re_)
        zs.append(z)
        print(f"{name:13s} {obs:31s} gpu {m:.7f} +- {e:.7f} (tau {tau:4.1f})  thesis {rm:.7f} +- {re_:.7f}  "
              f"z {z:+.2f}")
    print(f"family of {len(zs)}: max |z| = {max(map(abs, zs)):.2f}, bound {zc:.2f} (family-wise rate {FWER}); "
          f"{sum(abs(z) <= 2.0 for z in zs)} of {len(zs)} within 2 sigma")
    assert max(map(abs, zs)) < zc, zs


def _thermalised_field():
    L = Lattice(DIMS, precision="fp64", beta=BETA, seed=24100, start="haar")
    L.sweep(500, 1, 4)
    U = L.download()
    L.close()
    return U


def test_fp32_error_against_fp64_on_thermalised_field():
    U = _thermalised_field()
    h = {p: Lattice(DIMS, precision=p, beta=BETA) for p in ("fp32", "fp64")}
    for L in h.values():
        L.upload(U)
    p32, p64 = h["fp32"].plaquette(), h["fp64"].plaquette()
    rel = abs(p32 - p64) / abs(p64)
    print(f"plaquette: fp64 {p64:.12f}  relative error of fp32 {rel:.2e}")
    assert rel <= 1e-6
    R = [r for r in range(1, 11) for t in range(1, 17)]
    T = [t for r in range(1, 11) for t in range(1, 17)]
    for n in (100, 200, 400):
        w = {p: L.measure(R=R, T=T, ns_s=n, alpha_s=0.5)[1] for p, L in h.items()}
        d = np.abs(w["fp32"] - w["fp64"])
        rel = d / np.abs(w["fp64"])
        print(f"W after {n} spatial APE: max relative error {rel.max():.2e} over all {len(d)} loops "
              f"(smallest |W| {np.abs(w['fp64']).min():.1e}, W(10,16) {w['fp64'][-1]:.4e} to {rel[-1]:.1e}); "
              f"max |dW| {d.max():.2e}")
        # 1e-6 relative; for a loop whose mean falls below 1e-3 (a sum of site terms of both signs,
        # each |w_x| <= 1) the bound becomes 1e-9 absolute
        assert np.all(d <= 1e-6 * np.maximum(np.abs(w["fp64"]), 1e-3)), rel.max()
    q = {p: L.measure(q_ape=[15, 30], alpha_q=0.5)[0] for p, L in h.items()}
    # condition number of Q: sum_x |q_x| / (32 pi^2) on the FP64 field after the same smearing
    L64 = h["fp64"]
    sabs = []
    for n in (15, 30):
        L64.upload(U)
        L64.ape(n, 0.5, "all")
        sabs.append(L64.qtop(with_abs=True)[1])
    for i, n in enumerate((15, 30)):
        dq = abs(q["fp32"][i] - q["fp64"][i])
        print(f"Q after {n} APE_all: fp64 {q['fp64'][i]:+.9f}  |dQ| {dq:.2e}  = {dq / sabs[i]:.2e} of sum|q| "
              f"({sabs[i]:.3e}); relative {dq / max(abs(q['fp64'][i]), 1e-300):.2e}")
        assert dq <= 1e-6 * sabs[i]
    for L in h.values():
        L.close()
