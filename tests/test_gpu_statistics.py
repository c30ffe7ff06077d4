"""Statistical parity of the GPU chains with the reference's own chain.

The reference sweeps sites in lexicographic order with RANLUX randoms; the GPU sweeps by
checkerboard with Philox, and adds overrelaxation.  Bitwise agreement is impossible, so the
equilibrium averages are compared, the errors corrected for autocorrelation with the reference's
own method (LGT_Code/Autocorrelation/t_int.c:32-74, tests/_stats.py).  The reference chain (8^4,
beta = 3.09, cold start, 6000 heatbath sweeps, seed 1) is in tests/golden/golden.json.

The twelve comparisons (<plaquette> and five W(R,T), for the FP32 1HB+4OR and the FP64 heatbath
chain) are one family tested at a family-wise false-alarm rate of 1e-3 (Bonferroni: every
|z| < z(1 - 1e-3/24) = 3.54, z = (GPU - reference) / sqrt(err_GPU^2 + err_ref^2)).  Held to
2 sigma one by one, six observables fail a correct chain in about one trajectory in five; the
z values and how many lie within 2 sigma are printed.
"""
from statistics import NormalDist

import numpy as np
import pytest

import _stats
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu


def _chain(precision, n_or, sweeps, seed, R, T, every=10):
    L = Lattice((8, 8, 8, 8), precision=precision, beta=3.09, seed=seed, start="cold")
    plaq, wil = [], []
    for i in range(sweeps):
        L.sweep(1, 1, n_or)
        plaq.append(L.plaquette())
        if (i + 1) % every == 0:
            wil.append(L.wilson(R, T))
    L.close()
    return np.array(plaq), np.array(wil)


FWER = 1e-3


def _z(name, gpu, ref_mean, ref_err):
    m, e, t = _stats.mean_err(gpu)
    z = (m - ref_mean) / float(np.hypot(e, ref_err))
    print(f"{name}: gpu {m:.6f} +- {e:.6f} (tau_int {t:.2f})  reference {ref_mean:.6f} +- {ref_err:.6f}  "
          f"-> z {z:+.2f}")
    return z


def test_chains_agree_with_reference_chain(golden):
    ref = golden["chain_8x8x8x8_b3.09"]
    R = [w["R"] for w in ref["wilson"]]
    T = [w["T"] for w in ref["wilson"]]
    therm = ref["therm"]
    zs = []
    for precision, n_or, seed in (("fp32", 4, 4242), ("fp64", 0, 777)):
        plaq, wil = _chain(precision, n_or, 20000, seed, R, T)
        zs.append(_z(f"{precision} 1HB+{n_or}OR <P>", plaq[therm:], ref["plaquette"]["mean"], ref["plaquette"]["err"]))
        for j, w in enumerate(ref["wilson"]):
            zs.append(_z(f"{precision} W({w['R']},{w['T']})", wil[therm // 10:, j], w["mean"], w["err"]))
    zc = NormalDist().inv_cdf(1.0 - FWER / (2 * len(zs)))
    print(f"family of {len(zs)}: max |z| = {max(map(abs, zs)):.2f}, bound {zc:.2f} (family-wise rate {FWER}); "
          f"{sum(abs(z) <= 2.0 for z in zs)} of {len(zs)} within 2 sigma")
    assert max(map(abs, zs)) < zc, zs
