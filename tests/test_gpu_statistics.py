"""Statistical parity of the GPU chains with the reference's own chain.

The reference sweeps sites in lexicographic order with RANLUX randoms; the GPU sweeps by
checkerboard with Philox, and adds overrelaxation.  Bitwise agreement is impossible, so the
equilibrium averages are compared: <plaquette> and W(R,T) must agree within 2 sigma combined, the
errors corrected for autocorrelation with the reference's own method (LGT_Code/Autocorrelation/
t_int.c:32-74, tests/_stats.py).  The reference chain (8^4, beta = 3.09, cold start, 6000
heatbath sweeps, seed 1) is in tests/golden/golden.json.
"""
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


def _agree(name, gpu, ref_mean, ref_err):
    m, e, t = _stats.mean_err(gpu)
    sigma = float(np.hypot(e, ref_err))
    print(f"{name}: gpu {m:.6f} +- {e:.6f} (tau_int {t:.2f})  reference {ref_mean:.6f} +- {ref_err:.6f}  "
          f"-> {abs(m - ref_mean) / sigma:.2f} sigma")
    assert abs(m - ref_mean) <= 2.0 * sigma, name


@pytest.mark.parametrize("precision,n_or,seed", [("fp32", 4, 4242), ("fp64", 0, 777)])
def test_chain_agrees_with_reference_chain(golden, precision, n_or, seed):
    ref = golden["chain_8x8x8x8_b3.09"]
    R = [w["R"] for w in ref["wilson"]]
    T = [w["T"] for w in ref["wilson"]]
    therm = ref["therm"]
    plaq, wil = _chain(precision, n_or, 20000, seed, R, T)
    _agree(f"{precision} 1HB+{n_or}OR <P>", plaq[therm:], ref["plaquette"]["mean"], ref["plaquette"]["err"])
    for j, w in enumerate(ref["wilson"]):
        _agree(f"{precision} W({w['R']},{w['T']})", wil[therm // 10:, j], w["mean"], w["err"])
