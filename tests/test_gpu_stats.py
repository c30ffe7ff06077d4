"""The reference's analysis tools on the device (su2g_stats_tau_int, su2g_stats_veff,
su2g_batch_tau_int) against the oracle's restatements -- which equal the tools' own output
(tests/test_oracle_cpu.py) -- and against the tools' printed results directly."""
import numpy as np
import pytest

import _oracle as O
import _stats
from masterarbeit_b200.su2g import Batch, Su2gError, stats_tau_int, stats_veff

pytestmark = pytest.mark.gpu


def test_tau_int_equals_tool(golden):
    cols = []
    for g in golden["stats"]["t_int"]:
        x = _stats.ar1_series(g["seed"], g["phi"], g["n"])
        out, ok = stats_tau_int(x)
        ref, rok = O.tau_int(x)
        assert ok[0] == rok
        # the same sums in the same order: equal up to the last bit (sqrt and division are IEEE)
        assert np.array_equal(out[0], ref), (out[0], ref)
        assert abs(out[0, 0] - g["mean"]) <= 6e-7 and abs(2 * out[0, 1] - g["two_tau"]) <= 6e-7
        assert abs(out[0, 3] - g["err"]) <= 6e-7
        cols.append(x[:2000])
    # several series in one call, element-major layout
    X = np.stack(cols, axis=1)
    out, ok = stats_tau_int(X)
    for s in range(X.shape[1]):
        assert np.array_equal(out[s], O.tau_int(X[:, s])[0])


def test_veff_equals_tool(golden):
    g = golden["stats"]["veff"]
    w = _stats.veff_data()
    ve, er, v, verr = stats_veff(w, g["n_bins"], g["t_fit_start"], g["t_fit_end"])
    ove, oer, ov, overr = O.veff(w, g["n_bins"], g["t_fit_start"], g["t_fit_end"])
    # the device log may differ from the host's by an ulp; the jackknife errors are spreads of
    # samples that agree to ~1e-5, which magnifies that ulp by ~1e5
    for a, b, tol in ((ve, ove, 1e-12), (v, ov, 1e-12), (er, oer, 1e-9), (verr, overr, 1e-9)):
        assert np.allclose(a, b, rtol=tol, atol=0)
    for r, t, val in g["veff"]:
        assert abs(ve[r - 1, t - 1] - val) <= 6e-7 * abs(val) + 1e-12
    for r, val, sig in g["v"]:
        assert abs(v[r - 1] - val) <= 6e-7 * abs(val) and abs(verr[r - 1] - sig) <= 6e-7 * abs(sig)


def test_batch_trace_analysed_on_device():
    reps = [{"dims": (8, 8, 8, 8), "beta": 2.3 + 0.2 * i, "seed": 50 + i, "replica": i, "start": "cold"}
            for i in range(6)]
    B = Batch(reps, precision="fp64")
    trace, _ = B.run(600, 1, 1, 1)
    out, ok = B.tau_int(skip=100)
    for r in range(len(reps)):
        ref, rok = O.tau_int(trace[100:, r])
        assert np.array_equal(out[r], ref) and ok[r] == rok
    with pytest.raises(Su2gError):
        B.tau_int(skip=599)
    B.close()


def test_stats_reject_bad_arguments():
    with pytest.raises(Su2gError):
        stats_tau_int(np.ones(1))
    w = _stats.veff_data(n_conf=40, n_r=2, n_t=6)
    with pytest.raises(Su2gError):
        stats_veff(w, 20, [0, 0], [6, 5])   # fit range past the last V_eff index
    with pytest.raises(Su2gError):
        stats_veff(w, 41, [0, 0], [3, 3])   # more bins than configurations
