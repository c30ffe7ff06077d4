"""Autocorrelation-corrected errors, the method of the reference's analysis tool
LGT_Code/Autocorrelation/t_int.c:32-74 (Gamma method, summation up to the first negative
Gamma(k), error = sqrt(2 tau_int) x naive error).  Test infrastructure only."""
import numpy as np


def autocorrelation(a, k):
    """Gamma(k) with separate means of the two windows (t_int.c:32-41)."""
    a = np.asarray(a, dtype=np.float64)
    n = len(a)
    x, y = a[: n - k], a[k:]
    return float(np.mean((x - x.mean()) * (y - y.mean())))


def tau_int(a):
    """Integrated autocorrelation time, summed until the first negative Gamma(k) (t_int.c:44-55)."""
    g0 = autocorrelation(a, 0)
    t = 0.5 * g0
    for k in range(1, len(a)):
        gk = autocorrelation(a, k)
        if gk < 0.0:
            break
        t += gk
    return t / g0


def mean_err(a):
    """(mean, error, tau_int) with error = sqrt(2 tau_int) * sqrt(Gamma(0)/(N-1)) (t_int.c:58-74)."""
    a = np.asarray(a, dtype=np.float64)
    t = tau_int(a)
    naive = np.sqrt(autocorrelation(a, 0) / (len(a) - 1))
    return float(a.mean()), float(np.sqrt(2.0 * t) * naive), float(t)
