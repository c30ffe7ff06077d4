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


# Synthetic inputs of the statistics fixtures (tests/golden/make_golden.py, golden.json["stats"]).
AR1_SERIES = [(101, 0.9, 5000), (202, 0.3, 2000)]   # (seed, phi, length)


def ar1_series(seed, phi, n):
    """x_i = phi x_{i-1} + N(0,1), x_0 = 0."""
    g = np.random.default_rng(seed).standard_normal(n)
    x = np.zeros(n)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + g[i]
    return x


def veff_data(n_conf=1000, n_r=12, n_t=20, seed=303):
    """W(R, T) per configuration, [n_conf][n_r][n_t], rounded to the %.8e of the WIL lines:
    W = exp(-V(R) T - 0.1) (1 + 0.01 noise), V(R) = 0.1 + 0.05 R, noise ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    R = np.arange(1, n_r + 1)[:, None]
    T = np.arange(1, n_t + 1)[None, :]
    base = np.exp(-(0.1 + 0.05 * R) * T - 0.1)
    w = base[None] * (1.0 + 0.01 * rng.standard_normal((n_conf, n_r, n_t)))
    return np.array([float("%.8e" % v) for v in w.ravel()]).reshape(w.shape)


def veff_meas_text(w):
    """The WIL lines of meas.c (meas.c:113) for every configuration."""
    n_conf, n_r, n_t = w.shape
    lines = []
    for c in range(n_conf):
        for r in range(n_r):
            for t in range(n_t):
                lines.append("WIL %d %d\t%.8e\n" % (r + 1, t + 1, w[c, r, t]))
    return "".join(lines)
