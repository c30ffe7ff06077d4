"""ctypes access to the CPU oracle (oracle/su2_oracle.c) -- test infrastructure only.

The oracle is the checker: tests compare the CUDA library against it.  It is built with
`make -C oracle` into oracle/_build/libsu2oracle.so on first use.
"""
import ctypes
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "libsu2oracle.so")
GOLDEN = os.path.join(REPO, "tests", "golden")

_lib = None
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(ORACLE_DIR, "su2_oracle.c")
        if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        L = ctypes.CDLL(ORACLE_LIB)
        L.su2o_plaquette.argtypes = [_IP, _DP, _DP]
        L.su2o_ape.argtypes = [_IP, _DP, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.su2o_wilson.argtypes = [_IP, _DP, _IP, _IP, ctypes.c_int, _DP]
        L.su2o_qtop.argtypes = [_IP, _DP, _DP, _DP]
        L.su2o_ape_qtop.argtypes = [_IP, _DP, ctypes.c_int, ctypes.c_double, _DP]
        L.su2o_philox.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                  ctypes.POINTER(ctypes.c_uint32)]
        L.su2o_philox.restype = None
        L.su2o_start.argtypes = [_IP, _DP, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32]
        L.su2o_sweep.argtypes = [_IP, _DP, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32,
                                 ctypes.c_uint32, _DP]
        L.su2o_link_action.argtypes = [_IP, _DP, _DP]
        L.su2o_kp_samples.argtypes = [ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64, _DP]
        L.su2o_reflect.argtypes = [_IP, _DP, _DP]
        L.su2o_tau_int.argtypes = [_DP, ctypes.c_int64, ctypes.c_int64, _DP]
        L.su2o_veff.argtypes = [_DP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _IP, _IP, _DP, _DP, _DP,
                                _DP]
        L.su2o_visit_sweep.argtypes = [_IP, _DP, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32, _DP]
        _lib = L
    return _lib


def _dims(d):
    return (ctypes.c_int * 4)(*[int(x) for x in d])


def _dp(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def _ok(rc):
    if rc != 0:
        raise RuntimeError(f"oracle call failed with {rc}")


def plaquette(dims, U):
    v = ctypes.c_double()
    _ok(lib().su2o_plaquette(_dims(dims), _dp(U), ctypes.byref(v)))
    return v.value


def ape(dims, U, ns, alpha, mode):
    W = np.ascontiguousarray(U, dtype=np.float64).copy()
    m = {"all": 0, "spatial": 1, "temporal": 2}.get(mode, mode)
    _ok(lib().su2o_ape(_dims(dims), _dp(W), int(ns), float(alpha), int(m)))
    return W


def wilson(dims, U, R, T):
    R = np.ascontiguousarray(R, dtype=np.int32)
    T = np.ascontiguousarray(T, dtype=np.int32)
    w = np.empty(len(R))
    _ok(lib().su2o_wilson(_dims(dims), _dp(U), R.ctypes.data_as(_IP), T.ctypes.data_as(_IP), len(R), _dp(w)))
    return w


def qtop(dims, U):
    q, a = ctypes.c_double(), ctypes.c_double()
    _ok(lib().su2o_qtop(_dims(dims), _dp(U), ctypes.byref(q), ctypes.byref(a)))
    return q.value, a.value


def ape_qtop(dims, U, ns, alpha):
    q = ctypes.c_double()
    _ok(lib().su2o_ape_qtop(_dims(dims), _dp(np.ascontiguousarray(U)), int(ns), float(alpha), ctypes.byref(q)))
    return q.value


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().su2o_philox(c, k, o)
    return tuple(o)


def start(dims, mode, seed, replica=0):
    V = int(np.prod(dims))
    U = np.empty((V, 4, 4))
    m = {"cold": 0, "haar": 1, "ref": 2}.get(mode, mode)
    _ok(lib().su2o_start(_dims(dims), _dp(U), int(m), int(seed), int(replica)))
    return U


def sweep(dims, U, kind, beta=0.0, seed=0, sweep_index=0, replica=0):
    """In-place checkerboard sweep: kind 'hb' or 'or'. Returns mean 1/trials for 'hb'."""
    acc = ctypes.c_double()
    k = 0 if kind in ("hb", 0) else 1
    _ok(lib().su2o_sweep(_dims(dims), _dp(U), k, float(beta), int(seed), int(sweep_index), int(replica),
                         ctypes.byref(acc)))
    return acc.value


def link_action(dims, U):
    v = ctypes.c_double()
    _ok(lib().su2o_link_action(_dims(dims), _dp(U), ctypes.byref(v)))
    return v.value


def kp_samples(alpha, seed, n):
    x = np.empty(int(n))
    _ok(lib().su2o_kp_samples(float(alpha), int(seed), int(n), _dp(x)))
    return x


def reflect(dims, small):
    """readConfigForThermalisation's 16 mirror images: a field of extents dims from one of dims/2."""
    small = np.ascontiguousarray(small, dtype=np.float64)
    out = np.zeros((int(np.prod(dims)), 4, 4))
    _ok(lib().su2o_reflect(_dims(dims), _dp(small), _dp(out)))
    return out


def visit_sweep(dims, U, utype, stype, beta, eps, hits, seed, sweep_index, replica=0):
    """One gaugefieldUpdate sweep (utype 1 heatbath / 0 Metropolis, stype 0 / 1 random sites) in
    checkerboard order, in place on U; returns the mean acceptance per link visit."""
    assert U.dtype == np.float64 and U.flags["C_CONTIGUOUS"]
    a = ctypes.c_double()
    _ok(lib().su2o_visit_sweep(_dims(dims), _dp(U), int(utype), int(stype), float(beta), float(eps), int(hits),
                               int(seed), int(sweep_index), int(replica), ctypes.byref(a)))
    return a.value


def tau_int(x):
    """t_int.c on one series: ((mean, tau_int, naive error, error), resolved)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(4)
    ok = lib().su2o_tau_int(_dp(x), len(x), 1, _dp(out))
    return out, bool(ok)


def veff(w, n_bins, t0, t1):
    """static_potential.py's jackknife: (veff, veff_err) [n_r][n_t-1] and (v, v_err) [n_r]."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    n_conf, n_r, n_t = w.shape
    ve, er = np.zeros((n_r, n_t - 1)), np.zeros((n_r, n_t - 1))
    v, ve_r = np.zeros(n_r), np.zeros(n_r)
    a0, a1 = (ctypes.c_int * n_r)(*t0), (ctypes.c_int * n_r)(*t1)
    _ok(lib().su2o_veff(_dp(w), n_conf, n_r, n_t, n_bins, a0, a1, _dp(ve), _dp(er), _dp(v), _dp(ve_r)))
    return ve, er, v, ve_r


def golden():
    import json
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def golden_config(name):
    from masterarbeit_b200.configio import read_config
    return read_config(os.path.join(GOLDEN, name))


def kp_density(alpha, edges):
    """Probability of each bin for the x0 law sqrt(1-x^2) exp(alpha x) on [-1, 1]."""
    x = np.linspace(-1.0, 1.0, 200001)
    f = np.sqrt(np.clip(1.0 - x * x, 0.0, None)) * np.exp(alpha * (x - 1.0))
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (f[1:] + f[:-1]) * np.diff(x))])
    cdf /= cdf[-1]
    return np.diff(np.interp(edges, x, cdf))
