"""ctypes binding of libsu2g.so (include/su2g.h).

This is a thin host-side convenience layer over the C ABI for tests, benchmarks and Python
callers; the C ABI itself is the product boundary.  Every call goes to the CUDA library; if
the library cannot be loaded or no sm_100 GPU is present, the calls raise -- there is no CPU
fallback.
"""
import ctypes
import os
import re

import numpy as np

from . import build as _build

FP32, FP64 = 0, 1
START = {"cold": 0, "haar": 1, "ref": 2}
APE = {"all": 0, "spatial": 1, "temporal": 2}
HEATBATH, OVERRELAX = 0, 1
KERNEL_CLASSES = ["heatbath", "overrelax", "plaquette", "ape", "wilson", "qtop", "reduce", "other", "metropolis"]

_HEADER = os.path.join(_build.REPO, "include", "su2g.h")


class Su2gError(RuntimeError):
    """A libsu2g call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"su2g error {code}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int32 * 4),
        ("precision", ctypes.c_int32),
        ("start", ctypes.c_int32),
        ("beta", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("replica", ctypes.c_uint32),
        ("device", ctypes.c_int32),
    ]


class ReplicaSpec(ctypes.Structure):
    _fields_ = [
        ("dims", ctypes.c_int32 * 4),
        ("beta", ctypes.c_double),
        ("seed", ctypes.c_uint64),
        ("replica", ctypes.c_uint32),
        ("start", ctypes.c_int32),
    ]


class MeasSpec(ctypes.Structure):
    _fields_ = [
        ("n_q", ctypes.c_int32),
        ("q_ape", ctypes.POINTER(ctypes.c_int32)),
        ("alpha_q", ctypes.c_double),
        ("n_w", ctypes.c_int32),
        ("R", ctypes.POINTER(ctypes.c_int32)),
        ("T", ctypes.POINTER(ctypes.c_int32)),
        ("ns_t", ctypes.c_int32),
        ("alpha_t", ctypes.c_double),
        ("ns_s", ctypes.c_int32),
        ("alpha_s", ctypes.c_double),
    ]


_lib = None
_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_I32P = ctypes.POINTER(ctypes.c_int32)
_I64P = ctypes.POINTER(ctypes.c_int64)

_SIGS = {
    "su2g_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.POINTER(_P)]),
    "su2g_destroy": (ctypes.c_int, [_P]),
    "su2g_last_error": (ctypes.c_char_p, [_P]),
    "su2g_start": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_uint64]),
    "su2g_info": (ctypes.c_int, [_P, _I32P, _I32P, _I64P, ctypes.POINTER(ctypes.c_uint32)]),
    "su2g_set_beta": (ctypes.c_int, [_P, ctypes.c_double]),
    "su2g_set_sweep_counter": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "su2g_upload_aos_f64": (ctypes.c_int, [_P, _DP]),
    "su2g_download_aos_f64": (ctypes.c_int, [_P, _DP]),
    "su2g_sweep": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP]),
    "su2g_sweep_plaquette": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]),
    "su2g_update_pass": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32]),
    "su2g_graph_run": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]),
    "su2g_graph_release": (ctypes.c_int, [_P]),
    "su2g_read_config": (ctypes.c_int, [_P, ctypes.c_char_p, _DP, _DP]),
    "su2g_write_config": (ctypes.c_int, [_P, ctypes.c_char_p, _DP]),
    "su2g_read_config_reflect": (ctypes.c_int, [_P, ctypes.c_char_p, _DP, _DP]),
    "su2g_measure": (ctypes.c_int, [_P, ctypes.POINTER(MeasSpec), _DP, _DP]),
    "su2g_measure_release": (ctypes.c_int, [_P]),
    "su2g_gauge_update": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                         ctypes.c_int32, _DP]),
    "su2g_stats_tau_int": (ctypes.c_int, [_DP, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                          ctypes.c_int32, _DP, _I32P]),
    "su2g_stats_veff": (ctypes.c_int, [_DP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _I32P,
                                       _I32P, ctypes.c_int32, _DP, _DP, _DP, _DP]),
    "su2g_batch_tau_int": (ctypes.c_int, [_P, ctypes.c_int32, _DP, _I32P]),
    "su2g_selftest_bounded_wait": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "su2g_plaquette": (ctypes.c_int, [_P, _DP]),
    "su2g_ape": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32]),
    "su2g_wilson": (ctypes.c_int, [_P, _I32P, _I32P, ctypes.c_int32, _DP]),
    "su2g_qtop": (ctypes.c_int, [_P, _DP, _DP]),
    "su2g_ape_qtop_vjp": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _DP, _DP]),
    "su2g_vjp_plan": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _I32P, _I64P]),
    "su2g_tangent_step": (ctypes.c_int, [_P, _DP, ctypes.c_double]),
    "su2g_kp_histogram":(ctypes.c_int, [_P, ctypes.c_double, ctypes.c_uint64, ctypes.c_int64, ctypes.c_int32, _I64P]),
    "su2g_ape_inplace_noalloc": (ctypes.c_int, [_P, _I32P, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _P]),
    "su2g_batch_create": (ctypes.c_int, [ctypes.POINTER(ReplicaSpec), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                         ctypes.POINTER(_P)]),
    "su2g_batch_destroy": (ctypes.c_int, [_P]),
    "su2g_batch_last_error": (ctypes.c_char_p, [_P]),
    "su2g_batch_run": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _DP, _DP]),
    "su2g_batch_autotune": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, _I32P]),
    "su2g_batch_configure": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "su2g_batch_config": (ctypes.c_int, [_P, _I32P, _I32P]),
    "su2g_batch_selftest_grid_barrier": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int64]),
    "su2g_batch_download": (ctypes.c_int, [_P, ctypes.c_int32, _DP]),
    "su2g_batch_upload": (ctypes.c_int, [_P, ctypes.c_int32, _DP]),
    "su2g_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(_P)]),
    "su2g_host_free": (ctypes.c_int, [_P]),
    "su2g_stream": (ctypes.c_int, [_P, ctypes.POINTER(_P)]),
    "su2g_synchronize": (ctypes.c_int, [_P]),
    "su2g_timer_begin": (ctypes.c_int, [_P]),
    "su2g_timer_end": (ctypes.c_int, [_P, _DP]),
    "su2g_profile_enable": (ctypes.c_int, [_P, ctypes.c_int32]),
    "su2g_profile_read": (ctypes.c_int, [_P, ctypes.c_int32, _I64P, _DP]),
    "su2g_set_kernel_variant": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "su2g_kernel_variant": (ctypes.c_int, [_P, ctypes.c_int32, _I32P]),
}


def header_functions(path=_HEADER):
    """Names of every function declared in include/su2g.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(su2g_[a-z0-9_]+)\s*\(", text)))


def load(path=None, build_if_missing=True):
    """Load libsu2g.so (building it with nvcc if it is missing or stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = _build.build() if build_if_missing else _build.LIB
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _as_dp(a):
    return a.ctypes.data_as(_DP)


class PinnedArray:
    """A numpy array over page-locked host memory from su2g_host_alloc."""

    def __init__(self, shape, dtype=np.float64):
        self.lib = load()
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = _P()
        rc = self.lib.su2g_host_alloc(nbytes, ctypes.byref(p))
        if rc != 0:
            raise Su2gError(rc, self.lib.su2g_last_error(None).decode())
        self.ptr = p
        buf = (ctypes.c_char * nbytes).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if getattr(self, "ptr", None):
            self.array = None
            self.lib.su2g_host_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Lattice:
    """One SU(2) gauge field resident on a B200, driven through the C ABI."""

    def __init__(self, dims, precision="fp32", beta=2.3, seed=1, start="cold", replica=0, device=0):
        self.lib = load()
        p = Params()
        for i in range(4):
            p.dims[i] = int(dims[i])
        p.precision = FP64 if str(precision).lower() in ("fp64", "f64", "double", "1") else FP32
        p.start = START[start] if isinstance(start, str) else int(start)
        p.beta = float(beta)
        p.seed = int(seed)
        p.replica = int(replica)
        p.device = int(device)
        h = _P()
        rc = self.lib.su2g_create(ctypes.byref(p), ctypes.byref(h))
        if rc != 0:
            raise Su2gError(rc, self.lib.su2g_last_error(None).decode())
        self.h = h
        self.dims = tuple(int(d) for d in dims)
        self.volume = int(np.prod(self.dims))
        self.precision = "fp64" if p.precision == FP64 else "fp32"

    # -- plumbing
    def _check(self, rc):
        if rc != 0:
            raise Su2gError(rc, self.lib.su2g_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.su2g_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state
    def start(self, mode="cold", seed=1):
        self._check(self.lib.su2g_start(self.h, START[mode] if isinstance(mode, str) else int(mode), int(seed)))

    def info(self):
        dims = (ctypes.c_int32 * 4)()
        prec, vol, sw = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_uint32()
        self._check(self.lib.su2g_info(self.h, dims, ctypes.byref(prec), ctypes.byref(vol), ctypes.byref(sw)))
        return {"dims": tuple(dims), "precision": prec.value, "volume": vol.value, "hb_sweeps": sw.value}

    def set_beta(self, beta):
        self._check(self.lib.su2g_set_beta(self.h, float(beta)))

    def set_sweep_counter(self, n):
        self._check(self.lib.su2g_set_sweep_counter(self.h, int(n)))

    def upload(self, links):
        a = np.ascontiguousarray(links, dtype=np.float64).reshape(self.volume * 16)
        self._check(self.lib.su2g_upload_aos_f64(self.h, _as_dp(a)))

    def download(self, out=None):
        a = out if out is not None else np.empty((self.volume, 4, 4), dtype=np.float64)
        self._check(self.lib.su2g_download_aos_f64(self.h, _as_dp(a)))
        return a

    # -- updates
    def sweep(self, n_sweeps=1, n_hb=1, n_or=0, acc=False):
        if acc:
            v = ctypes.c_double()
            self._check(self.lib.su2g_sweep(self.h, n_sweeps, n_hb, n_or, ctypes.byref(v)))
            return v.value
        self._check(self.lib.su2g_sweep(self.h, n_sweeps, n_hb, n_or, None))
        return None

    def sweep_plaquette(self, n_sweeps=1, n_hb=1, n_or=0, acc=False):
        """sweep() and the plaquette of the resulting field, summed inside the last sweep's update
        passes; returns the plaquette, or (plaquette, acceptance) with acc=True."""
        p, a = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.su2g_sweep_plaquette(self.h, n_sweeps, n_hb, n_or, ctypes.byref(p),
                                                  ctypes.byref(a) if acc else None))
        return (p.value, a.value) if acc else p.value

    def gauge_update(self, nup=1, utype=1, stype=0, eps=0.15, hits=1):
        """gaugefieldUpdate(iup, nup, utype, stype): utype 1 heatbath / 0 Metropolis (step eps,
        `hits` hits per visit); stype 0 every link once / 1 random site selection.  Returns the
        mean acceptance per link visit."""
        v = ctypes.c_double()
        self._check(self.lib.su2g_gauge_update(self.h, int(nup), int(utype), int(stype), float(eps), int(hits),
                                                ctypes.byref(v)))
        return v.value

    def update_pass(self, kind, mu, parity, sweep=0):
        self._check(self.lib.su2g_update_pass(self.h, int(kind), int(mu), int(parity), int(sweep)))

    def graph_run(self, n_blocks, meas_every=1, n_hb=1, n_or=0):
        """n_blocks x [meas_every x (n_hb HB + n_or OR sweeps), plaquette] from one replayed CUDA
        graph; returns (plaquette trace, acceptance trace), one entry per block."""
        plaq = np.zeros(int(n_blocks))
        acc = np.zeros(int(n_blocks))
        self._check(self.lib.su2g_graph_run(self.h, int(n_blocks), int(meas_every), int(n_hb), int(n_or),
                                            plaq.ctypes.data_as(_DP), acc.ctypes.data_as(_DP)))
        return plaq, acc

    def graph_release(self):
        self._check(self.lib.su2g_graph_release(self.h))

    # -- configuration files (the reference's binary format)
    def read_config(self, path):
        """Stream a configuration file into the field; returns (file plaquette, computed plaquette)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.su2g_read_config(self.h, os.fsencode(path), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def write_config(self, path):
        """Write the field to a configuration file; returns the plaquette stored in its header."""
        v = ctypes.c_double()
        self._check(self.lib.su2g_write_config(self.h, os.fsencode(path), ctypes.byref(v)))
        return v.value

    def read_config_reflect(self, path):
        """readConfigForThermalisation: fill the field from a file of half the extents by 16
        mirror images; returns (file plaquette, computed plaquette)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.su2g_read_config_reflect(self.h, os.fsencode(path), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def measure(self, q_ape=(), alpha_q=0.0, R=(), T=(), ns_t=0, alpha_t=0.0, ns_s=0, alpha_s=0.0):
        """One measurement of the meas / qtop drivers on a copy of the field (one CUDA graph):
        Q after each cumulative APE_all step count in q_ape, and W(R[i], T[i]) after ns_t temporal
        and ns_s spatial steps.  Returns (q array, w array); the field is left unchanged."""
        qa = (ctypes.c_int32 * max(1, len(q_ape)))(*[int(x) for x in q_ape])
        Ra = (ctypes.c_int32 * max(1, len(R)))(*[int(x) for x in R])
        Ta = (ctypes.c_int32 * max(1, len(T)))(*[int(x) for x in T])
        if len(R) != len(T):
            raise ValueError("R and T differ in length")
        spec = MeasSpec(len(q_ape), qa, float(alpha_q), len(R), Ra, Ta, int(ns_t), float(alpha_t), int(ns_s),
                        float(alpha_s))
        q = np.zeros(max(1, len(q_ape)))
        w = np.zeros(max(1, len(R)))
        self._check(self.lib.su2g_measure(self.h, ctypes.byref(spec), q.ctypes.data_as(_DP), w.ctypes.data_as(_DP)))
        return q[:len(q_ape)], w[:len(R)]

    def measure_release(self):
        self._check(self.lib.su2g_measure_release(self.h))

    def selftest_bounded_wait(self, poll_limit=1 << 12):
        """Run the bounded-wait diagnostic; raises Su2gError (SU2G_EDEVICE, timeout) as designed."""
        self._check(self.lib.su2g_selftest_bounded_wait(self.h, int(poll_limit)))

    # -- observables
    def plaquette(self):
        v = ctypes.c_double()
        self._check(self.lib.su2g_plaquette(self.h, ctypes.byref(v)))
        return v.value

    def ape(self, ns, alpha, mode="all"):
        self._check(self.lib.su2g_ape(self.h, int(ns), float(alpha), APE[mode] if isinstance(mode, str) else int(mode)))

    def wilson(self, R, T):
        R = np.ascontiguousarray(R, dtype=np.int32)
        T = np.ascontiguousarray(T, dtype=np.int32)
        w = np.empty(len(R), dtype=np.float64)
        self._check(self.lib.su2g_wilson(self.h, R.ctypes.data_as(_I32P), T.ctypes.data_as(_I32P), len(R), _as_dp(w)))
        return w

    def qtop(self, with_abs=False):
        q, a = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.su2g_qtop(self.h, ctypes.byref(q), ctypes.byref(a)))
        return (q.value, a.value) if with_abs else q.value

    def ape_qtop_vjp(self, n_ape, alpha, ckpt=0, grad=True):
        """Q after n_ape APE_all steps and dQ/dU as su(2) coefficients per link, shape (V, 4, 3)."""
        q = ctypes.c_double()
        g = np.empty((self.volume, 4, 3), dtype=np.float64) if grad else None
        self._check(self.lib.su2g_ape_qtop_vjp(self.h, int(n_ape), float(alpha), int(ckpt), ctypes.byref(q),
                                               _as_dp(g) if grad else None))
        return (q.value, g) if grad else q.value

    def tangent_step(self, x, eps):
        """U -> exp(eps X) U for every link, x = su(2) coefficients in the gradient's layout (V, 4, 3)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != 12 * self.info()["volume"]:
            raise ValueError("tangent coefficients must have V x 4 x 3 entries")
        self._check(self.lib.su2g_tangent_step(self.h, x.ctypes.data_as(_DP), float(eps)))

    def vjp_plan(self, n_ape, ckpt=0):
        lev, nb = ctypes.c_int32(), ctypes.c_int64()
        self._check(self.lib.su2g_vjp_plan(self.h, int(n_ape), int(ckpt), ctypes.byref(lev), ctypes.byref(nb)))
        return lev.value, nb.value

    def kp_histogram(self, alpha, seed, n, nbins=200):
        c = np.zeros(nbins, dtype=np.int64)
        self._check(self.lib.su2g_kp_histogram(self.h, float(alpha), int(seed), int(n), int(nbins),
                                               c.ctypes.data_as(_I64P)))
        return c

    # -- timing
    def synchronize(self):
        self._check(self.lib.su2g_synchronize(self.h))

    def timer_begin(self):
        self._check(self.lib.su2g_timer_begin(self.h))

    def timer_end(self):
        v = ctypes.c_double()
        self._check(self.lib.su2g_timer_end(self.h, ctypes.byref(v)))
        return v.value

    def set_kernel_variant(self, kernel_class, variant):
        cls = KERNEL_CLASSES.index(kernel_class) if isinstance(kernel_class, str) else int(kernel_class)
        self._check(self.lib.su2g_set_kernel_variant(self.h, cls, int(variant)))

    def kernel_variant(self, kernel_class):
        cls = KERNEL_CLASSES.index(kernel_class) if isinstance(kernel_class, str) else int(kernel_class)
        v = ctypes.c_int32()
        self._check(self.lib.su2g_kernel_variant(self.h, cls, ctypes.byref(v)))
        return v.value

    def profile(self, enable=True):
        self._check(self.lib.su2g_profile_enable(self.h, 1 if enable else 0))

    def profile_read(self):
        out = {}
        for i, name in enumerate(KERNEL_CLASSES):
            n, ms = ctypes.c_int64(), ctypes.c_double()
            self._check(self.lib.su2g_profile_read(self.h, i, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (n.value, ms.value)
        return out


def stats_tau_int(series, device=0):
    """t_int.c on the device for each column of `series` ([n] or [n, n_series]): returns
    (array [n_series, 4] of mean, tau_int, naive error, error; resolved flags)."""
    lib = load()
    x = np.ascontiguousarray(series, dtype=np.float64)
    n, ns = (x.shape[0], 1) if x.ndim == 1 else x.shape
    out = np.zeros((ns, 4))
    res = np.zeros(ns, dtype=np.int32)
    rc = lib.su2g_stats_tau_int(x.ctypes.data_as(_DP), n, ns, ns, 1, int(device), out.ctypes.data_as(_DP),
                                res.ctypes.data_as(_I32P))
    if rc:
        raise Su2gError(rc, lib.su2g_last_error(None).decode())
    return out, res.astype(bool)


def stats_veff(w, n_bins, t_fit_start, t_fit_end, device=0):
    """static_potential.py's jackknife on the device; w[c][r][t] = W(R_r, T_t).  Returns
    (veff, veff_err) [n_r][n_t - 1] and (v, v_err) [n_r]."""
    lib = load()
    w = np.ascontiguousarray(w, dtype=np.float64)
    n_conf, n_r, n_t = w.shape
    ve, er = np.zeros((n_r, n_t - 1)), np.zeros((n_r, n_t - 1))
    v, verr = np.zeros(n_r), np.zeros(n_r)
    t0 = (ctypes.c_int32 * n_r)(*[int(x) for x in t_fit_start])
    t1 = (ctypes.c_int32 * n_r)(*[int(x) for x in t_fit_end])
    rc = lib.su2g_stats_veff(w.ctypes.data_as(_DP), n_conf, n_r, n_t, int(n_bins), t0, t1, int(device),
                             ve.ctypes.data_as(_DP), er.ctypes.data_as(_DP), v.ctypes.data_as(_DP),
                             verr.ctypes.data_as(_DP))
    if rc:
        raise Su2gError(rc, lib.su2g_last_error(None).decode())
    return ve, er, v, verr


class Batch:
    """Many independent replicas (extents, beta, seed, start per replica) driven together."""

    def __init__(self, replicas, precision="fp32", device=0):
        """replicas: list of dicts with keys dims, beta, seed, replica (default: index), start."""
        self.lib = load()
        n = len(replicas)
        arr = (ReplicaSpec * n)()
        for i, r in enumerate(replicas):
            for d in range(4):
                arr[i].dims[d] = int(r["dims"][d])
            arr[i].beta = float(r["beta"])
            arr[i].seed = int(r["seed"])
            arr[i].replica = int(r.get("replica", i))
            s = r.get("start", "cold")
            arr[i].start = START[s] if isinstance(s, str) else int(s)
        prec = FP64 if str(precision).lower() in ("fp64", "f64", "double") else FP32
        h = _P()
        rc = self.lib.su2g_batch_create(arr, n, prec, int(device), ctypes.byref(h))
        if rc != 0:
            raise Su2gError(rc, self.lib.su2g_last_error(None).decode())
        self.h = h
        self.n = n
        self.replicas = [dict(r) for r in replicas]

    def _check(self, rc):
        if rc != 0:
            raise Su2gError(rc, self.lib.su2g_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.su2g_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n_sweeps, n_hb=1, n_or=0, meas_every=1):
        """Returns (plaquette trace [n_sweeps // meas_every, n] or None, device ms)."""
        nmeas = n_sweeps // meas_every if meas_every else 0
        trace = np.empty((nmeas, self.n)) if nmeas else None
        ms = ctypes.c_double()
        self._check(self.lib.su2g_batch_run(self.h, int(n_sweeps), int(n_hb), int(n_or), int(meas_every),
                                            _as_dp(trace) if trace is not None else None, ctypes.byref(ms)))
        return trace, ms.value

    def tau_int(self, skip=0):
        """t_int.c of every replica's plaquette trace from the last run, on the device: (array
        [n, 4] of mean, tau_int, naive error, error; resolved flags)."""
        out = np.zeros((self.n, 4))
        res = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.su2g_batch_tau_int(self.h, int(skip), out.ctypes.data_as(_DP), res.ctypes.data_as(_I32P)))
        return out, res.astype(bool)

    def autotune(self, n_hb=1, n_or=4):
        b = ctypes.c_int32()
        self._check(self.lib.su2g_batch_autotune(self.h, int(n_hb), int(n_or), ctypes.byref(b)))
        return b.value

    MODES = {"graph": 0, "persistent": 1}

    def configure(self, mode="graph", block=256):
        """Run the sweeps as a replayed graph of per-pass launches or as one persistent launch."""
        self._check(self.lib.su2g_batch_configure(self.h, self.MODES[mode], int(block)))

    def selftest_grid_barrier(self, missing=1, wait_cycles=100_000_000):
        """The persistent form's bounded barrier waiting for `missing` CTAs that do not exist; raises
        Su2gError (SU2G_EDEVICE) when the wait runs out, as designed."""
        self._check(self.lib.su2g_batch_selftest_grid_barrier(self.h, int(missing), int(wait_cycles)))

    def config(self):
        m, b = ctypes.c_int32(), ctypes.c_int32()
        self._check(self.lib.su2g_batch_config(self.h, ctypes.byref(m), ctypes.byref(b)))
        return {v: k for k, v in self.MODES.items()}[m.value], b.value

    def download(self, r):
        V = int(np.prod(self.replicas[r]["dims"]))
        a = np.empty((V, 4, 4))
        self._check(self.lib.su2g_batch_download(self.h, int(r), _as_dp(a)))
        return a

    def upload(self, r, links):
        a = np.ascontiguousarray(links, dtype=np.float64)
        self._check(self.lib.su2g_batch_upload(self.h, int(r), _as_dp(a)))
