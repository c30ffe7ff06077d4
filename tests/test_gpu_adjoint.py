"""The APE + clover-charge adjoint (su2g_ape_qtop_vjp) against central finite differences.

Directions: per link an su(2) element X = i x.sigma with x ~ N(0,1), applied as U -> exp(eps X) U
(exact SU(2) exponential).  The directional derivative sum g.x from the VJP must match
(Q(+eps) - Q(-eps)) / (2 eps), eps = 1e-4, with the FP64 forward of the GPU (itself pinned to the
reference) and, on a small lattice, with the FP64 forward of the CPU oracle.
"""
import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu

EPS = 1e-4


def qmul(a, b):
    """Quaternion product in the reference's convention (LGT_Code/include/gauge.h:83-91), arrays [..., 4]."""
    a0, a1, a2, a3 = np.moveaxis(a, -1, 0)
    b0, b1, b2, b3 = np.moveaxis(b, -1, 0)
    return np.stack([a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3,
                     a0 * b1 + a1 * b0 - a2 * b3 + a3 * b2,
                     a0 * b2 + a1 * b3 + a2 * b0 - a3 * b1,
                     a0 * b3 - a1 * b2 + a2 * b1 + a3 * b0], axis=-1)


def expi(x, eps):
    """exp(eps * i x.sigma) as a quaternion: (cos(eps|x|), sin(eps|x|) x/|x|)."""
    nx = np.linalg.norm(x, axis=-1, keepdims=True)
    th = eps * nx
    return np.concatenate([np.cos(th), np.sin(th) * x / np.where(nx > 0, nx, 1.0)], axis=-1)


def perturb(U, X, eps):
    return qmul(expi(X, eps), U)


def gpu_q(dims, U, n, alpha):
    L = Lattice(dims, precision="fp64")
    L.upload(U)
    L.ape(n, alpha, "all")
    q = L.qtop()
    L.close()
    return q


@pytest.fixture(scope="module")
def thermalized_8():
    dims, _, U = O.golden_config("cfg_8x8x8x8_base.cfg")
    return dims, U


@pytest.mark.parametrize("n_ape", [1, 5, 30])
def test_vjp_matches_finite_differences(thermalized_8, n_ape):
    dims, U = thermalized_8
    alpha = 0.5
    L = Lattice(dims, precision="fp64")
    L.upload(U)
    q, g = L.ape_qtop_vjp(n_ape, alpha)
    assert abs(q - gpu_q(dims, U, n_ape, alpha)) <= 1e-12 * max(1.0, abs(q))
    rng = np.random.default_rng(100 + n_ape)
    for d in range(16 if n_ape <= 5 else 6):
        X = rng.standard_normal((U.shape[0], 4, 3))
        ad = float(np.sum(g * X))
        fd = (gpu_q(dims, perturb(U, X, EPS), n_ape, alpha) - gpu_q(dims, perturb(U, X, -EPS), n_ape, alpha)) / (2 * EPS)
        scale = float(np.sqrt(np.sum((g * X) ** 2)))  # size of the terms that cancel in sum g.x
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), scale), (n_ape, d, fd, ad, scale)


def test_vjp_matches_oracle_finite_differences():
    """On 4^4 (a configuration written by the reference), with the CPU oracle's FP64 forward."""
    dims, _, U = O.golden_config("cfg_4x4x4x4_base.cfg")
    n_ape, alpha = 3, 0.4
    L = Lattice(dims, precision="fp64")
    L.upload(U)
    q, g = L.ape_qtop_vjp(n_ape, alpha)
    assert abs(q - O.ape_qtop(dims, U, n_ape, alpha)) <= 1e-12 * max(1.0, abs(q))
    rng = np.random.default_rng(7)
    for d in range(8):
        X = rng.standard_normal((U.shape[0], 4, 3))
        ad = float(np.sum(g * X))
        fd = (O.ape_qtop(dims, np.ascontiguousarray(perturb(U, X, EPS)), n_ape, alpha)
              - O.ape_qtop(dims, np.ascontiguousarray(perturb(U, X, -EPS)), n_ape, alpha)) / (2 * EPS)
        scale = float(np.sqrt(np.sum((g * X) ** 2)))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), scale), (d, fd, ad, scale)


def test_checkpointing_does_not_change_the_result(thermalized_8):
    dims, U = thermalized_8
    L = Lattice(dims, precision="fp64")
    L.upload(U)
    ref_q, ref_g = L.ape_qtop_vjp(12, 0.5, ckpt=1)       # every level stored
    for ckpt in (0, 3, 5, 12):                           # sqrt(N) segments, uneven, one segment
        q, g = L.ape_qtop_vjp(12, 0.5, ckpt=ckpt)
        assert q == ref_q
        # the charge adjoint accumulates with atomics, so the order of FP64 additions varies
        assert np.max(np.abs(g - ref_g)) <= 1e-11 * np.max(np.abs(ref_g))
    lev_sqrt, bytes_sqrt = L.vjp_plan(30, 0)
    lev_all, bytes_all = L.vjp_plan(30, 1)
    assert lev_sqrt == 5 + 5 and lev_all == 30 and bytes_sqrt < bytes_all
    # the field of the handle is untouched
    assert np.array_equal(L.download(), U)


def test_fp32_adjoint_tracks_fp64_adjoint(thermalized_8):
    dims, U = thermalized_8
    out = {}
    for prec in ("fp64", "fp32"):
        L = Lattice(dims, precision=prec)
        L.upload(U)
        out[prec] = L.ape_qtop_vjp(10, 0.5)
    q64, g64 = out["fp64"]
    q32, g32 = out["fp32"]
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print("FP32 vs FP64 adjoint: relative L2 error", rel, "dQ", abs(q32 - q64))
    assert rel < 1e-4


# ---- the adjoint configuration of the throughput runs: 24^4 and 48^4 hot starts thermalised by 500
# sweeps (1 heatbath + 4 overrelaxation) at beta = 3.09, N = 30 APE_all steps at alpha = 0.5, then Q.
# The perturbation exp(+-eps X) U runs on the device (su2g_tangent_step) after one upload of the base
# field, so a central difference costs two uploads and two forwards.

def _thermalised(L_, seed):
    L = Lattice((L_,) * 4, precision="fp64", beta=3.09, seed=seed, start="haar")
    L.sweep(500, 1, 4)
    U = L.download()
    L.close()
    return U


def _fd(L, U, X, n_ape, alpha):
    qs = []
    for sgn in (1.0, -1.0):
        L.upload(U)
        L.tangent_step(X, sgn * EPS)
        L.ape(n_ape, alpha, "all")
        qs.append(L.qtop())
    return (qs[0] - qs[1]) / (2 * EPS)


@pytest.mark.parametrize("L_,n_dirs", [(24, 16), (48, 4)])
def test_vjp_matches_finite_differences_at_throughput_sizes(L_, n_dirs):
    """FP64 VJP against FP64 central differences (eps = 1e-4) along N(0,1) su(2) directions, to 1e-6 of
    max(|FD|, the size of the terms of sum g.x); the FP32 VJP (same field rounded to FP32) against the
    same FP64 differences, to 2e-3 of that size (the FP32 VJP's error, ~1e-4 relative in L2, is the
    FP32 rounding of 30 smearing levels propagated backwards)."""
    n_ape, alpha = 30, 0.5
    U = _thermalised(L_, 5000 + L_)
    L64 = Lattice((L_,) * 4, precision="fp64")
    L64.upload(U)
    q64, g64 = L64.ape_qtop_vjp(n_ape, alpha)
    L32 = Lattice((L_,) * 4, precision="fp32")
    L32.upload(U)
    q32, g32 = L32.ape_qtop_vjp(n_ape, alpha)
    L32.close()
    rng = np.random.default_rng(300 + L_)
    worst64 = worst32 = 0.0
    for d in range(n_dirs):
        X = rng.standard_normal((U.shape[0], 4, 3))
        fd = _fd(L64, U, X, n_ape, alpha)
        ad64, ad32 = float(np.sum(g64 * X)), float(np.sum(g32 * X))
        scale = max(abs(fd), float(np.sqrt(np.sum((g64 * X) ** 2))))
        worst64 = max(worst64, abs(fd - ad64) / scale)
        worst32 = max(worst32, abs(fd - ad32) / scale)
        print(f"{L_}^4 direction {d}: FD {fd:+.10e}  VJP fp64 {ad64:+.10e}  fp32 {ad32:+.10e}  (scale {scale:.3e})")
    print(f"{L_}^4 N={n_ape}: Q fp64 {q64:+.9f} fp32 {q32:+.9f}; worst |FD - VJP| / scale: fp64 {worst64:.2e}, "
          f"fp32 {worst32:.2e}")
    L64.close()
    assert worst64 <= 1e-6
    assert worst32 <= 2e-3
