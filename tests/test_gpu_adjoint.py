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
