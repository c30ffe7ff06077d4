"""Parity of the CUDA path (libsu2g.so through the C ABI) with the reference and the oracle.

FP64 tolerances follow the reference's own convention (relative 1e-12, LGT_Code/main_test/
test_utils.h:27) with cancellation-aware bounds for sums: |dW| <= 1e-12 (per-site |w| <= 1) and
|dQ| <= 1e-12 * sum_x |q(x)| / (32 pi^2).  FP32 bounds are stated per test.
"""
import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu

LATS = ["4x4x4x4", "6x4x4x8", "8x8x8x8"]


def lattice_from(cfg, precision="fp64", **kw):
    dims, _, U = O.golden_config(cfg)
    lat = Lattice(dims, precision=precision, **kw)
    lat.upload(U)
    return lat, dims, U


@pytest.mark.parametrize("lat", LATS)
def test_plaquette(golden, lat):
    g = golden["lattices"][lat]
    L, dims, U = lattice_from(g["base"])
    assert abs(L.plaquette() - g["plaq"]) <= 1e-13 * abs(g["plaq"])
    back = L.download()
    assert np.array_equal(back, U)   # FP64 upload/download is exact
    L32, _, _ = lattice_from(g["base"], "fp32")
    assert abs(L32.plaquette() - g["plaq"]) <= 2e-7


@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("mode", ["all", "spatial", "temporal"])
def test_ape(golden, lat, mode):
    g = golden["lattices"][lat]
    e = g["ape"][mode]
    L, dims, U = lattice_from(g["base"])
    L.ape(e["ns"], e["alpha"], mode)
    assert abs(L.plaquette() - e["plaq"]) <= 1e-13
    W = L.download()
    ref = O.golden_config(e["cfg"])[2] if "cfg" in e else O.ape(dims, U, e["ns"], e["alpha"], mode)
    assert np.max(np.abs(W - ref)) <= 1e-13
    L32, _, _ = lattice_from(g["base"], "fp32")
    L32.ape(e["ns"], e["alpha"], mode)
    assert np.max(np.abs(L32.download() - ref)) <= 2e-6


@pytest.mark.parametrize("lat", LATS)
def test_wilson(golden, lat):
    g = golden["lattices"][lat]
    R = [x[0] for x in g["wilson"]]
    T = [x[1] for x in g["wilson"]]
    ref = np.array([x[2] for x in g["wilson"]])
    L, dims, U = lattice_from(g["base"])
    assert np.max(np.abs(L.wilson(R, T) - ref)) <= 1e-13
    # pairs in another order, a sub-list and repeated pairs
    perm = np.random.default_rng(1).permutation(len(R))
    w = L.wilson(np.array(R)[perm], np.array(T)[perm])
    assert np.max(np.abs(w - ref[perm])) <= 1e-13
    L32, _, _ = lattice_from(g["base"], "fp32")
    assert np.max(np.abs(L32.wilson(R, T) - ref)) <= 2e-6


def test_wilson_rejects_too_long_loops(golden):
    g = golden["lattices"]["4x4x4x4"]
    L, _, _ = lattice_from(g["base"])
    with pytest.raises(Exception, match="too small"):
        L.wilson([1], [4])


@pytest.mark.parametrize("lat", LATS)
def test_qtop_after_ape(golden, lat):
    g = golden["lattices"][lat]
    for run in g["qtop"]:
        for prec, tol in (("fp64", 1e-12), ("fp32", 2e-5)):
            L, dims, U = lattice_from(g["base"], prec)
            done = 0
            for N, qref in zip(run["N"], run["Q"]):
                L.ape(N - done, run["alpha"], "all")
                done = N
                q, sabs = L.qtop(with_abs=True)
                assert abs(q - qref) <= tol * sabs, (prec, N, q, qref, sabs)


@pytest.mark.parametrize("dims", [(4, 4, 6, 6), (6, 6, 4, 10), (4, 6, 8, 10), (2, 4, 6, 4)])
def test_ape_and_qtop_on_ragged_geometries(dims):
    """Half volumes that are not whole multiples of a CTA's run of sites (288 and 720 against the
    64 sites of a 128-thread CTA whose warps alternate parity; 960 against the 128 sites of the
    FP64 CTAs), so the last CTA of the APE and charge kernels is partly empty: APE in every mode,
    then Q, against the oracle on the same uploaded Haar field, in FP64 and FP32.  An extent of 2
    makes the charge's 3-link offsets wrap twice."""
    U = O.start(dims, "haar", 17)
    for mode in ("all", "spatial", "temporal"):
        ref = O.ape(dims, U, 3, 0.4, mode)
        qref, _ = O.qtop(dims, ref)
        for prec, tol, qtol in (("fp64", 1e-13, 1e-12), ("fp32", 2e-6, 2e-5)):
            L = Lattice(dims, precision=prec)
            L.upload(U)
            L.ape(3, 0.4, mode)
            assert np.max(np.abs(L.download() - ref)) <= tol, (prec, mode)
            q, sabs = L.qtop(with_abs=True)
            assert abs(q - qref) <= qtol * sabs, (prec, mode, q, qref)


@pytest.mark.parametrize("lat", LATS)
def test_heatbath_matches_reference_link_by_link(golden, lat):
    """GPU checkerboard heatbath vs the reference's localHeatbathUpdate on the same Philox uniforms."""
    g = golden["lattices"][lat]
    e = g["hbinj"]
    dims, _, U = O.golden_config(g["base"])
    L = Lattice(dims, precision="fp64", beta=e["beta"], seed=e["seed"], start="cold")
    L.upload(U)
    L.set_sweep_counter(e["sweep0"])
    acc = L.sweep(e["sweeps"], 1, 0, acc=True)
    assert abs(acc - np.mean(e["acc"])) <= 1e-12
    assert abs(L.plaquette() - e["plaq"][-1]) <= 1e-12
    ref = O.golden_config(e["cfg"])[2] if "cfg" in e else None
    if ref is None:
        ref = U.copy()
        for s in range(e["sweeps"]):
            O.sweep(dims, ref, "hb", e["beta"], e["seed"], e["sweep0"] + s)
    assert np.max(np.abs(L.download() - ref)) <= 1e-12


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (6, 4, 4, 8), (8, 8, 8, 8), (2, 4, 6, 4)])
@pytest.mark.parametrize("mode", ["haar", "ref"])
def test_start_matches_oracle(dims, mode):
    L = Lattice(dims, precision="fp64", seed=99, start=mode)
    ref = O.start(dims, mode, 99)
    assert np.max(np.abs(L.download() - ref)) <= 1e-14
    # FP32 uniforms keep the top 23 bits of each Philox word, so Box-Muller / sqrt(1 - c^2) near
    # their singular points move by more than FP32 rounding; typical links agree to ~1e-7.
    L32 = Lattice(dims, precision="fp32", seed=99, start=mode)
    d = np.abs(L32.download() - ref)
    assert np.max(d) <= 2e-4 and np.median(d) <= 1e-6


def test_ref_start_matches_reference(golden):
    for lat in ("4x4x4x4", "6x4x4x8"):
        e = golden["lattices"][lat]["hotinj"]
        L = Lattice(golden["lattices"][lat]["dims"], precision="fp64", seed=e["seed"], start="ref")
        assert np.max(np.abs(L.download() - O.golden_config(e["cfg"])[2])) <= 1e-14


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (6, 4, 4, 8), (4, 6, 8, 10)])
def test_heatbath_and_overrelaxation_vs_oracle(dims):
    """Several HB + OR sweeps from a Haar start, link by link against the oracle (FP64).  Rounding
    differences (FMA contraction, rsqrt vs division) grow through the chain; 1e-12 holds for one
    sweep, 3 sweeps of 1 HB + 2 OR stay below 1e-9."""
    L = Lattice(dims, precision="fp64", beta=2.7, seed=5, start="haar")
    U = O.start(dims, "haar", 5)
    for s in range(3):
        L.sweep(1, 1, 2)
        O.sweep(dims, U, "hb", 2.7, 5, s)
        O.sweep(dims, U, "or")
        O.sweep(dims, U, "or")
        if s == 0:
            assert np.max(np.abs(L.download() - U)) <= 1e-12
    assert np.max(np.abs(L.download() - U)) <= 1e-9


@pytest.mark.parametrize("mu", [0, 1, 2, 3])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 2e-6)])
def test_overrelaxation_invariants(mu, prec, tol):
    """A single OR pass keeps every updated link's Re tr(U A) (A its unchanged staple), keeps the
    plaquette sum, and applying it twice gives back the field."""
    dims = (6, 4, 4, 8)
    L = Lattice(dims, precision=prec, beta=2.5, seed=3, start="haar")
    L.sweep(2, 1, 0)
    U0 = L.download()
    p0 = L.plaquette()
    L.update_pass(1, mu, 1)
    U1 = L.download()
    assert abs(L.plaquette() - p0) <= tol
    assert np.max(np.abs(U1 - U0)) > 1e-3
    assert abs(O.link_action(dims, U1) - O.link_action(dims, U0)) <= tol * 4 * np.prod(dims) * 6
    L.update_pass(1, mu, 1)
    assert np.max(np.abs(L.download() - U0)) <= 4 * tol


def test_fp32_chain_tracks_fp64_chain():
    """FP32 and FP64 chains draw identical Philox words; the links differ at the FP32 rounding level
    until accept/reject flips (and the chaos of the update) separate the chains.  The first sweep
    agrees to FP32 accuracy; the separation sweep is printed."""
    g = O.golden()["lattices"]["8x8x8x8"]
    dims, _, U = O.golden_config(g["base"])
    L64 = Lattice(dims, precision="fp64", beta=3.09, seed=11)
    L32 = Lattice(dims, precision="fp32", beta=3.09, seed=11)
    L64.upload(U)
    L32.upload(U)
    diffs, linkd = [], []
    for s in range(6):
        L64.sweep(1, 1, 0)
        L32.sweep(1, 1, 0)
        diffs.append(abs(L64.plaquette() - L32.plaquette()))
        linkd.append(float(np.median(np.abs(L64.download() - L32.download()))))
    print("heatbath sweeps: plaquette |fp32 - fp64|:", diffs, "median link difference:", linkd)
    assert diffs[0] < 1e-6 and linkd[0] < 1e-5, (diffs, linkd)
    assert diffs[1] < 1e-5, diffs


def test_deterministic_repeat():
    dims = (8, 8, 8, 8)
    out = []
    for _ in range(2):
        L = Lattice(dims, precision="fp32", beta=3.09, seed=21, start="haar")
        L.sweep(3, 1, 4)
        out.append((L.download(), L.plaquette(), L.qtop()))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]


def _chi2_vs_law(counts, alpha, nb):
    n = int(counts.sum())
    p = O.kp_density(alpha, np.linspace(-1, 1, nb + 1))
    m = n * p > 20
    dof = int(m.sum()) - 1
    chi2 = float(np.sum((counts[m] - n * p[m]) ** 2 / (n * p[m])))
    return chi2, dof, m


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("alpha", [1.5, 4.0, 7.0, 12.0])
def test_kp_sampler_histogram_matches_law(prec, alpha):
    """The heatbath's own per-link sampler (heatbath_link in the handle's precision) against the
    analytic x0 law sqrt(1-x^2) exp(alpha x) by chi^2 over 200 bins, at alpha values that cover the
    batch runs' beta in [2.2, 3.2] (alpha = |A| beta: about 1.5 on a disordered start up to 12 near
    a cold one) and alpha = 7 of the reference's own sampler test (LGT_Code/main_test/test.c)."""
    L = Lattice((4, 4, 4, 4), precision=prec)
    n, nb = 20_000_000, 200
    counts = L.kp_histogram(alpha, 77 + int(10 * alpha), n, nb)
    L.close()
    assert counts.sum() == n
    chi2, dof, m = _chi2_vs_law(counts, alpha, nb)
    # 5 sigma of the chi^2 law with dof degrees of freedom
    assert chi2 < dof + 5 * np.sqrt(2 * dof), (chi2, dof)
    if alpha == 7.0:
        # two-sample chi^2 against the reference's own N=1e8 histogram improved.dat
        pref = np.loadtxt(O.GOLDEN + "/kp_improved.dat")[:, 1] / nb
        nref = 1e8
        a, b = counts[m].astype(float), nref * pref[m]
        chi2r = np.sum((a * np.sqrt(nref / n) - b * np.sqrt(n / nref)) ** 2 / (a + b))
        assert chi2r < dof + 5 * np.sqrt(2 * dof), (chi2r, dof)


def test_kp_sampler_matches_oracle_draws():
    """The same Philox draws give the same x0 in the FP64 heatbath sampler and in the oracle:
    identical histograms (bins computed as the kernel computes them)."""
    L = Lattice((4, 4, 4, 4), precision="fp64")
    n, nb = 200_000, 64
    x = O.kp_samples(5.0, 9, n)
    ref = np.bincount(np.clip(((x + 1.0) * 0.5 * nb).astype(int), 0, nb - 1), minlength=nb)
    assert np.array_equal(L.kp_histogram(5.0, 9, n, nb), ref)
    L.close()


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (10, 6, 4, 8)])
def test_observables_vs_oracle_random(dims):
    L = Lattice(dims, precision="fp64", beta=2.4, seed=13, start="haar")
    L.sweep(2, 1, 1)
    U = L.download()
    assert abs(L.plaquette() - O.plaquette(dims, U)) <= 1e-13
    R = [1, 2, 3, 5, 9, 1, 4]
    T = [1, 1, 2, 3, 2, dims[0] - 1, dims[0] - 1]
    assert np.max(np.abs(L.wilson(R, T) - O.wilson(dims, U, R, T))) <= 1e-13
    q, sabs = L.qtop(with_abs=True)
    qo, _ = O.qtop(dims, U)
    assert abs(q - qo) <= 1e-12 * sabs
    L.ape(2, 0.5, "spatial")
    assert np.max(np.abs(L.download() - O.ape(dims, U, 2, 0.5, "spatial"))) <= 1e-13


@pytest.mark.parametrize("dims", [(34, 4, 4, 4), (10, 6, 4, 6), (12, 4, 6, 2), (48, 2, 2, 2)])
def test_wilson_kernels_against_oracle(dims):
    """The column Wilson-loop kernel (time extents whose CTA fits: 10, 12, 48, with ragged last
    tiles) and the per-site kernel (L_t = 34, whose column CTA would exceed the thread limit),
    against the oracle, R up to 9 (chunks of 4/2/1 and 8/1) and T up to 31."""
    L = Lattice(dims, precision="fp64", seed=31, start="haar")
    U = L.download()
    rmax, tmax = 9, min(dims[0] - 1, 31)
    R = [r for r in range(1, rmax + 1) for t in range(1, tmax + 1)]
    T = [t for r in range(1, rmax + 1) for t in range(1, tmax + 1)]
    ref = O.wilson(dims, U, R, T)
    assert np.max(np.abs(L.wilson(R, T) - ref)) <= 1e-13
    L32 = Lattice(dims, precision="fp32")
    L32.upload(U)
    assert np.max(np.abs(L32.wilson(R, T) - ref)) <= 2e-6
