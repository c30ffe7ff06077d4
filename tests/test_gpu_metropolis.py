"""The reference's other update algorithm and sweep order on the GPU (su2g_gauge_update):
Metropolis (localMetropolisUpdate, metro.c:78-109) and random site selection (gaugefieldUpdate
stype 1, update.c:126-136).  Link by link against the reference's own Metropolis on the same Philox
uniforms and against the oracle for the random order; statistically against the reference's own
RANLUX chains (plaquette within 2 sigma, errors from the t_int.c Gamma method)."""
import numpy as np
import pytest

import _oracle as O
import _stats
from masterarbeit_b200 import Lattice
from masterarbeit_b200.su2g import Su2gError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lat", ["4x4x4x4", "6x4x4x8"])
def test_metropolis_matches_reference_link_by_link(golden, lat):
    e = golden["metropolis"]["inj"][lat]
    dims, _, U = O.golden_config(f"cfg_{lat}_base.cfg")
    _, _, R = O.golden_config(e["cfg"])
    L = Lattice(dims, precision="fp64", beta=e["beta"], seed=e["seed"])
    L.upload(U)
    L.set_sweep_counter(e["sweep0"])
    acc = L.gauge_update(e["sweeps"], utype=0, stype=0, eps=e["eps"], hits=1)
    assert np.max(np.abs(L.download() - R)) <= 1e-12
    assert abs(acc - np.mean(e["acc"])) <= 1e-12
    assert abs(L.plaquette() - e["plaq"][-1]) <= 1e-12


@pytest.mark.parametrize("utype,hits", [(0, 1), (0, 3), (1, 1)])
@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (6, 4, 4, 8)])
def test_random_order_matches_oracle(dims, utype, hits):
    L = Lattice(dims, precision="fp64", beta=2.7, seed=99, start="haar")
    U = L.download()
    L.set_sweep_counter(5)
    accs = [L.gauge_update(1, utype=utype, stype=1, eps=0.4, hits=hits) for _ in range(3)]
    W = U.copy()
    ref = [O.visit_sweep(dims, W, utype, 1, 2.7, 0.4, hits, 99, 5 + s) for s in range(3)]
    assert np.max(np.abs(L.download() - W)) <= 1e-12
    assert np.allclose(accs, ref, rtol=1e-12, atol=0)
    # some sites are visited twice and some not at all
    assert 0.0 < min(accs)


def test_fp32_metropolis_follows_fp64():
    dims = (6, 4, 4, 8)
    out = {}
    for prec in ("fp64", "fp32"):
        L = Lattice(dims, precision=prec, beta=3.09, seed=5, start="cold")
        L.gauge_update(1, utype=0, stype=0, eps=0.5)
        out[prec] = L.download()
    d = np.abs(out["fp64"] - out["fp32"]).max(axis=(1, 2))
    assert np.median(d) <= 1e-6 and np.mean(d <= 1e-5) >= 0.99


def test_gauge_update_rejects_bad_arguments():
    L = Lattice((4, 4, 4, 4), precision="fp64")
    for kw in (dict(utype=2), dict(stype=2), dict(utype=0, hits=0), dict(utype=0, eps=float("nan"))):
        with pytest.raises(Su2gError):
            L.gauge_update(1, **{**dict(utype=1, stype=0, eps=0.2, hits=1), **kw})


@pytest.mark.parametrize("utype,stype", [(0, 0), (0, 1), (1, 1)])
def test_chains_agree_with_reference_chains(golden, utype, stype):
    c = next(x for x in golden["metropolis"]["chains"] if (x["utype"], x["stype"]) == (utype, stype))
    L = Lattice(tuple(c["dims"]), precision="fp64", beta=c["beta"], seed=2024 + 7 * utype + stype, start="cold")
    n, therm = 20000, 500
    plaq = []
    for _ in range(n):
        L.gauge_update(1, utype=utype, stype=stype, eps=c["eps"], hits=1)
        plaq.append(L.plaquette())
    m, err, tau = _stats.mean_err(plaq[therm:])
    z = abs(m - c["mean"]) / np.hypot(err, c["err"])
    assert z <= 2.0, (m, err, tau, c["mean"], c["err"], z)
