"""su2g_measure -- one configuration's measurement of the meas / qtop drivers as one replayed CUDA
graph -- against the same steps issued call by call (su2g_ape, su2g_qtop, su2g_wilson on the
handle's own field) and against the reference's charges: identical results, the handle's field
left unchanged, the graph replayed on a new configuration and captured again for a new spec."""
import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice
from masterarbeit_b200.su2g import Su2gError

pytestmark = pytest.mark.gpu

R = [1, 2, 3, 1, 2, 3, 4]
T = [1, 1, 2, 3, 3, 3, 2]


def _plain(dims, U, prec, q_ape, alpha_q, ns_t, alpha_t, ns_s, alpha_s):
    L = Lattice(dims, precision=prec)
    L.upload(U)
    qs, done = [], 0
    for n in q_ape:
        L.ape(n - done, alpha_q, "all")
        done = n
        qs.append(L.qtop())
    L.upload(U)
    L.ape(ns_t, alpha_t, "temporal")
    L.ape(ns_s, alpha_s, "spatial")
    return np.array(qs), np.array(L.wilson(R, T))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("lat", ["6x4x4x8", "8x8x8x8"])
def test_measure_equals_call_by_call(golden, lat, prec):
    g = golden["lattices"][lat]
    dims, _, U = O.golden_config(g["base"])
    L = Lattice(dims, precision=prec)
    L.upload(U)
    spec = dict(q_ape=[0, 1, 5], alpha_q=0.1, ns_t=1, alpha_t=0.4, ns_s=3, alpha_s=0.5)
    q, w = L.measure(R=R, T=T, **spec)
    assert np.array_equal(L.download(), U if prec == "fp64" else U.astype(np.float32).astype(np.float64))
    qp, wp = _plain(dims, U, prec, **spec)
    assert np.array_equal(q, qp) and np.array_equal(w, wp)
    # the reference's charges after 0, 1, 5 APE_all steps at alpha 0.1 (topologicalcharge.c)
    ref = next(r for r in g["qtop"] if r["alpha"] == 0.1)
    tol = 1e-12 if prec == "fp64" else 2e-5
    L2 = Lattice(dims, precision=prec)
    L2.upload(U)
    sabs = L2.qtop(with_abs=True)[1]
    for qi, qr in zip(q, ref["Q"]):
        assert abs(qi - qr) <= tol * max(sabs, 1.0)
    # replay on another configuration, then a new spec (a new capture)
    V = O.ape(dims, U, 2, 0.3, "all")
    L.upload(V)
    q2, w2 = L.measure(R=R, T=T, **spec)
    qp2, wp2 = _plain(dims, V, prec, **spec)
    assert np.array_equal(q2, qp2) and np.array_equal(w2, wp2)
    spec3 = dict(q_ape=[2, 3], alpha_q=0.5, ns_t=0, alpha_t=0.0, ns_s=1, alpha_s=0.25)
    q3, w3 = L.measure(R=R, T=T, **spec3)
    qp3, wp3 = _plain(dims, V, prec, **spec3)
    assert np.array_equal(q3, qp3) and np.array_equal(w3, wp3)
    # the field's own buffers move after smearing it in place; the graph follows them
    L.ape(1, 0.2, "all")
    W1 = L.download()
    q4, w4 = L.measure(R=R, T=T, **spec3)
    qp4, wp4 = _plain(dims, W1, prec, **spec3)
    assert np.array_equal(q4, qp4) and np.array_equal(w4, wp4)
    L.measure_release()
    q5, _ = L.measure(q_ape=[0], alpha_q=0.1)
    assert q5[0] == L.qtop()


def test_measure_rejects_bad_specs():
    L = Lattice((4, 4, 4, 8), precision="fp64")
    with pytest.raises(Su2gError):
        L.measure(q_ape=[3, 1], alpha_q=0.1)
    with pytest.raises(Su2gError):
        L.measure(R=[1], T=[4])   # T > L_t - 1
    with pytest.raises(Su2gError):
        L.measure(R=[0], T=[1])
    q, w = L.measure()
    assert q.size == 0 and w.size == 0
