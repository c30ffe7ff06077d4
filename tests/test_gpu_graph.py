"""su2g_graph_run (the qcd.c:55-60 update/measure loop as one replayed CUDA graph) against the same
su2g_sweep_plaquette sequence issued call by call: identical fields and plaquette traces (and the
plaquette kernel's value to rounding), the Philox sweep counter carried across calls, and a new
capture whenever the field's buffers (APE ping-pong), beta or the block shape change."""
import numpy as np
import pytest

from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu


def _plain(L, n_blocks, every, n_hb, n_or):
    plaq, acc = [], []
    for _ in range(n_blocks):
        p, a = L.sweep_plaquette(every, n_hb, n_or, acc=True)
        # the sum inside the update passes against the plaquette kernel on the same field
        assert abs(p - L.plaquette()) <= (1e-14 if L.precision == "fp64" else 5e-7) * abs(p)
        plaq.append(p)
        acc.append(a)
    return np.array(plaq), np.array(acc)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("dims,start", [((8, 8, 8, 8), "cold"), ((6, 4, 4, 8), "haar")])
def test_graph_run_equals_plain_sequence(dims, start, prec):
    g = Lattice(dims, precision=prec, beta=3.09, seed=5, start=start)
    p = Lattice(dims, precision=prec, beta=3.09, seed=5, start=start)
    # reuse; a longer trace (new buffer, possibly at the old address); a new block shape
    for shape in ((5, 2, 1, 2), (3, 2, 1, 2), (12, 2, 1, 2), (4, 1, 2, 0)):
        gp, ga = g.graph_run(*shape)
        pp, pa = _plain(p, *shape)
        assert np.array_equal(gp, pp)
        assert np.allclose(ga, pa, rtol=1e-12, atol=0)
        assert np.array_equal(g.download(), p.download())
    # the field's directions move to the other buffer after smearing; beta changes
    for L in (g, p):
        L.ape(1, 0.3, "spatial")
        L.set_beta(2.7)
    gp, ga = g.graph_run(3, 1, 1, 1)
    pp, pa = _plain(p, 3, 1, 1, 1)
    assert np.array_equal(gp, pp)
    assert np.array_equal(g.download(), p.download())
    assert 0.0 < ga.min() and ga.max() <= 1.0


def test_graph_run_arguments():
    L = Lattice((4, 4, 4, 4), precision="fp64")
    with pytest.raises(RuntimeError):
        L.graph_run(2, meas_every=0)
    p, a = L.graph_run(0)
    assert p.size == 0
    L.graph_release()
    p, a = L.graph_run(2, 1, 1, 0)
    assert p.shape == (2,) and np.all(a > 0)
