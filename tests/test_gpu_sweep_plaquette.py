"""su2g_sweep_plaquette: the sweep with the plaquette summed inside its last sub-sweep's update
passes.  The summed value is the plaquette of the field the call leaves (against the plaquette
kernel on that field), for heatbath-only, overrelaxation-last and multi-sweep calls; the field is
that of su2g_sweep from the same start to rounding (the fused passes are separately compiled
kernels, whose multiply-adds may round differently in the last bit)."""
import numpy as np
import pytest

from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-14, "fp32": 5e-7}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("dims,start", [((8, 8, 8, 8), "cold"), ((6, 4, 4, 8), "haar"), ((2, 4, 6, 4), "haar"),
                                        ((48, 48, 48, 48), "haar")])
def test_fused_plaquette_is_the_plaquette_of_the_field_it_leaves(dims, start, prec):
    shapes = ((1, 1, 0), (2, 1, 2), (1, 0, 1), (3, 2, 1)) if np.prod(dims) < 1e6 else ((1, 1, 0), (1, 1, 4))
    a = Lattice(dims, precision=prec, beta=3.09, seed=11, start=start)
    b = Lattice(dims, precision=prec, beta=3.09, seed=11, start=start)
    for shape in shapes:
        b.upload(a.download())
        b.set_sweep_counter(a.info()["hb_sweeps"])
        pa, acc_a = a.sweep_plaquette(*shape, acc=True)
        ref = a.plaquette()
        assert abs(pa - ref) <= TOL[prec] * abs(ref), (shape, pa, ref)
        # the same sweeps through su2g_sweep: same Philox draws, fields equal to rounding.  An FP32
        # accept/reject decision at a last-bit boundary may flip (about once in 1e7 trials) and then
        # moves that link entirely, so FP32 bounds the fraction of links that differ.
        acc_b = b.sweep(*shape, acc=True)
        d = np.abs(a.download() - b.download())
        if prec == "fp64":
            assert np.max(d) <= 1e-9, shape
            assert abs(acc_a - acc_b) <= 1e-12 * acc_b
        else:
            assert np.mean(d > 1e-4) <= 1e-3, shape
            assert abs(acc_a - acc_b) <= 1e-3 * acc_b
    a.close()
    b.close()


def test_no_sub_sweep_runs_the_plaquette_kernel():
    L = Lattice((6, 4, 4, 8), precision="fp64", seed=3, start="haar")
    p0 = L.plaquette()
    assert L.sweep_plaquette(0, 1, 0) == p0
    assert L.sweep_plaquette(2, 0, 0) == p0


def test_fused_plaquette_after_smearing_buffers_moved():
    """After APE the directions live in the other buffer; the fused sum reads the handle's pointers."""
    L = Lattice((8, 8, 8, 8), precision="fp64", seed=2, start="haar")
    L.ape(1, 0.5, "spatial")
    p = L.sweep_plaquette(1, 1, 1)
    assert abs(p - L.plaquette()) <= 1e-14


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_wide_reduction_is_reproducible(prec):
    """At 32^4 the fused sweep's 49152 per-warp partials and the plaquette kernel's 8192 CTA
    partials go through the multi-CTA final reduction (a CTA result per chunk, combined in index
    order by whichever CTA arrives last): repeated and independent runs agree bit for bit."""
    dims = (32, 32, 32, 32)
    a = Lattice(dims, precision=prec, beta=3.09, seed=21, start="haar")
    b = Lattice(dims, precision=prec, beta=3.09, seed=21, start="haar")
    pa = [a.sweep_plaquette(1, 1, 1) for _ in range(3)]
    pb = [b.sweep_plaquette(1, 1, 1) for _ in range(3)]
    assert pa == pb
    assert len({a.plaquette() for _ in range(5)}) == 1
    assert a.plaquette() == b.plaquette()
