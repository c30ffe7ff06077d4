"""The TMA-tiled FP32 APE_all kernel (csrc/ape_tma.cu, opt-in) against the per-site kernel and the
oracle, on geometries that exercise the y-halo wrap (L_y = rows per CTA, several wraps per tile),
short and long z rows and the 48^4 production size."""
import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(8, 8, 8, 16), (6, 4, 8, 32), (4, 6, 4, 24), (10, 6, 4, 48), (2, 4, 8, 64),
                                  (48, 48, 48, 48)])
def test_tma_ape_matches_generic_and_oracle(dims):
    tma = Lattice(dims, precision="fp32", seed=17, start="haar")
    gen = Lattice(dims, precision="fp32", seed=17, start="haar")
    tma.set_kernel_variant("ape", 1)
    gen.set_kernel_variant("ape", 0)
    assert tma.kernel_variant("ape") == 1 and gen.kernel_variant("ape") == 0
    U = tma.download()
    tma.ape(3, 0.5, "all")
    gen.ape(3, 0.5, "all")
    A, B = tma.download(), gen.download()
    # the two kernels associate the staple sums differently: FP32 rounding only, over three steps
    assert np.max(np.abs(A - B)) <= 5e-6
    if np.prod(dims) <= 40000:
        assert np.max(np.abs(A - O.ape(dims, U, 3, 0.5, "all"))) <= 5e-6
    # smearing keeps working on the TMA path after other kernels ran (ping-pong of directions)
    tma.sweep(1, 1, 1)
    gen.upload(tma.download())
    tma.ape(2, 0.4, "all")
    gen.ape(2, 0.4, "all")
    assert np.max(np.abs(tma.download() - gen.download())) <= 5e-6


def test_tma_not_used_where_it_does_not_apply():
    for dims, prec in (((8, 8, 8, 8), "fp32"), ((8, 8, 8, 16), "fp64")):   # too few threads / FP64 tiles too big
        L = Lattice(dims, precision=prec)
        L.set_kernel_variant("ape", 1)
        assert L.kernel_variant("ape") == 0
