"""The largest lattice of the thesis runs, 96^4 (84.9 M sites, 5.4 GB of FP32 links), through the
update, smearing and measurement kernels.  Checks are size-independent properties: a cold start
has plaquette 1; an overrelaxation sweep keeps the action, hence the plaquette; heatbath sweeps
from a cold start at beta = 3.09 move the plaquette below 1 towards its equilibrium ~0.7326;
smeared loops and the charge are finite and in range."""
import math

import numpy as np
import pytest

from masterarbeit_b200 import Lattice

pytestmark = pytest.mark.gpu


def test_96x96x96x96_fp32():
    L = Lattice((96, 96, 96, 96), precision="fp32", beta=3.09, seed=12, start="cold")
    assert abs(L.plaquette() - 1.0) <= 1e-6
    acc = L.sweep(3, 1, 0, acc=True)
    p = L.plaquette()
    assert 0.95 < acc <= 1.0 and 0.70 < p < 0.99
    L.sweep(1, 0, 1)   # one overrelaxation sweep
    assert abs(L.plaquette() - p) <= 2e-5
    L.ape(2, 0.5, "spatial")
    w = L.wilson([1, 2, 9], [1, 2, 9])
    assert all(math.isfinite(x) for x in w) and 0 < w[0] <= 1 and abs(w[2]) <= w[0]
    q, sabs = L.qtop(with_abs=True)
    assert math.isfinite(q) and sabs > 0
    L.close()
