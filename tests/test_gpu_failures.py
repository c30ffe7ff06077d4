"""Device-side failure detection without a GPU fault: a wait that runs out and a heatbath past its
trial bound are reported as SU2G_EDEVICE at the next synchronising call, the status word is cleared,
and the handle keeps working."""
import numpy as np
import pytest

from masterarbeit_b200 import Lattice
from masterarbeit_b200.su2g import Su2gError

pytestmark = pytest.mark.gpu

SU2G_EDEVICE = -4


def test_bounded_wait_runs_out_and_handle_survives():
    L = Lattice((4, 4, 4, 4), precision="fp32", seed=3, start="haar")
    p0 = L.plaquette()
    with pytest.raises(Su2gError) as e:
        L.selftest_bounded_wait(1 << 12)
    assert e.value.code == SU2G_EDEVICE and "did not complete in time" in str(e.value)
    # reported once, then cleared: the handle keeps working
    assert L.plaquette() == p0
    L.sweep(1, 1, 1)
    assert 0.0 < L.plaquette() < 1.0
    with pytest.raises(Su2gError):
        L.selftest_bounded_wait(0)   # outside the allowed range: refused before any launch


def test_heatbath_trial_bound_is_reported():
    # at beta ~ 1e-30 every Kennedy-Pendleton trial is rejected (delta >> 2): each link stops at
    # the trial bound, keeps its value, and the pass reports it
    L = Lattice((4, 4, 4, 4), precision="fp64", beta=1e-30, seed=5, start="haar")
    U = L.download()
    with pytest.raises(Su2gError) as e:
        L.sweep(1, 1, 0, acc=True)
    assert e.value.code == SU2G_EDEVICE and "Kennedy-Pendleton" in str(e.value)
    assert np.array_equal(L.download(), U)
    L.set_beta(2.5)
    assert 0.9 < L.sweep(1, 1, 0, acc=True) <= 1.0
