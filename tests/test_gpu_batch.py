"""Batched replicas: one launch per pass over many lattices of mixed extents, beta, seeds and starts,
with the sweep + measurement block replayed from a CUDA graph."""
import time

import numpy as np
import pytest

from masterarbeit_b200 import Lattice
from masterarbeit_b200.su2g import Batch

pytestmark = pytest.mark.gpu

REPS = [
    {"dims": (4, 4, 4, 4), "beta": 2.5, "seed": 11, "replica": 0, "start": "cold"},
    {"dims": (6, 4, 4, 8), "beta": 3.0, "seed": 12, "replica": 1, "start": "haar"},
    {"dims": (8, 8, 8, 8), "beta": 2.2, "seed": 13, "replica": 2, "start": "ref"},
    {"dims": (10, 10, 10, 10), "beta": 3.2, "seed": 14, "replica": 3, "start": "haar"},
]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_equals_single_lattices(precision):
    """The replayed graph of per-pass launches draws the Philox streams of single handles: plaquette traces
    agree to 1e-14, FP32 fields bit for bit, FP64 fields to rounding (the FP64 heatbath kernels of the
    batch and of a handle are compiled separately; a last-bit difference of a staple, amplified through
    three sweeps, stays below 1e-9)."""
    B = Batch(REPS, precision=precision)
    B.configure("graph", 256)
    assert B.config() == ("graph", 256)
    trace, _ = B.run(3, n_hb=1, n_or=2, meas_every=1)
    assert trace.shape == (3, len(REPS))
    for i, r in enumerate(REPS):
        L = Lattice(r["dims"], precision=precision, beta=r["beta"], seed=r["seed"], start=r["start"],
                    replica=r["replica"])
        for s in range(3):
            L.sweep(1, 1, 2)
            assert abs(trace[s, i] - L.plaquette()) <= 1e-14, (i, s)
        if precision == "fp32":
            assert np.array_equal(B.download(i), L.download()), i
        else:
            assert np.max(np.abs(B.download(i) - L.download())) <= 1e-9, i
        L.close()
    # a second run continues the same chains (Philox sweep index kept on the device)
    trace2, _ = B.run(2, n_hb=1, n_or=2, meas_every=2)
    L = Lattice(REPS[2]["dims"], precision=precision, beta=REPS[2]["beta"], seed=REPS[2]["seed"],
                start=REPS[2]["start"], replica=2)
    L.sweep(5, 1, 2)
    # after five sweeps an FP64 last-bit difference has grown (measured 2.4e-12 on B200)
    assert abs(trace2[0, 2] - L.plaquette()) <= (1e-14 if precision == "fp32" else 1e-10)
    B.close()


@pytest.mark.parametrize("precision,block,sweeps,tol_field,tol_trace",
                         [("fp64", 128, 1, 1e-11, 1e-13), ("fp64", 256, 1, 1e-11, 1e-13),
                          ("fp32", 128, 1, 2e-4, 1e-6), ("fp32", 256, 1, 2e-4, 1e-6)])
def test_persistent_batch_agrees_with_graph_batch(precision, block, sweeps, tol_field, tol_trace):
    """The persistent form (one cooperative launch, links tiled over all replicas so that the 4^4 and
    6x4x4x8 replicas, 128 and 384 links a pass, share CTAs) draws the same Philox streams as the graph
    form; compiled as a separate kernel, its multiply-adds may round differently in the last bit, so
    fields and traces agree to rounding after one sweep (where an accept/reject decision that a
    last-bit difference flips is unlikely).  The heatbath amplifies a last-bit difference of a staple:
    measured on B200, FP64 links differed by up to 1.2e-10 after three sweeps (beta = 2.2) and FP32
    links by up to 2.2e-5 after one, while the plaquette traces agreed to 1e-14 and 1e-8."""
    out = {}
    for mode, blk in (("graph", 256), ("persistent", block)):
        B = Batch(REPS, precision=precision)
        B.configure(mode, blk)
        trace, _ = B.run(sweeps, n_hb=1, n_or=2, meas_every=1)
        out[mode] = (trace, [B.download(i) for i in range(len(REPS))])
        # a second run continues the chains from the device counters in both forms
        t2, _ = B.run(2, n_hb=1, n_or=1, meas_every=2)
        out[mode] += (t2,)
        B.close()
    tg, fg, t2g = out["graph"]
    tp, fp, t2p = out["persistent"]
    assert np.max(np.abs(tg - tp)) <= tol_trace
    assert np.max(np.abs(t2g - t2p)) <= 10 * tol_trace
    for i in range(len(REPS)):
        assert np.max(np.abs(fg[i] - fp[i])) <= tol_field, i


def test_autotune_leaves_the_chains_untouched():
    B = Batch(REPS, precision="fp32")
    B.run(2, 1, 1, 0)
    before = [B.download(i) for i in range(len(REPS))]
    block = B.autotune(1, 4)
    assert block in (64, 128, 256)
    mode, blk = B.config()
    assert blk == block and mode in ("graph", "persistent")
    print("autotuned:", mode, block)
    for i in range(len(REPS)):
        assert np.array_equal(B.download(i), before[i])
    t1, _ = B.run(1, 1, 1, 1)
    A = Batch(REPS, precision="fp32")
    A.run(2, 1, 1, 0)
    t2, _ = A.run(1, 1, 1, 1)
    assert np.array_equal(t1, t2)


def test_upload_download_roundtrip():
    B = Batch(REPS[:2], precision="fp64")
    U = B.download(1)
    B.upload(0, B.download(0))
    B.upload(1, U)
    assert np.array_equal(B.download(1), U)


def test_batched_beats_sequential_handles():
    """64 replicas of 12^4 (beta in [2.2, 3.2], distinct seeds, alternating starts): one graph replay per
    sweep for all replicas against 64 single handles swept one after another."""
    rng = np.random.default_rng(5)
    reps = [{"dims": (12, 12, 12, 12), "beta": float(rng.uniform(2.2, 3.2)), "seed": 1000 + i, "replica": i,
             "start": "haar" if i % 2 else "cold"} for i in range(64)]
    B = Batch(reps, precision="fp32")
    B.autotune(1, 4)
    B.run(5, 1, 4, 1)
    nb = 50
    _, ms_b = B.run(nb, 1, 4, 1)
    Ls = [Lattice(r["dims"], precision="fp32", beta=r["beta"], seed=r["seed"], start=r["start"], replica=r["replica"])
          for r in reps]
    for L in Ls:
        L.sweep(1, 1, 4)
        L.plaquette()
    ns = 5
    t0 = time.perf_counter()
    for _ in range(ns):
        for L in Ls:
            L.sweep(1, 1, 4)
            L.plaquette()
    t_seq = (time.perf_counter() - t0) / ns
    t_bat = ms_b / 1e3 / nb
    print(f"64 x 12^4: batched {t_bat * 1e3:.3f} ms/sweep, sequential {t_seq * 1e3:.3f} ms/sweep, "
          f"speed-up {t_seq / t_bat:.1f}x")
    assert t_seq / t_bat > 2.0


def test_persistent_barrier_wait_is_bounded():
    """The grid-wide barrier of the persistent form, made to wait for a CTA that does not exist, gives up
    after its limit and reports it (SU2G_EDEVICE) without a fault; the batch keeps working."""
    from masterarbeit_b200.su2g import Su2gError
    B = Batch(REPS[:2], precision="fp32")
    B.selftest_grid_barrier(missing=0)
    with pytest.raises(Su2gError) as e:
        B.selftest_grid_barrier(missing=1, wait_cycles=50_000_000)
    assert e.value.code == -4 and b"grid-wide barrier" in B.lib.su2g_batch_last_error(B.h)
    B.configure("persistent", 128)
    trace, _ = B.run(2, 1, 1, 1)
    assert np.all(np.isfinite(trace))
    B.close()
