"""su2g_ape_inplace_noalloc: APE smearing for callers that may not allocate device memory.

Such a caller owns its field in device memory it got elsewhere (memory handed out by another
component or a fixed budget) and cannot create a su2g handle, because su2g_create allocates.  The
entry point smears the caller's buffer in place and keeps the intermediate level in a static
device array.  This file is collected last on purpose; it checks, through the C ABI, that two calls
in a row give what the handle path (su2g_upload_aos_f64 + su2g_ape + su2g_download_aos_f64) gives,
at the FP64 tolerance of the other APE tests, and that oversized lattices are refused.
"""
import ctypes

import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice, su2g

pytestmark = pytest.mark.gpu

_CUDART = "/usr/local/cuda/lib64/libcudart.so"


class DeviceBuffer:
    """Device memory owned by the test (the caller), from the CUDA runtime directly."""

    def __init__(self, nbytes):
        self.rt = ctypes.CDLL(_CUDART)
        self.rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
        self.rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        self.rt.cudaFree.argtypes = [ctypes.c_void_p]
        self.ptr = ctypes.c_void_p()
        assert self.rt.cudaMalloc(ctypes.byref(self.ptr), nbytes) == 0
        self.nbytes = nbytes

    def upload(self, a):
        assert self.rt.cudaMemcpy(self.ptr, a.ctypes.data, self.nbytes, 1) == 0   # host to device

    def download(self, a):
        assert self.rt.cudaDeviceSynchronize() == 0
        assert self.rt.cudaMemcpy(a.ctypes.data, self.ptr, self.nbytes, 2) == 0   # device to host

    def free(self):
        self.rt.cudaFree(self.ptr)


def test_ape_without_allocation_matches_handle_path():
    lib = su2g.load()
    dims, _, U = O.golden_config("cfg_8x8x8x8_base.cfg")
    cdims = (ctypes.c_int32 * 4)(*dims)
    buf = DeviceBuffer(U.nbytes)
    buf.upload(np.ascontiguousarray(U))
    ref = Lattice(dims, precision="fp64")
    ref.upload(U)
    got = np.empty_like(U)
    # two calls in a row on the same buffer: an odd number of steps (result copied back from the
    # static array) and then a spatial smearing (directions left alone must stay intact)
    for ns, alpha, mode in ((3, 0.5, "all"), (2, 0.4, "spatial")):
        rc = lib.su2g_ape_inplace_noalloc(buf.ptr, cdims, ns, alpha, su2g.APE[mode], None)
        assert rc == 0, lib.su2g_last_error(None)
        ref.ape(ns, alpha, mode)
        buf.download(got)
        assert np.max(np.abs(got - ref.download())) <= 1e-13
    buf.free()
    ref.close()


def test_ape_without_allocation_temporal_on_non_cubic_lattice():
    """Temporal smearing on 6x4x4x8 (other strides, only the t links change): the handle path and the
    reference's own smearing_APE_temporal output agree with the no-allocation entry point."""
    lib = su2g.load()
    g = O.golden()["lattices"]["6x4x4x8"]
    spec = g["ape"]["temporal"]
    dims, _, U = O.golden_config(g["base"])
    _, _, want = O.golden_config(spec["cfg"])
    cdims = (ctypes.c_int32 * 4)(*dims)
    buf = DeviceBuffer(U.nbytes)
    buf.upload(np.ascontiguousarray(U))
    ref = Lattice(dims, precision="fp64")
    ref.upload(U)
    got = np.empty_like(U)
    rc = lib.su2g_ape_inplace_noalloc(buf.ptr, cdims, spec["ns"], spec["alpha"], su2g.APE["temporal"], None)
    assert rc == 0, lib.su2g_last_error(None)
    ref.ape(spec["ns"], spec["alpha"], "temporal")
    buf.download(got)
    assert np.max(np.abs(got - ref.download())) <= 1e-13
    assert np.max(np.abs(got - want)) <= 1e-13
    buf.free()
    ref.close()


def test_ape_without_allocation_rejects_bad_pointers():
    """A field pointer that is not 16-byte aligned, or not device memory, is refused before any launch."""
    lib = su2g.load()
    dims = (ctypes.c_int32 * 4)(4, 4, 4, 4)
    nbytes = 4 ** 4 * 16 * 8
    buf = DeviceBuffer(nbytes + 16)
    off8 = ctypes.c_void_p(buf.ptr.value + 8)
    assert lib.su2g_ape_inplace_noalloc(off8, dims, 1, 0.5, 0, None) == -1
    assert b"not 16-byte aligned" in lib.su2g_last_error(None)
    host = np.zeros(4 ** 4 * 16 + 2, dtype=np.float64)
    hp = host.ctypes.data + (-host.ctypes.data) % 16
    assert lib.su2g_ape_inplace_noalloc(ctypes.c_void_p(hp), dims, 1, 0.5, 0, None) == -1
    assert b"not device memory" in lib.su2g_last_error(None)
    # the device is still usable: a correct call on the aligned buffer goes through
    assert lib.su2g_ape_inplace_noalloc(buf.ptr, dims, 0, 0.5, 0, None) == 0
    assert buf.rt.cudaDeviceSynchronize() == 0
    buf.free()


def test_ape_without_allocation_rejects_oversized_lattice():
    lib = su2g.load()
    buf = DeviceBuffer(64)
    big = (ctypes.c_int32 * 4)(26, 26, 26, 26)   # 456976 sites > 393216
    assert lib.su2g_ape_inplace_noalloc(buf.ptr, big, 1, 0.5, 0, None) == -1
    assert b"exceeds the static scratch" in lib.su2g_last_error(None)
    buf.free()
