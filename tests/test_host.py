"""Host-side checks that need no GPU: the C-ABI library builds, loads and exports every symbol the
header declares; the configuration format; the index arithmetic of the kernels."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import build, configio, su2g


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    names = su2g.header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the binding covers the whole header
    assert set(names) <= set(su2g._SIGS), sorted(set(names) - set(su2g._SIGS))


def test_create_without_gpu_fails_loudly():
    import torch  # noqa: F401  (only to learn whether a GPU is visible)
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(su2g.Su2gError, match="no CUDA device|not sm_100"):
        su2g.Lattice((4, 4, 4, 4))


def test_create_rejects_bad_extents():
    lib = su2g.load()
    p = su2g.Params()
    for i, d in enumerate((4, 5, 4, 4)):
        p.dims[i] = d
    h = ctypes.c_void_p()
    assert lib.su2g_create(ctypes.byref(p), ctypes.byref(h)) == -1
    assert b"even" in lib.su2g_last_error(None)


def test_null_handle_is_an_error_not_a_crash():
    lib = su2g.load()
    v = ctypes.c_double()
    assert lib.su2g_plaquette(None, ctypes.byref(v)) == -1
    assert lib.su2g_sweep(None, 1, 1, 0, None) == -1
    assert lib.su2g_sweep_plaquette(None, 1, 1, 0, ctypes.byref(v), None) == -1


@pytest.mark.parametrize("name", ["cfg_4x4x4x4_base.cfg", "cfg_6x4x4x8_base.cfg", "cfg_8x8x8x8_base.cfg"])
def test_config_roundtrip(tmp_path, name):
    dims, plaq, U = configio.read_config(os.path.join(O.GOLDEN, name))
    assert abs(O.plaquette(dims, U) - plaq) <= configio.plaquette_tolerance(np.prod(dims))
    out = tmp_path / "x.cfg"
    configio.write_config(out, dims, U, plaq)
    assert open(out, "rb").read() == open(os.path.join(O.GOLDEN, name), "rb").read()


def test_config_rejects_corrupt_files(tmp_path):
    src = open(os.path.join(O.GOLDEN, "cfg_4x4x4x4_base.cfg"), "rb").read()
    (tmp_path / "trunc.cfg").write_bytes(src[:-8])
    with pytest.raises(configio.ConfigError, match="truncated"):
        configio.read_config(tmp_path / "trunc.cfg")
    bad = bytearray(src)
    bad[4] = 3  # SUN = 3
    (tmp_path / "sun3.cfg").write_bytes(bytes(bad))
    with pytest.raises(configio.ConfigError, match="incompatible"):
        configio.read_config(tmp_path / "sun3.cfg")
    (tmp_path / "long.cfg").write_bytes(src + b"\0")
    with pytest.raises(configio.ConfigError, match="trailing"):
        configio.read_config(tmp_path / "long.cfg")


def test_fastdiv_and_site_decoding(tmp_path):
    """Compile the kernels' host-callable index helpers (su2.cuh) with nvcc and check the fast
    division and checkerboard decoding exhaustively on several lattices."""
    src = tmp_path / "t.cu"
    src.write_text(r'''
#include "su2.cuh"
#include <cstdio>
using namespace su2g;
int main() {
  const uint32_t ds[] = {1u, 2u, 3u, 4u, 6u, 7u, 8u, 10u, 12u, 48u, 2304u, 110592u, 9216u, 884736u, 1000003u};
  for (uint32_t d : ds) {
    FastDiv f = make_fastdiv(d);
    for (uint64_t n = 0; n < (1ull << 22); n += 1) if (fdiv((uint32_t)n, f) != (uint32_t)n / d) { printf("FAIL %u %llu\n", d, (unsigned long long)n); return 1; }
    for (uint64_t n = 0xffffffffull - 5000; n <= 0xffffffffull; ++n) if (fdiv((uint32_t)n, f) != (uint32_t)n / d) { printf("FAIL %u %llu\n", d, (unsigned long long)n); return 1; }
    for (uint64_t n = 1; n < 0xffffffffull; n = n * 3 + 1) if (fdiv((uint32_t)n, f) != (uint32_t)n / d) { printf("FAIL %u %llu\n", d, (unsigned long long)n); return 1; }
  }
  printf("OK\n");
  return 0;
}
''')
    exe = tmp_path / "t"
    subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-I", build.CSRC, str(src), "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)], capture_output=True, text=True).stdout.strip() == "OK"


def test_checkerboard_enumeration_is_a_bijection():
    """The device layout enumerates each parity once via h = n >> 1 (L_z even)."""
    for dims in [(4, 4, 4, 4), (6, 4, 4, 8), (2, 4, 6, 4), (10, 6, 4, 8)]:
        V = int(np.prod(dims))
        n = np.arange(V)
        t, r = np.divmod(n, dims[1] * dims[2] * dims[3])
        x, r = np.divmod(r, dims[2] * dims[3])
        y, z = np.divmod(r, dims[3])
        par = (t + x + y + z) & 1
        for p in (0, 1):
            h = n[par == p] >> 1
            assert np.array_equal(np.sort(h), np.arange(V // 2))


def test_su2meas_argument_and_input_errors(tmp_path):
    """The native measurement driver refuses bad command lines, missing input files and two-point
    functions before it touches a GPU."""
    import subprocess

    driver = os.path.join(O.REPO, "masterarbeit_b200", "_lib", "su2meas")
    if not os.path.exists(driver):
        pytest.skip("su2meas not built")
    assert subprocess.run([driver], capture_output=True).returncode == 2
    assert subprocess.run([driver, "-i", "x", "--qtop", "y", "-d", "4x4x4x4"], capture_output=True).returncode == 2
    r = subprocess.run([driver, "-i", str(tmp_path / "none.in"), "-d", "4x4x4x4"], capture_output=True, text=True)
    assert r.returncode == 1 and "unable to open input file" in r.stderr
    inp = tmp_path / "meas.in"
    inp.write_text("outFileId 1\nodir .\nbeta 3.09\nsconf 1\nfconf 1\neconf 1\nmtopcharge 0\nsmear_tc 0 0.1\n"
                   "mwil 0 6\ntSmear 0 0.5\nrSmear 0 0.5\nmcorrs 1\n")
    r = subprocess.run([driver, "-i", str(inp), "-d", "4x4x4x4"], capture_output=True, text=True)
    assert r.returncode == 1 and "two-point functions" in r.stderr


def test_su2qcd_input_errors(tmp_path):
    """The native qcd driver refuses incomplete input files and existing logs before it touches a GPU."""
    import subprocess

    driver = os.path.join(O.REPO, "masterarbeit_b200", "_lib", "su2qcd")
    if not os.path.exists(driver):
        pytest.skip("su2qcd not built")
    assert subprocess.run([driver], capture_output=True).returncode == 2
    inp = tmp_path / "qcd.in"
    inp.write_text("outFileId 1\noutputDir %s\nstart 0\nbeta 3.09\n" % tmp_path)
    r = subprocess.run([driver, "-i", str(inp), "-d", "4x4x4x4"], capture_output=True, text=True)
    assert r.returncode == 1 and "missing field" in r.stderr
    inp.write_text("outFileId 1\noutputDir %s\nstart 0\nbeta 3.09\nepsilon 0.1\nnconf 2\nntherm 0\nndecorr 1\n"
                   "writeConfFreq 0\nseed 1\n" % tmp_path)
    (tmp_path / "4x4x4x4_SU2_b3.090000_id1.log").write_text("old run\n")
    r = subprocess.run([driver, "-i", str(inp), "-d", "4x4x4x4"], capture_output=True, text=True)
    assert r.returncode == 1 and "overwrite" in r.stderr
