"""Configuration files streamed between the file and the device field (su2g_read_config,
su2g_write_config, su2g_read_config_reflect) against the reference's files and the oracle:
the reference's writeConfig output reads back exactly, a written file is byte-identical to the
same field written by the host-side writer, files of several chunks round-trip, the reflection
start equals the reference's readConfigForThermalisation byte for byte, and malformed files are
refused with SU2G_EFILE as readConfig refuses them."""
import hashlib
import os
import shutil
import struct

import numpy as np
import pytest

import _oracle as O
from masterarbeit_b200 import Lattice
from masterarbeit_b200.configio import plaquette_tolerance, read_config, write_config
from masterarbeit_b200.su2g import Su2gError

pytestmark = pytest.mark.gpu

SU2G_EFILE = -6
BASES = ["4x4x4x4", "6x4x4x8", "8x8x8x8"]


def _path(name):
    return os.path.join(O.GOLDEN, name)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("lat", BASES)
def test_read_reference_file(golden, lat, prec):
    dims, plaq0, U = read_config(_path(f"cfg_{lat}_base.cfg"))
    L = Lattice(dims, precision=prec)
    pf, p = L.read_config(_path(f"cfg_{lat}_base.cfg"))
    assert pf == plaq0
    got = L.download()
    if prec == "fp64":
        assert np.array_equal(got, U)
        assert abs(p - golden["lattices"][lat]["plaq"]) <= plaquette_tolerance(np.prod(dims))
    else:
        assert np.array_equal(got, U.astype(np.float32).astype(np.float64))
        assert abs(p - plaq0) <= 1e-5


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_write_matches_host_writer(tmp_path, prec):
    dims = (6, 4, 4, 8)
    L = Lattice(dims, precision=prec, seed=41, start="haar")
    L.sweep(2, 1, 1)
    p = L.write_config(str(tmp_path / "dev.cfg"))
    assert p == L.plaquette()
    write_config(str(tmp_path / "host.cfg"), dims, L.download(), p)
    assert (tmp_path / "dev.cfg").read_bytes() == (tmp_path / "host.cfg").read_bytes()
    M = Lattice(dims, precision=prec)
    pf, q = M.read_config(str(tmp_path / "dev.cfg"))
    assert pf == p and np.array_equal(M.download(), L.download())


def test_multi_chunk_round_trip(tmp_path):
    dims = (48, 40, 40, 32)   # 2,457,600 sites: several staging chunks and a partial last one
    L = Lattice(dims, precision="fp64", seed=9, start="haar")
    f = str(tmp_path / "big.cfg")
    p = L.write_config(f)
    assert os.path.getsize(f) == 32 + 128 * int(np.prod(dims))
    M = Lattice(dims, precision="fp64", seed=1, start="cold")
    pf, q = M.read_config(f)
    assert pf == p and abs(q - p) <= plaquette_tolerance(np.prod(dims))
    assert np.array_equal(M.download(), L.download())
    os.remove(f)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("big", ["8x8x8x8", "12x8x8x16"])
def test_reflection_matches_reference(golden, big, prec):
    g = golden["reflect"][big]
    dims = tuple(int(x) for x in big.split("x"))
    sdims, plaq0, small = read_config(_path(g["small"]))
    L = Lattice(dims, precision=prec)
    pf, p = L.read_config_reflect(_path(g["small"]))
    assert pf == plaq0
    got = L.download()
    ref = O.reflect(dims, small)
    if prec == "fp64":
        assert np.array_equal(got, ref)
        assert hashlib.sha256(got.astype("<f8").tobytes()).hexdigest() == g["payload_sha256"]
        assert abs(p - g["plaq"]) <= plaquette_tolerance(np.prod(dims))
    else:
        assert np.array_equal(got, ref.astype(np.float32).astype(np.float64))


def test_malformed_files_are_refused(tmp_path):
    src = _path("cfg_4x4x4x4_base.cfg")
    raw = open(src, "rb").read()
    L = Lattice((4, 4, 4, 4), precision="fp64")
    cases = {
        "missing": None,
        "truncated": raw[:-128],
        "short_header": raw[:20],
        "su3": struct.pack("<2i", 4, 3) + raw[8:],
        "plaquette": raw[:24] + struct.pack("<d", struct.unpack("<d", raw[24:32])[0] + 1e-9) + raw[32:],
    }
    for name, data in cases.items():
        f = tmp_path / f"{name}.cfg"
        if data is not None:
            f.write_bytes(data)
        with pytest.raises(Su2gError) as e:
            L.read_config(str(f))
        assert e.value.code == SU2G_EFILE, name
    wrong = Lattice((6, 4, 4, 8), precision="fp64")
    with pytest.raises(Su2gError) as e:
        wrong.read_config(src)
    assert e.value.code == SU2G_EFILE and "incompatible lattice size" in str(e.value)
    with pytest.raises(Su2gError) as e:   # the reflection wants half the extents
        wrong.read_config_reflect(src)
    assert e.value.code == SU2G_EFILE
    shutil.copyfile(src, tmp_path / "ok.cfg")
    assert L.read_config(str(tmp_path / "ok.cfg"))[0] == struct.unpack("<d", raw[24:32])[0]
    with pytest.raises(Su2gError) as e:
        L.write_config(str(tmp_path / "no_such_dir" / "x.cfg"))
    assert e.value.code == SU2G_EFILE
