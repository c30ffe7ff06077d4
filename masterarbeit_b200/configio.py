"""Configuration files in the reference's binary format.

Format (writeConfig / readConfig, LGT_Code/modules/io/config_IO.c:40-117, :537-621):
  int32 DIM (=4), int32 SUN (=2), int32 L[4] (T, X, Y, Z), float64 plaquette,
  then V x 4 x 4 float64: per site (lexicographic), per direction (0 = t), c0..c3.
Files are little-endian (the reference byte-swaps on big-endian hosts).  readConfig checks the
stored plaquette against a recomputed one within sqrt(6V) * DBL_EPSILON (config_IO.c:611-614).
"""
import struct

import numpy as np

HEADER = struct.Struct("<2i4id")


class ConfigError(ValueError):
    pass


def read_config(path):
    """Return (dims, stored_plaquette, links[V, 4, 4])."""
    with open(path, "rb") as f:
        head = f.read(HEADER.size)
        if len(head) != HEADER.size:
            raise ConfigError(f"{path}: truncated header")
        dim, sun, lt, lx, ly, lz, plaq = HEADER.unpack(head)
        if dim != 4 or sun != 2:
            raise ConfigError(f"{path}: incompatible parameters DIM={dim} SUN={sun}")
        dims = (lt, lx, ly, lz)
        if min(dims) < 2 or any(d % 2 for d in dims):
            raise ConfigError(f"{path}: bad lattice extents {dims}")
        vol = lt * lx * ly * lz
        body = np.fromfile(f, dtype="<f8", count=vol * 16)
        if body.size != vol * 16:
            raise ConfigError(f"{path}: truncated body ({body.size} of {vol * 16} doubles)")
        if f.read(1):
            raise ConfigError(f"{path}: trailing bytes after the body")
    return dims, plaq, body.astype(np.float64).reshape(vol, 4, 4)


def write_config(path, dims, links, plaquette):
    dims = tuple(int(d) for d in dims)
    links = np.ascontiguousarray(links, dtype="<f8").reshape(-1)
    if links.size != 16 * int(np.prod(dims)):
        raise ConfigError("link array does not match the lattice extents")
    with open(path, "wb") as f:
        f.write(HEADER.pack(4, 2, *dims, float(plaquette)))
        links.tofile(f)


def plaquette_tolerance(volume):
    """readConfig's acceptance bound |P - P0| <= sqrt(6 V) DBL_EPSILON (config_IO.c:612)."""
    return float(np.sqrt(6.0 * volume) * np.finfo(np.float64).eps)
