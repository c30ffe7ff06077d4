"""B200-native (sm_100a) SU(2) pure-gauge lattice hot path.

The product is libsu2g.so (CUDA C++ kernels behind the C ABI in include/su2g.h); this
package builds it in-tree (build.py), binds it (su2g.py) and reads/writes the reference's
configuration format (configio.py).  The C shim that gives the reference's own drivers their
function names is shim/ref_shim.c.
"""
from .su2g import Lattice, Su2gError, load, header_functions  # noqa: F401
from .configio import read_config, write_config  # noqa: F401

__all__ = ["Lattice", "Su2gError", "load", "header_functions", "read_config", "write_config"]
