#!/usr/bin/env python3
"""Time the CPU oracle's heatbath on a bounded slice of a lattice (ORACLE / TEST INFRASTRUCTURE).

Used by bench.py's CPU-baseline leg only when the reference itself was not compiled
(oracle/_ref missing): the port's restatement of localHeatbathUpdate
(LGT_Code/modules/update/heatbath.c:124-149) then stands in for it.
usage: port_bench.py T,X,Y,Z seed beta nsites reps   -> lines "RESULT hb_s rep n seconds acc"
"""
import ctypes
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    dims = [int(x) for x in sys.argv[1].split(",")]
    seed, beta, nsites, reps = int(sys.argv[2]), float(sys.argv[3]), int(sys.argv[4]), int(sys.argv[5])
    lib_path = os.path.join(HERE, "_build", "libsu2oracle.so")
    if not os.path.exists(lib_path):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    lib = ctypes.CDLL(lib_path)
    DP = ctypes.POINTER(ctypes.c_double)
    d = (ctypes.c_int * 4)(*dims)
    vol = int(np.prod(dims))
    U = np.empty((vol, 4, 4))
    lib.su2o_start.argtypes = [ctypes.POINTER(ctypes.c_int), DP, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32]
    lib.su2o_hb_slice.argtypes = [ctypes.POINTER(ctypes.c_int), DP, ctypes.c_double, ctypes.c_uint64,
                                  ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, DP]
    lib.su2o_start(d, U.ctypes.data_as(DP), 2, seed, 0)
    nsites = min(nsites, vol)
    for r in range(reps):
        acc = ctypes.c_double()
        t0 = time.perf_counter()
        lib.su2o_hb_slice(d, U.ctypes.data_as(DP), beta, seed, r, 0, nsites, ctypes.byref(acc))
        t = time.perf_counter() - t0
        print(f"RESULT hb_s {r} {nsites * 4} {t:.9f} {acc.value / (nsites * 4):.6f}", flush=True)


if __name__ == "__main__":
    main()
